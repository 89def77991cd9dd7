// scan_sort.cuh -- device-wide exclusive scan and a stable LSD radix sort of
// 64-bit keys with an int payload, on preallocated buffers (no allocation per
// call, unlike the reference's thrust::sort_by_key, lbvh.cu:1473-1474).
#pragma once
#include "common.cuh"

namespace admm {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048

// Block-local exclusive scan of kScanTile ints (in place in registers).
ADMM_DEV int block_exclusive_scan(int v, int* sh_warp) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) sh_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        int w = lane < nw ? sh_warp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < nw) sh_warp[lane] = wi - w;  // exclusive warp offsets
    }
    __syncthreads();
    const int r = inc - v + sh_warp[wid];
    __syncthreads();
    return r;
}

// Phase 1: per-tile exclusive scan in place (out) and tile totals.  FLAGS
// scans (in[i] != 0) instead of in[i].
template <bool FLAGS>
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int* __restrict__ in, int* __restrict__ out,
                                                            int n, int* __restrict__ tile_sums) {
    ADMM_PDL_PROLOGUE();
    __shared__ int sh[32];
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    int v[kScanItems];
    int t = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        if (FLAGS) v[k] = v[k] != 0;
        t += v[k];
    }
    const int off = block_exclusive_scan(t, sh);
    int run = off;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == blockDim.x - 1) tile_sums[blockIdx.x] = run;
}

// Phase 2: one block scans the tile totals (any count, in chunks with carry);
// total written to *total (may be NULL) and tile_sums becomes exclusive.
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int* __restrict__ tile_sums, int ntiles,
                                                           int* __restrict__ total) {
    ADMM_PDL_PROLOGUE();
    __shared__ int sh[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ntiles; base += kScanThreads) {
        const int i = base + threadIdx.x;
        const int v = i < ntiles ? tile_sums[i] : 0;
        const int ex = block_exclusive_scan(v, sh);
        const int c = carry;
        if (i < ntiles) tile_sums[i] = ex + c;
        __syncthreads();
        if (threadIdx.x == kScanThreads - 1) carry = c + ex + v;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

// Phase 3: add tile offsets.
__global__ void __launch_bounds__(kScanThreads) k_scan_add(int* __restrict__ out, int n,
                                                          const int* __restrict__ tile_sums) {
    ADMM_PDL_PROLOGUE();
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    const int add = tile_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (base + k < n) out[base + k] += add;
}

inline int scan_tiles(int n) { return (n + kScanTile - 1) / kScanTile; }

// exclusive scan of n ints: out[i] = sum_{j<i} in[j] (flags: of in[j] != 0);
// *total = sum (device).  tmp needs scan_tiles(n) ints.  in and out may alias.
inline void exclusive_scan(const int* in, int* out, int n, int* tmp, int* total, cudaStream_t st, bool pdl = false,
                           bool flags = false) {
    if (n <= 0) return;
    const int nt = scan_tiles(n);
    if (flags) launch_k(k_scan_tiles<true>, dim3(nt), dim3(kScanThreads), 0, st, pdl, in, out, n, tmp);
    else launch_k(k_scan_tiles<false>, dim3(nt), dim3(kScanThreads), 0, st, pdl, in, out, n, tmp);
    launch_k(k_scan_sums, dim3(1), dim3(kScanThreads), 0, st, pdl, tmp, nt, total);
    launch_k(k_scan_add, dim3(nt), dim3(kScanThreads), 0, st, pdl, out, n, (const int*)tmp);
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort, 8-bit digits.  Each pass: per-tile digit histograms
// (digit-major), an exclusive scan of them, and a stable scatter in which each
// tile ranks its keys with warp match masks and per-warp digit counters.
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortTile = 2048;

__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const unsigned long long* __restrict__ keys, int n,
                                                            int shift, int* __restrict__ hist, int ntiles) {
    ADMM_PDL_PROLOGUE();
    __shared__ int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
        const int k = base + i;
        if (k < n) atomicAdd(&h[(int)((keys[k] >> shift) & 0xffu)], 1);
    }
    __syncthreads();
    hist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const unsigned long long* __restrict__ kin,
                                                               const int* __restrict__ vin,
                                                               unsigned long long* __restrict__ kout,
                                                               int* __restrict__ vout, int n, int shift,
                                                               const int* __restrict__ offs, int ntiles) {
    ADMM_PDL_PROLOGUE();
    __shared__ int run[256];
    __shared__ int wcnt[kSortWarps][256];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    run[threadIdx.x] = offs[threadIdx.x * ntiles + blockIdx.x];
    const int base = blockIdx.x * kSortTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int chunk = 0; chunk < kSortTile; chunk += kSortThreads) {
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        const int k = base + chunk + threadIdx.x;
        const bool ok = k < n;
        unsigned long long key = 0;
        int val = 0, d = 256;
        if (ok) {
            key = kin[k];
            val = vin[k];
            d = (int)((key >> shift) & 0xffu);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & lt);
        if (ok && rank == 0) wcnt[wid][d] = __popc(peers);
        __syncthreads();
        if (ok) {
            int pos = run[d] + rank;
            for (int w = 0; w < wid; w++) pos += wcnt[w][d];
            kout[pos] = key;
            vout[pos] = val;
        }
        __syncthreads();
        int add = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) add += wcnt[w][threadIdx.x];
        run[threadIdx.x] += add;
        __syncthreads();
    }
}

inline int sort_tiles(int n) { return (n + kSortTile - 1) / kSortTile; }

// Sorts (keys, vals) by the low `bits` bits of the keys.  Ping-pongs between
// (keys, vals) and (keys_alt, vals_alt); the result ends in (keys, vals) when
// the number of passes is even, which holds for bits = 64.  hist needs
// 256 * sort_tiles(n) ints, scan_tmp scan_tiles(256 * sort_tiles(n)) ints.
inline void radix_sort(unsigned long long* keys, int* vals, unsigned long long* keys_alt, int* vals_alt, int n,
                       int bits, int* hist, int* scan_tmp, cudaStream_t st, bool pdl = false) {
    if (n <= 1) return;
    const int nt = sort_tiles(n);
    unsigned long long *ki = keys, *ko = keys_alt;
    int *vi = vals, *vo = vals_alt;
    for (int shift = 0; shift < bits; shift += 8) {
        launch_k(k_radix_hist, dim3(nt), dim3(kSortThreads), 0, st, pdl, (const unsigned long long*)ki, n, shift, hist,
                 nt);
        exclusive_scan(hist, hist, 256 * nt, scan_tmp, nullptr, st, pdl);
        launch_k(k_radix_scatter, dim3(nt), dim3(kSortThreads), 0, st, pdl, (const unsigned long long*)ki,
                 (const int*)vi, ko, vo, n, shift, (const int*)hist, nt);
        unsigned long long* tk = ki; ki = ko; ko = tk;
        int* tv = vi; vi = vo; vo = tv;
    }
}

}  // namespace admm
