// gnn.cu -- the learned per-vertex block preconditioner of the PCG global step:
// a 3-layer message-passing network (width 64) over the graph of the global
// matrix A, its loss and gradients, and an Adam update, all on the GPU with
// the project's own kernels.  An addition with no reference
// counterpart; the network and loss are specified in the header of the CPU
// restatement that the tests check these kernels against.
//
// Layout: every activation is a row-major FP32 matrix (rows = vertices or
// directed edges of A's off-diagonal pattern, in CSR order).  Dense layers are
// Z = X W^T + b with W row-major [out][in]; with bf16 set, the forward and
// input-gradient passes use the weights rounded to BF16 (FP32 accumulation),
// the master weights and Adam moments stay FP32.  Weight gradients are per-block
// partial sums reduced in a fixed order, node sums over edges run in CSR order,
// so a training step is deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "admm_b200.h"
#include "umma.cuh"

namespace {

constexpr int kH = 64;        // hidden width
constexpr int kFin = 6;       // node features
constexpr int kFe = 2;        // edge features
constexpr int kEdgeIn = 2 * kH + kFe;
constexpr int kNodeIn = 2 * kH;
constexpr int kOut = 7;       // head: lower-triangular factor of the block (6), warm-start coefficient (1)
constexpr int kRowsPerBlockW = 2048;  // rows per partial of a weight gradient

__device__ __forceinline__ float wval(const float* W, int i, int bf16) {
    const float w = W[i];
    return bf16 ? __bfloat162float(__float2bfloat16_rn(w)) : w;
}

// Z[R x N] = X[R x K] W^T + b;  act: 0 none, 1 Y = relu(Z) into Y, 2 Y = res + relu(Z).
// Block: 4 rows x 64 threads (N <= 64); W and the 4 input rows in shared memory.
__global__ void __launch_bounds__(256) k_dense_fwd(const float* __restrict__ X, int R, int K, const float* __restrict__ W,
                                                   const float* __restrict__ b, int N, float* __restrict__ Z,
                                                   float* __restrict__ Y, const float* __restrict__ res, int act,
                                                   int bf16) {
    extern __shared__ float sm[];
    float* Ws = sm;             // [N * K]
    float* Xs = sm + N * K;     // [4 * K]
    for (int i = threadIdx.x; i < N * K; i += blockDim.x) Ws[i] = wval(W, i, bf16);
    const int r0 = blockIdx.x * 4;
    for (int i = threadIdx.x; i < 4 * K; i += blockDim.x) {
        const int r = r0 + i / K;
        Xs[i] = r < R ? X[(size_t)r * K + i % K] : 0.f;
    }
    __syncthreads();
    const int rl = threadIdx.x / 64, c = threadIdx.x % 64, r = r0 + rl;
    if (c >= N || r >= R) return;
    float acc = b[c];
    const float* xr = Xs + rl * K;
    const float* wr = Ws + c * K;
    for (int k = 0; k < K; k++) acc = fmaf(xr[k], wr[k], acc);
    Z[(size_t)r * N + c] = acc;
    if (act == 1) Y[(size_t)r * N + c] = fmaxf(acc, 0.f);
    else if (act == 2) Y[(size_t)r * N + c] = res[(size_t)r * N + c] + fmaxf(acc, 0.f);
}

// The same layer on the tensor cores (tcgen05, kind::tf32, FP32 accumulation in
// tensor memory) for N = 64 outputs: one CTA of 4 warps per 128 rows.  The
// rows of X and the weights (rounded to BF16 first when bf16 is set) are
// rounded to TF32 and staged in shared memory in the canonical K-major layout,
// K padded with zeros to KP (a multiple of 8); thread 0 issues KP / 8 MMAs of
// 128 x 64 x 8 into 64 TMEM columns and commits them to an mbarrier; each warp
// then reads its 32 rows of the accumulator and applies bias and activation.
// The wait for the MMAs is bounded: a wait that gives up sets err[0] and the
// CTA releases its TMEM and leaves without writing.
constexpr int kTcRows = 128, kTcN = 64;

__global__ void __launch_bounds__(128) k_dense_fwd_tc(const float* __restrict__ X, int R, int K, int KP,
                                                      const float* __restrict__ W, const float* __restrict__ b,
                                                      float* __restrict__ Z, float* __restrict__ Y,
                                                      const float* __restrict__ res, int act, int bf16,
                                                      int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int C = KP / 4;  // 16-byte K chunks per row
    unsigned char* As = tc_smem;
    unsigned char* Bs = tc_smem + (size_t)kTcRows * KP * 4;
    const int row0 = blockIdx.x * kTcRows;
    for (int i = threadIdx.x; i < kTcRows * KP; i += blockDim.x) {
        const int m = i / KP, k = i % KP;
        const float v = (row0 + m < R && k < K) ? X[(size_t)(row0 + m) * K + k] : 0.f;
        *(float*)(As + umma::core_offset(m, k >> 2, C) + (k & 3) * 4) = umma::tf32_round(v);
    }
    for (int i = threadIdx.x; i < kTcN * KP; i += blockDim.x) {
        const int n = i / KP, k = i % KP;
        const float v = k < K ? wval(W, n * K + k, bf16) : 0.f;
        *(float*)(Bs + umma::core_offset(n, k >> 2, C) + (k & 3) * 4) = umma::tf32_round(v);
    }
    umma::fence_operands();
    if (threadIdx.x == 0) umma::mbar_init(&mbar, 1);
    if (threadIdx.x < 32) umma::tmem_alloc(&tmem_base, kTcN);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t td = tmem_base;
    if (threadIdx.x == 0) {
        const uint32_t idesc = umma::idesc_tf32(kTcRows, kTcN);
        const uint32_t a0 = umma::smem_u32(As), b0 = umma::smem_u32(Bs);
        for (int k = 0; k < KP / 8; k++)  // 8 TF32 values of K = two 16-byte chunks per MMA
            umma::mma_tf32(td, umma::smem_desc(a0 + 256u * k, C), umma::smem_desc(b0 + 256u * k, C), idesc, k > 0);
        umma::commit(&mbar);
    }
    bool ok = umma::mbar_wait(&mbar, 0, 1 << 22);
    if (!ok) umma::mbar_wait(&mbar, 0, 1 << 22);  // the MMAs in flight, once more with a bound
    ok = __syncthreads_and(ok) != 0;              // uniform: the TMEM loads below are warp-wide
    umma::fence_after();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = row0 + warp * 32 + lane;
    if (ok) {
        const uint32_t tw = td + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int c0 = 0; c0 < kTcN; c0 += 16) {
            uint32_t r[16];
            umma::tmem_load16(tw + c0, r);
            umma::tmem_wait16(r);
            if (row < R) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int c = c0 + j;
                    const float z = __uint_as_float(r[j]) + b[c];
                    Z[(size_t)row * kTcN + c] = z;
                    if (act == 1) Y[(size_t)row * kTcN + c] = fmaxf(z, 0.f);
                    else if (act == 2) Y[(size_t)row * kTcN + c] = res[(size_t)row * kTcN + c] + fmaxf(z, 0.f);
                }
            }
        }
    } else if (threadIdx.x == 0) {
        atomicExch(err, 1);
    }
    umma::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::fence_after();
        umma::tmem_dealloc(td, kTcN);
    }
}

// The backward products on the tensor cores (bf16 set), the same tcgen05 path as
// k_dense_fwd_tc: operands rounded to TF32 (the weights to BF16 first) and staged in
// shared memory in the canonical K-major layout, MMAs of 128 x NP x 8 issued by one
// thread into FP32 accumulators in tensor memory, an mbarrier per batch of MMAs
// (bounded waits: a wait that gives up sets err[0], waits once more with a bound for the
// MMAs in flight, releases the TMEM and leaves without writing).
//
// dX[R x K] = dZ[R x N] W[N x K]: one CTA of 4 warps per 128 rows; A = the rows of dZ
// (reduction over N, padded to NP8 = 8 * ceil(N / 8)), B = W^T (row k holds W[., k]),
// the MMA's N = KP (K padded to 16).
constexpr int kTcCols = 256;  // TMEM columns of a backward CTA (KP <= 256)

// Every thread of the CTA waits (bounded); the result is the same in all threads (a
// block-wide AND), so the warp-wide TMEM loads and the barriers after it stay convergent.
__device__ __forceinline__ bool tc_wait_or_fail(uint64_t* mbar, uint32_t parity, int* err) {
    bool ok = umma::mbar_wait(mbar, parity, 1 << 22);
    if (!ok) umma::mbar_wait(mbar, parity, 1 << 22);  // the MMAs in flight, once more with a bound
    ok = __syncthreads_and(ok) != 0;
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    return ok;
}

__global__ void __launch_bounds__(128) k_dense_dx_tc(const float* __restrict__ dZ, int R, int N, int NP8,
                                                     const float* __restrict__ W, int K, int KP,
                                                     float* __restrict__ dX, int bf16, int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int C = NP8 / 4;
    unsigned char* As = tc_smem;
    unsigned char* Bs = tc_smem + (size_t)kTcRows * NP8 * 4;
    const int row0 = blockIdx.x * kTcRows;
    for (int i = threadIdx.x; i < kTcRows * NP8; i += blockDim.x) {
        const int m = i / NP8, k = i % NP8;
        const float v = (row0 + m < R && k < N) ? dZ[(size_t)(row0 + m) * N + k] : 0.f;
        *(float*)(As + umma::core_offset(m, k >> 2, C) + (k & 3) * 4) = umma::tf32_round(v);
    }
    for (int i = threadIdx.x; i < KP * NP8; i += blockDim.x) {
        const int j = i / NP8, n = i % NP8;
        const float v = (j < K && n < N) ? wval(W, n * K + j, bf16) : 0.f;
        *(float*)(Bs + umma::core_offset(j, n >> 2, C) + (n & 3) * 4) = umma::tf32_round(v);
    }
    umma::fence_operands();
    if (threadIdx.x == 0) umma::mbar_init(&mbar, 1);
    if (threadIdx.x < 32) umma::tmem_alloc(&tmem_base, kTcCols);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t td = tmem_base;
    if (threadIdx.x == 0) {
        const uint32_t idesc = umma::idesc_tf32(kTcRows, KP);
        const uint32_t a0 = umma::smem_u32(As), b0 = umma::smem_u32(Bs);
        for (int k = 0; k < NP8 / 8; k++)
            umma::mma_tf32(td, umma::smem_desc(a0 + 256u * k, C), umma::smem_desc(b0 + 256u * k, C), idesc, k > 0);
        umma::commit(&mbar);
    }
    const bool ok = tc_wait_or_fail(&mbar, 0, err);
    umma::fence_after();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = row0 + warp * 32 + lane;
    if (ok) {
        const uint32_t tw = td + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < KP; c0 += 16) {
            uint32_t r[16];
            umma::tmem_load16(tw + c0, r);
            umma::tmem_wait16(r);
            if (row < R) {
#pragma unroll
                for (int j = 0; j < 16; j++)
                    if (c0 + j < K) dX[(size_t)row * K + c0 + j] = __uint_as_float(r[j]);
            }
        }
    }
    umma::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::fence_after();
        umma::tmem_dealloc(td, kTcCols);
    }
}

// Partials of dW[N x K] = dZ^T X and db[N] = sum_r dZ over rows [blockIdx * kRowsPerBlockW, ...):
// part[block][n * K + k], part[block][N * K + n] (the layout of k_dense_dw).  The D
// accumulator is 128 x KP with rows n < N (N <= 64; rows N.. are zero), columns k < K
// and column K = the row sum (a column of ones appended to X gives db); the block's rows
// go through in chunks of kDwChunk, one MMA batch and mbarrier phase per chunk.
constexpr int kDwChunk = 64;

__global__ void __launch_bounds__(128) k_dense_dw_tc(const float* __restrict__ dZ, const float* __restrict__ X, int R,
                                                     int N, int K, int KP, float* __restrict__ part,
                                                     int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    constexpr int C = kDwChunk / 4;
    unsigned char* As = tc_smem;
    unsigned char* Bs = tc_smem + (size_t)kTcRows * kDwChunk * 4;
    if (threadIdx.x == 0) umma::mbar_init(&mbar, 1);
    if (threadIdx.x < 32) umma::tmem_alloc(&tmem_base, kTcCols);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
    const uint32_t td = tmem_base;
    const int rbeg = blockIdx.x * kRowsPerBlockW, rend = min(R, rbeg + kRowsPerBlockW);
    bool ok = true;
    uint32_t phase = 0;
    for (int rc = rbeg; rc < rend && ok; rc += kDwChunk) {
        // operands of this chunk: A row n = dZ[rc.., n], B row k = X[rc.., k] (row K: ones)
        for (int i = threadIdx.x; i < kTcRows * kDwChunk; i += blockDim.x) {
            const int n = i / kDwChunk, r = i % kDwChunk;
            const float v = (n < N && rc + r < rend) ? dZ[(size_t)(rc + r) * N + n] : 0.f;
            *(float*)(As + umma::core_offset(n, r >> 2, C) + (r & 3) * 4) = umma::tf32_round(v);
        }
        for (int i = threadIdx.x; i < KP * kDwChunk; i += blockDim.x) {
            const int k = i / kDwChunk, r = i % kDwChunk;
            float v = 0.f;
            if (rc + r < rend) v = k < K ? X[(size_t)(rc + r) * K + k] : (k == K ? 1.f : 0.f);
            *(float*)(Bs + umma::core_offset(k, r >> 2, C) + (r & 3) * 4) = umma::tf32_round(v);
        }
        umma::fence_operands();
        umma::fence_before();
        __syncthreads();
        umma::fence_after();
        if (threadIdx.x == 0) {
            const uint32_t idesc = umma::idesc_tf32(kTcRows, KP);
            const uint32_t a0 = umma::smem_u32(As), b0 = umma::smem_u32(Bs);
            for (int k = 0; k < kDwChunk / 8; k++)
                umma::mma_tf32(td, umma::smem_desc(a0 + 256u * k, C), umma::smem_desc(b0 + 256u * k, C), idesc,
                               (rc > rbeg || k > 0) ? 1u : 0u);
            umma::commit(&mbar);
        }
        ok = tc_wait_or_fail(&mbar, phase, err);
        phase ^= 1u;
        umma::fence_after();
        __syncthreads();  // the next chunk overwrites the operands
    }
    const int nout = N * K + N;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = warp * 32 + lane;
    if (ok && rbeg < rend) {
        const uint32_t tw = td + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < KP; c0 += 16) {
            uint32_t r[16];
            umma::tmem_load16(tw + c0, r);
            umma::tmem_wait16(r);
            if (n < N) {
#pragma unroll
                for (int j = 0; j < 16; j++) {
                    const int k = c0 + j;
                    if (k < K) part[(size_t)blockIdx.x * nout + n * K + k] = __uint_as_float(r[j]);
                    else if (k == K) part[(size_t)blockIdx.x * nout + N * K + n] = __uint_as_float(r[j]);
                }
            }
        }
    }
    umma::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) {
        umma::fence_after();
        umma::tmem_dealloc(td, kTcCols);
    }
}

// dX[R x K] = dZ[R x N] W  (W [N x K]).  Block: 4 rows x 256/4 threads over k.
__global__ void __launch_bounds__(256) k_dense_dx(const float* __restrict__ dZ, int R, int N, const float* __restrict__ W,
                                                  int K, float* __restrict__ dX, int bf16) {
    extern __shared__ float sm[];
    float* Ws = sm;            // [N * K]
    float* Ds = sm + N * K;    // [4 * N]
    for (int i = threadIdx.x; i < N * K; i += blockDim.x) Ws[i] = wval(W, i, bf16);
    const int r0 = blockIdx.x * 4;
    for (int i = threadIdx.x; i < 4 * N; i += blockDim.x) {
        const int r = r0 + i / N;
        Ds[i] = r < R ? dZ[(size_t)r * N + i % N] : 0.f;
    }
    __syncthreads();
    const int rl = threadIdx.x / 64, r = r0 + rl;
    if (r >= R) return;
    for (int k = threadIdx.x % 64; k < K; k += 64) {
        float acc = 0.f;
        for (int c = 0; c < N; c++) acc = fmaf(Ds[rl * N + c], Ws[c * K + k], acc);
        dX[(size_t)r * K + k] = acc;
    }
}

// Per-block partials of dW[N x K] = dZ^T X and db[N] = sum_r dZ over rows
// [blockIdx * kRowsPerBlockW, ...): part[block][N * K + N].
__global__ void __launch_bounds__(256) k_dense_dw(const float* __restrict__ dZ, const float* __restrict__ X, int R,
                                                  int N, int K, float* __restrict__ part) {
    __shared__ float Ds[32 * 64];
    __shared__ float Xs[32 * kEdgeIn];
    const int nout = N * K + N;
    float acc[40];
    const int per = (nout + blockDim.x - 1) / blockDim.x;  // <= 40 for N*K+N <= 10240
#pragma unroll
    for (int j = 0; j < 40; j++) acc[j] = 0.f;
    const int rbeg = blockIdx.x * kRowsPerBlockW, rend = min(R, rbeg + kRowsPerBlockW);
    for (int rc = rbeg; rc < rend; rc += 32) {
        const int nr = min(32, rend - rc);
        __syncthreads();
        for (int i = threadIdx.x; i < 32 * N; i += blockDim.x) Ds[i] = (i / N) < nr ? dZ[(size_t)(rc + i / N) * N + i % N] : 0.f;
        for (int i = threadIdx.x; i < 32 * K; i += blockDim.x) Xs[i] = (i / K) < nr ? X[(size_t)(rc + i / K) * K + i % K] : 0.f;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < 40; j++) {
            if (j >= per) break;
            const int o = threadIdx.x + j * blockDim.x;
            if (o >= nout) break;
            float a = acc[j];
            if (o < N * K) {
                const int c = o / K, k = o % K;
                for (int r = 0; r < nr; r++) a = fmaf(Ds[r * N + c], Xs[r * K + k], a);
            } else {
                const int c = o - N * K;
                for (int r = 0; r < nr; r++) a += Ds[r * N + c];
            }
            acc[j] = a;
        }
    }
#pragma unroll
    for (int j = 0; j < 40; j++) {
        if (j >= per) break;
        const int o = threadIdx.x + j * blockDim.x;
        if (o < nout) part[(size_t)blockIdx.x * nout + o] = acc[j];
    }
}

// grad[o] += sum_b part[b][o] (fixed order).
__global__ void k_reduce_parts(const float* __restrict__ part, int nparts, int nout, float* __restrict__ grad) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= nout) return;
    float a = 0.f;
    for (int b = 0; b < nparts; b++) a += part[(size_t)b * nout + o];
    grad[o] += a;
}

// inp[e] = [h[row(e)], h[col(e)], ef[e]]
__global__ void k_edge_input(const float* __restrict__ h, const float* __restrict__ ef, const int* __restrict__ rows,
                             const int* __restrict__ col, int E, float* __restrict__ inp) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int e = (int)(t / kEdgeIn), k = (int)(t % kEdgeIn);
    if (e >= E) return;
    float v;
    if (k < kH) v = h[(size_t)rows[e] * kH + k];
    else if (k < 2 * kH) v = h[(size_t)col[e] * kH + k - kH];
    else v = ef[(size_t)e * kFe + k - 2 * kH];
    inp[t] = v;
}

// nin[i] = [h[i], mean_{e in row i} relu(zm[e])]  (agg stored in the second half)
__global__ void k_node_input(const float* __restrict__ h, const float* __restrict__ zm, const int* __restrict__ start,
                             int n, float* __restrict__ nin) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / kH, c = t % kH;
    if (i >= n) return;
    float a = 0.f;
    const int b = start[i], e1 = start[i + 1];
    for (int e = b; e < e1; e++) a += fmaxf(zm[(size_t)e * kH + c], 0.f);
    nin[(size_t)i * kNodeIn + c] = h[(size_t)i * kH + c];
    nin[(size_t)i * kNodeIn + kH + c] = a / (float)max(e1 - b, 1);
}

// B_i = L_i L_i^T / a_ii from the head output o_i (L: exp of o0..2 clamped to
// [-8, 8] on the diagonal, o3, o4, o5 at (1,0), (2,0), (2,1)).
__device__ __forceinline__ float clamp8(float v) { return fminf(fmaxf(v, -8.f), 8.f); }

__device__ __forceinline__ void lower_of(const float* o, float L[9]) {
    L[0] = expf(clamp8(o[0])); L[1] = 0.f; L[2] = 0.f;
    L[3] = o[3]; L[4] = expf(clamp8(o[1])); L[5] = 0.f;
    L[6] = o[4]; L[7] = o[5]; L[8] = expf(clamp8(o[2]));
}

__global__ void k_blocks(const float* __restrict__ o, const float* __restrict__ adiag, int n, float* __restrict__ B) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float L[9];
    lower_of(o + (size_t)i * kOut, L);
    const float ia = 1.f / adiag[i];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            float a = 0.f;
            for (int k = 0; k < 3; k++) a = fmaf(L[3 * r + k], L[3 * c + k], a);
            B[(size_t)i * 9 + 3 * r + c] = a * ia;
        }
}

// out = A v  (A = diag + CSR off-diagonal), v and out [n x 3]
__global__ void k_spmv3(const int* __restrict__ start, const int* __restrict__ col, const float* __restrict__ val,
                        const float* __restrict__ adiag, const float* __restrict__ v, int n, float* __restrict__ out,
                        const float* __restrict__ sub) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float a0 = adiag[i] * v[3 * i], a1 = adiag[i] * v[3 * i + 1], a2 = adiag[i] * v[3 * i + 2];
    for (int e = start[i]; e < start[i + 1]; e++) {
        const int j = col[e];
        a0 = fmaf(val[e], v[3 * j], a0);
        a1 = fmaf(val[e], v[3 * j + 1], a1);
        a2 = fmaf(val[e], v[3 * j + 2], a2);
    }
    if (sub) {
        a0 -= sub[3 * i];
        a1 -= sub[3 * i + 1];
        a2 -= sub[3 * i + 2];
    }
    out[3 * i] = a0;
    out[3 * i + 1] = a1;
    out[3 * i + 2] = a2;
}

__global__ void k_apply_blocks(const float* __restrict__ B, const float* __restrict__ r, int n, float* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* b = B + (size_t)i * 9;
    const float x = r[3 * i], y = r[3 * i + 1], w = r[3 * i + 2];
    z[3 * i] = b[0] * x + b[1] * y + b[2] * w;
    z[3 * i + 1] = b[3] * x + b[4] * y + b[5] * w;
    z[3 * i + 2] = b[6] * x + b[7] * y + b[8] * w;
}

// per-block partial sums of a . b (FP64) over 3n entries; one reduction slot per block
__global__ void k_dot_parts(const float* __restrict__ a, const float* __restrict__ b, int m, double* __restrict__ part) {
    __shared__ double sh[256];
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) s += (double)a[i] * (double)b[i];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// gB_i += (scale_k * gz_i) r_i^T with scale_k = 2 / (|r_k|^2 K) read from dots[k]
__global__ void k_accum_gB(const float* __restrict__ gz, const float* __restrict__ r, int n, const double* __restrict__ scale,
                           float* __restrict__ gB) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float s = (float)scale[0];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) gB[(size_t)i * 9 + 3 * a + b] += s * gz[3 * i + a] * r[3 * i + b];
}

// Head backward: go from gB (dL/dB) -- G = gB / a, gL = (G + G^T) L, go as in the header.
__global__ void k_head_grad(const float* __restrict__ gB, const float* __restrict__ o, const float* __restrict__ adiag,
                            int n, float* __restrict__ go, const float* __restrict__ gth) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float L[9], G[9], gL[9];
    lower_of(o + (size_t)i * kOut, L);
    const float ia = 1.f / adiag[i];
    for (int k = 0; k < 9; k++) G[k] = gB[(size_t)i * 9 + k] * ia;
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            float a = 0.f;
            for (int k = 0; k < 3; k++) a = fmaf(G[3 * r + k] + G[3 * k + r], L[3 * k + c], a);
            gL[3 * r + c] = a;
        }
    float* g = go + (size_t)i * kOut;
    const float* oi = o + (size_t)i * kOut;
    g[0] = fabsf(oi[0]) < 8.f ? gL[0] * L[0] : 0.f;
    g[1] = fabsf(oi[1]) < 8.f ? gL[4] * L[4] : 0.f;
    g[2] = fabsf(oi[2]) < 8.f ? gL[8] * L[8] : 0.f;
    g[3] = gL[3];
    g[4] = gL[6];
    g[5] = gL[7];
    g[6] = (gth && fabsf(oi[6]) < 1.f) ? gth[i] : 0.f;
}

// m_i = trace(B_i) / 3 (the isotropic part of the block: the system is A (x) I3),
// theta_i = clamp(o_i6, -1, 1).
__global__ void k_outputs(const float* __restrict__ B, const float* __restrict__ o, int n, float* __restrict__ m,
                          float* __restrict__ th) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    m[i] = (B[(size_t)i * 9] + B[(size_t)i * 9 + 4] + B[(size_t)i * 9 + 8]) * (1.f / 3.f);
    th[i] = fminf(fmaxf(o[(size_t)i * kOut + 6], -1.f), 1.f);
}

// gB_i = (gm_i / 3) I
__global__ void k_gm_to_gB(const float* __restrict__ gm, int n, float* __restrict__ gB) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float v = gm[i] * (1.f / 3.f);
    for (int k = 0; k < 9; k++) gB[(size_t)i * 9 + k] = (k % 4 == 0) ? v : 0.f;
}

// d = g * (z > 0)
__global__ void k_relu_mask(const float* __restrict__ g, const float* __restrict__ z, size_t m, float* __restrict__ d) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m) d[t] = z[t] > 0.f ? g[t] : 0.f;
}

// gzm[e] = gnin[row(e)][64 + c] / deg(row(e)) * (zm[e] > 0)   (gradient of the averaged messages)
__global__ void k_edge_grad(const float* __restrict__ gnin, const float* __restrict__ zm, const int* __restrict__ rows,
                            const int* __restrict__ start, int E, float* __restrict__ gzm) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int e = (int)(t / kH), c = (int)(t % kH);
    if (e >= E) return;
    const int i = rows[e];
    gzm[t] = zm[t] > 0.f ? gnin[(size_t)i * kNodeIn + kH + c] / (float)max(start[i + 1] - start[i], 1) : 0.f;
}

// gh[i] = gh_next[i] + gnin[i][c] + sum_{e in row i} ginp[e][c] + sum_{e in row i} ginp[rev(e)][64 + c]
__global__ void k_node_grad(const float* __restrict__ gh_next, const float* __restrict__ gnin, const float* __restrict__ ginp,
                            const int* __restrict__ start, const int* __restrict__ rev, int n, float* __restrict__ gh) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = t / kH, c = t % kH;
    if (i >= n) return;
    float a = gh_next[(size_t)i * kH + c] + gnin[(size_t)i * kNodeIn + c];
    for (int e = start[i]; e < start[i + 1]; e++) {
        a += ginp[(size_t)e * kEdgeIn + c];
        a += ginp[(size_t)rev[e] * kEdgeIn + kH + c];
    }
    gh[(size_t)i * kH + c] = a;
}

__global__ void k_adam(float* __restrict__ th, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1, float b2, float c1, float c2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    th[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline int nblk(size_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

struct AdmmGnn {
    int n = 0, E = 0, P = 0, bf16 = 1, steps = 0;
    std::vector<void*> allocs, gallocs;  // parameters and optimiser state; per-graph buffers
    int *start = nullptr, *col = nullptr, *rows = nullptr, *rev = nullptr;
    float *val = nullptr, *adiag = nullptr, *x = nullptr, *ef = nullptr;
    float *theta = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    float *z0 = nullptr, *h[4] = {nullptr, nullptr, nullptr, nullptr};
    float *inp[3] = {nullptr, nullptr, nullptr}, *zm[3] = {nullptr, nullptr, nullptr};
    float *nin[3] = {nullptr, nullptr, nullptr}, *zn[3] = {nullptr, nullptr, nullptr};
    float *o = nullptr, *B = nullptr;
    float *gh = nullptr, *gh2 = nullptr, *gz = nullptr, *ginp = nullptr, *gnin = nullptr, *go = nullptr, *gB = nullptr;
    float *part = nullptr, *r = nullptr, *zv = nullptr, *res = nullptr, *gzv = nullptr;
    double *dots = nullptr, *scal = nullptr;
    int* derr = nullptr;    // set by a tensor-core layer whose bounded wait gave up
    bool failed = false;    // a tensor-core layer timed out: outputs undefined, the handle refuses work
    cudaStream_t st = nullptr;
    std::string err;
};

namespace {

// parameter offsets (same order as the CPU restatement)
struct Off {
    int W0, b0, We[3], be[3], Wn[3], bn[3], Wo, bo, total;
};
Off offsets() {
    Off f;
    int k = 0;
    f.W0 = k; k += kH * kFin;
    f.b0 = k; k += kH;
    for (int l = 0; l < 3; l++) {
        f.We[l] = k; k += kH * kEdgeIn;
        f.be[l] = k; k += kH;
        f.Wn[l] = k; k += kH * kNodeIn;
        f.bn[l] = k; k += kH;
    }
    f.Wo = k; k += kOut * kH;
    f.bo = k; k += kOut;
    f.total = k;
    return f;
}

template <class T>
int galloc(AdmmGnn* g, T** p, size_t count, bool graph) {
    if (count == 0) count = 1;
    if (cudaMalloc((void**)p, count * sizeof(T)) != cudaSuccess) return ADMM_ERR_OOM;
    (graph ? g->gallocs : g->allocs).push_back(*p);
    cudaMemset(*p, 0, count * sizeof(T));
    return ADMM_OK;
}

#define GTRY(x)                  \
    do {                         \
        int r_ = (x);            \
        if (r_) return r_;       \
    } while (0)

// With BF16 weights the 64-output layers run on the tensor cores, the others
// (and every layer with FP32 weights) on the SIMT kernel.
void dense_fwd(AdmmGnn* g, const float* X, int R, int K, int wo, int bo, int N, float* Z, float* Y, const float* res,
               int act) {
    if (g->bf16 && N == kTcN && R > 0) {
        const int KP = (K + 7) / 8 * 8;
        const size_t sm = sizeof(float) * (size_t)(kTcRows + kTcN) * KP;
        k_dense_fwd_tc<<<nblk(R, kTcRows), 128, sm, g->st>>>(X, R, K, KP, g->theta + wo, g->theta + bo, Z, Y, res, act,
                                                            g->bf16, g->derr);
        return;
    }
    const size_t sm = sizeof(float) * (size_t)(N * K + 4 * K);
    k_dense_fwd<<<nblk(R, 4), 256, sm, g->st>>>(X, R, K, g->theta + wo, g->theta + bo, N, Z, Y, res, act, g->bf16);
}

// With BF16 weights the backward products run on the tensor cores (N <= 64 outputs of the
// layer, K + 1 <= 256 inputs plus the bias column), else on the SIMT kernels.
void dense_bwd(AdmmGnn* g, const float* dZ, const float* X, int R, int K, int wo, int N, float* dX) {
    const int KP = (K + 1 + 15) / 16 * 16;
    if (g->bf16 && N <= kTcN && KP <= kTcCols && R > 0) {
        const int NP8 = (N + 7) / 8 * 8;
        if (dX) {
            const int KPx = (K + 15) / 16 * 16;
            const size_t sm = std::max<size_t>(sizeof(float) * (size_t)(kTcRows + KPx) * NP8, 100 * 1024);
            k_dense_dx_tc<<<nblk(R, kTcRows), 128, sm, g->st>>>(dZ, R, N, NP8, g->theta + wo, K, KPx, dX, g->bf16,
                                                              g->derr);
        }
        const int nparts = nblk(R, kRowsPerBlockW), nout = N * K + N;
        const size_t sm = std::max<size_t>(sizeof(float) * (size_t)(kTcRows + KP) * kDwChunk, 100 * 1024);
        k_dense_dw_tc<<<nparts, 128, sm, g->st>>>(dZ, X, R, N, K, KP, g->part, g->derr);
        k_reduce_parts<<<nblk(nout, 256), 256, 0, g->st>>>(g->part, nparts, nout, g->grad + wo);
        return;
    }
    if (dX) {
        const size_t sm = sizeof(float) * (size_t)(N * K + 4 * N);
        k_dense_dx<<<nblk(R, 4), 256, sm, g->st>>>(dZ, R, N, g->theta + wo, K, dX, g->bf16);
    }
    const int nparts = nblk(R, kRowsPerBlockW), nout = N * K + N;
    k_dense_dw<<<nparts, 256, 0, g->st>>>(dZ, X, R, N, K, g->part);
    // the bias follows its weight in the parameter vector
    k_reduce_parts<<<nblk(nout, 256), 256, 0, g->st>>>(g->part, nparts, nout, g->grad + wo);
}

void forward(AdmmGnn* g) {
    const Off f = offsets();
    dense_fwd(g, g->x, g->n, kFin, f.W0, f.b0, kH, g->z0, g->h[0], nullptr, 1);
    for (int l = 0; l < 3; l++) {
        k_edge_input<<<nblk((size_t)g->E * kEdgeIn, 256), 256, 0, g->st>>>(g->h[l], g->ef, g->rows, g->col, g->E, g->inp[l]);
        dense_fwd(g, g->inp[l], g->E, kEdgeIn, f.We[l], f.be[l], kH, g->zm[l], nullptr, nullptr, 0);
        k_node_input<<<nblk((size_t)g->n * kH, 256), 256, 0, g->st>>>(g->h[l], g->zm[l], g->start, g->n, g->nin[l]);
        dense_fwd(g, g->nin[l], g->n, kNodeIn, f.Wn[l], f.bn[l], kH, g->zn[l], g->h[l + 1], g->h[l], 2);
    }
    dense_fwd(g, g->h[3], g->n, kH, f.Wo, f.bo, kOut, g->o, nullptr, nullptr, 0);
    k_blocks<<<nblk(g->n, 256), 256, 0, g->st>>>(g->o, g->adiag, g->n, g->B);
}

// ADMM_ERR_TIMEOUT once a tensor-core layer gave up waiting for its MMAs (the
// flag is cleared for the next call).
int tc_status(AdmmGnn* g) {
    int e = 0;
    if (cudaMemcpy(&e, g->derr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return ADMM_ERR_CUDA;
    if (!e) return ADMM_OK;
    // a CTA that gave up may have left its MMAs reading shared memory and writing TMEM:
    // the outputs of that launch are undefined and the handle takes no further work
    g->failed = true;
    return ADMM_ERR_TIMEOUT;
}

void backward_from_head(AdmmGnn* g);

}  // namespace

extern "C" {

int admm_gnn_create(int bf16, AdmmGnn** out) {
    if (!out) return ADMM_ERR_INVALID;
    *out = nullptr;
    AdmmGnn* g = new (std::nothrow) AdmmGnn;
    if (!g) return ADMM_ERR_OOM;
    g->bf16 = bf16 ? 1 : 0;
    g->P = offsets().total;
    int rc;
    if ((rc = galloc(g, &g->theta, g->P, false)) || (rc = galloc(g, &g->grad, g->P, false)) ||
        (rc = galloc(g, &g->m, g->P, false)) || (rc = galloc(g, &g->v, g->P, false)) ||
        (rc = galloc(g, &g->derr, 1, false))) {
        admm_gnn_destroy(g);
        return rc;
    }
    if (cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking) != cudaSuccess) {
        admm_gnn_destroy(g);
        return ADMM_ERR_CUDA;
    }
    cudaFuncSetAttribute(k_dense_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    cudaFuncSetAttribute(k_dense_dx, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    cudaFuncSetAttribute(k_dense_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(k_dense_dx_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    cudaFuncSetAttribute(k_dense_dw_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    *out = g;
    return ADMM_OK;
}

// The graph the next calls work on (replaces the previous one; parameters and
// optimiser state are kept, so one network trains on many systems).
int admm_gnn_set_graph(AdmmGnn* g, int n, int n_edges, const int32_t* start, const int32_t* col, const float* val,
                       const float* adiag, const float* node_feat, const float* edge_feat) {
    if (!g || n <= 0 || n_edges < 0 || !start || !adiag || !node_feat || (n_edges > 0 && (!col || !val || !edge_feat)))
        return ADMM_ERR_INVALID;
    cudaStreamSynchronize(g->st);
    for (void* p : g->gallocs) cudaFree(p);
    g->gallocs.clear();
    g->n = n;
    g->E = n_edges;
    std::vector<int> rows(n_edges), rev(n_edges, 0);
    for (int i = 0; i < n; i++)
        for (int e = start[i]; e < start[i + 1]; e++) rows[e] = i;
    for (int i = 0; i < n; i++)  // reverse edge: (j -> i) in row j, binary search (columns sorted)
        for (int e = start[i]; e < start[i + 1]; e++) {
            const int j = col[e];
            int lo = start[j], hi = start[j + 1] - 1, k = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) / 2;
                if (col[mid] == i) { k = mid; break; }
                if (col[mid] < i) lo = mid + 1; else hi = mid - 1;
            }
            if (k < 0) return ADMM_ERR_INVALID;  // the pattern must be symmetric with sorted columns
            rev[e] = k;
        }
    auto up = [&](auto** p, const auto* src, size_t cnt) -> int {
        GTRY(galloc(g, p, cnt, true));
        if (cnt && src) cudaMemcpy(*p, src, cnt * sizeof(**p), cudaMemcpyHostToDevice);
        return ADMM_OK;
    };
    auto ga = [&](auto** p, size_t cnt) -> int { return galloc(g, p, cnt, true); };
    const size_t H = kH, N = n, Ee = n_edges;
    int rc = ADMM_OK;
    if ((rc = up(&g->start, start, N + 1)) || (rc = up(&g->col, col, Ee)) || (rc = up(&g->rows, rows.data(), Ee)) ||
        (rc = up(&g->rev, rev.data(), Ee)) || (rc = up(&g->val, val, Ee)) || (rc = up(&g->adiag, adiag, N)) ||
        (rc = up(&g->x, node_feat, N * kFin)) || (rc = up(&g->ef, edge_feat, Ee * kFe)) || (rc = ga(&g->z0, N * H)) ||
        (rc = ga(&g->o, N * kOut)) || (rc = ga(&g->B, N * 9)) || (rc = ga(&g->gh, N * H)) || (rc = ga(&g->gh2, N * H)) ||
        (rc = ga(&g->gz, std::max(Ee, N) * H)) || (rc = ga(&g->ginp, Ee * kEdgeIn)) || (rc = ga(&g->gnin, N * kNodeIn)) ||
        (rc = ga(&g->go, N * kOut)) || (rc = ga(&g->gB, N * 9)) ||
        (rc = ga(&g->part, (size_t)nblk(std::max(n_edges, n), kRowsPerBlockW) * (kH * kEdgeIn + kH))) ||
        (rc = ga(&g->r, N * 3)) || (rc = ga(&g->zv, N * 3)) || (rc = ga(&g->res, N * 3)) || (rc = ga(&g->gzv, N * 3)) ||
        (rc = ga(&g->dots, 1024)) || (rc = ga(&g->scal, 4)))
        return rc;
    for (int l = 0; l < 4; l++) GTRY(ga(&g->h[l], N * H));
    for (int l = 0; l < 3; l++) {
        GTRY(ga(&g->inp[l], Ee * kEdgeIn));
        GTRY(ga(&g->zm[l], Ee * H));
        GTRY(ga(&g->nin[l], N * kNodeIn));
        GTRY(ga(&g->zn[l], N * H));
    }
    return cudaGetLastError() == cudaSuccess ? ADMM_OK : ADMM_ERR_CUDA;
}

void admm_gnn_destroy(AdmmGnn* g) {
    if (!g) return;
    if (g->st) {
        cudaStreamSynchronize(g->st);
        cudaStreamDestroy(g->st);
    }
    for (void* p : g->allocs) cudaFree(p);
    for (void* p : g->gallocs) cudaFree(p);
    delete g;
}

int admm_gnn_num_params(void) { return offsets().total; }

int admm_gnn_set_params(AdmmGnn* g, const float* theta, int P) {
    if (!g || !theta || P != g->P) return ADMM_ERR_INVALID;
    if (cudaMemcpy(g->theta, theta, sizeof(float) * P, cudaMemcpyHostToDevice) != cudaSuccess) return ADMM_ERR_CUDA;
    cudaMemset(g->m, 0, sizeof(float) * P);  // a new starting point: the optimiser starts afresh
    cudaMemset(g->v, 0, sizeof(float) * P);
    g->steps = 0;
    return ADMM_OK;
}

int admm_gnn_get_params(AdmmGnn* g, float* theta, int P) {
    if (!g || !theta || P != g->P) return ADMM_ERR_INVALID;
    cudaStreamSynchronize(g->st);
    return cudaMemcpy(theta, g->theta, sizeof(float) * P, cudaMemcpyDeviceToHost) == cudaSuccess ? ADMM_OK : ADMM_ERR_CUDA;
}

// Forward pass; blocks9 (host, n x 9 row-major) receives B_i = L_i L_i^T / a_ii.
int admm_gnn_forward(AdmmGnn* g, float* blocks9) {
    if (!g || g->n <= 0) return ADMM_ERR_INVALID;
    if (g->failed) return ADMM_ERR_STATE;
    forward(g);
    if (blocks9 && cudaMemcpyAsync(blocks9, g->B, sizeof(float) * 9 * (size_t)g->n, cudaMemcpyDeviceToHost, g->st) != cudaSuccess)
        return ADMM_ERR_CUDA;
    if (cudaStreamSynchronize(g->st) != cudaSuccess) return ADMM_ERR_CUDA;
    if (cudaGetLastError() != cudaSuccess) return ADMM_ERR_CUDA;
    return tc_status(g);
}

// Loss mean_k |A B r_k - r_k|^2 / |r_k|^2 over K residual samples (host, K x n x 3)
// and, into the gradient buffer (zeroed first), its gradient; grad (host, may be
// null) receives it.
int admm_gnn_loss_grad(AdmmGnn* g, const float* R, int K, double* loss, float* grad) {
    if (!g || g->n <= 0 || !R || K <= 0) return ADMM_ERR_INVALID;
    if (g->failed) return ADMM_ERR_STATE;
    const int n = g->n;
    forward(g);
    cudaMemsetAsync(g->grad, 0, sizeof(float) * g->P, g->st);
    cudaMemsetAsync(g->gB, 0, sizeof(float) * 9 * (size_t)n, g->st);
    double total = 0.0;
    const int nb = 256;
    for (int k = 0; k < K; k++) {
        cudaMemcpyAsync(g->r, R + (size_t)k * n * 3, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, g->st);
        k_apply_blocks<<<nblk(n, 256), 256, 0, g->st>>>(g->B, g->r, n, g->zv);
        k_spmv3<<<nblk(n, 256), 256, 0, g->st>>>(g->start, g->col, g->val, g->adiag, g->zv, n, g->res, g->r);
        k_dot_parts<<<nb, 256, 0, g->st>>>(g->r, g->r, 3 * n, g->dots);
        k_dot_parts<<<nb, 256, 0, g->st>>>(g->res, g->res, 3 * n, g->dots + nb);
        std::vector<double> d(2 * nb);
        cudaMemcpyAsync(d.data(), g->dots, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, g->st);
        if (cudaStreamSynchronize(g->st) != cudaSuccess) return ADMM_ERR_CUDA;
        double rr = 0.0, ee = 0.0;
        for (int b = 0; b < nb; b++) { rr += d[b]; ee += d[nb + b]; }
        if (!(rr > 0.0)) continue;
        total += ee / rr / K;
        const double sc = 2.0 / (rr * K);
        cudaMemcpyAsync(g->scal, &sc, sizeof(double), cudaMemcpyHostToDevice, g->st);
        k_spmv3<<<nblk(n, 256), 256, 0, g->st>>>(g->start, g->col, g->val, g->adiag, g->res, n, g->gzv, nullptr);
        k_accum_gB<<<nblk(n, 256), 256, 0, g->st>>>(g->gzv, g->r, n, g->scal, g->gB);
        if (cudaStreamSynchronize(g->st) != cudaSuccess) return ADMM_ERR_CUDA;
    }
    k_head_grad<<<nblk(n, 256), 256, 0, g->st>>>(g->gB, g->o, g->adiag, n, g->go, nullptr);
    backward_from_head(g);
    if (grad) cudaMemcpyAsync(grad, g->grad, sizeof(float) * g->P, cudaMemcpyDeviceToHost, g->st);
    if (cudaStreamSynchronize(g->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ADMM_ERR_CUDA;
    if (loss) *loss = total;
    return tc_status(g);
}

// Per-vertex outputs of the learned global step: m (n) and theta (n), host.
int admm_gnn_outputs(AdmmGnn* g, float* m, float* theta) {
    if (!g || g->n <= 0 || !m || !theta) return ADMM_ERR_INVALID;
    if (g->failed) return ADMM_ERR_STATE;
    forward(g);
    k_outputs<<<nblk(g->n, 256), 256, 0, g->st>>>(g->B, g->o, g->n, g->r, g->zv);
    cudaMemcpyAsync(m, g->r, sizeof(float) * g->n, cudaMemcpyDeviceToHost, g->st);
    cudaMemcpyAsync(theta, g->zv, sizeof(float) * g->n, cudaMemcpyDeviceToHost, g->st);
    if (cudaStreamSynchronize(g->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ADMM_ERR_CUDA;
    return tc_status(g);
}

// Gradient of a loss with respect to the parameters, given its gradients gm and
// gtheta (host, n each) with respect to the outputs of admm_gnn_outputs (at the
// current parameters and graph); grad (host, may be null) receives it, and the
// next admm_gnn_adam applies it.
int admm_gnn_backward(AdmmGnn* g, const float* gm, const float* gtheta, float* grad) {
    if (!g || g->n <= 0 || !gm || !gtheta) return ADMM_ERR_INVALID;
    if (g->failed) return ADMM_ERR_STATE;
    const int n = g->n;
    forward(g);
    cudaMemsetAsync(g->grad, 0, sizeof(float) * g->P, g->st);
    cudaMemcpyAsync(g->r, gm, sizeof(float) * n, cudaMemcpyHostToDevice, g->st);
    cudaMemcpyAsync(g->zv, gtheta, sizeof(float) * n, cudaMemcpyHostToDevice, g->st);
    k_gm_to_gB<<<nblk(n, 256), 256, 0, g->st>>>(g->r, n, g->gB);
    k_head_grad<<<nblk(n, 256), 256, 0, g->st>>>(g->gB, g->o, g->adiag, n, g->go, g->zv);
    backward_from_head(g);
    if (grad) cudaMemcpyAsync(grad, g->grad, sizeof(float) * g->P, cudaMemcpyDeviceToHost, g->st);
    if (cudaStreamSynchronize(g->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) return ADMM_ERR_CUDA;
    return tc_status(g);
}

}  // extern "C"

namespace {

// The backward pass from the head gradient go (dL/do) into g->grad.
void backward_from_head(AdmmGnn* g) {
    const Off f = offsets();
    const int n = g->n, E = g->E;
    dense_bwd(g, g->go, g->h[3], n, kH, f.Wo, kOut, g->gh);          // gh = dL/dh3
    for (int l = 2; l >= 0; l--) {
        const size_t nh = (size_t)n * kH;
        k_relu_mask<<<nblk(nh, 256), 256, 0, g->st>>>(g->gh, g->zn[l], nh, g->gz);   // gzn
        dense_bwd(g, g->gz, g->nin[l], n, kNodeIn, f.Wn[l], kH, g->gnin);
        k_edge_grad<<<nblk((size_t)E * kH, 256), 256, 0, g->st>>>(g->gnin, g->zm[l], g->rows, g->start, E, g->gz);  // gzm
        dense_bwd(g, g->gz, g->inp[l], E, kEdgeIn, f.We[l], kH, g->ginp);
        k_node_grad<<<nblk(nh, 256), 256, 0, g->st>>>(g->gh, g->gnin, g->ginp, g->start, g->rev, n, g->gh2);
        std::swap(g->gh, g->gh2);
    }
    k_relu_mask<<<nblk((size_t)n * kH, 256), 256, 0, g->st>>>(g->gh, g->z0, (size_t)n * kH, g->gz);
    dense_bwd(g, g->gz, g->x, n, kFin, f.W0, kH, nullptr);
}

}  // namespace

extern "C" {

// One Adam step on the gradient of the last admm_gnn_loss_grad.
int admm_gnn_adam(AdmmGnn* g, float lr) {
    if (!g) return ADMM_ERR_INVALID;
    g->steps++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)g->steps), c2 = 1.f - std::pow(b2, (float)g->steps);
    k_adam<<<nblk(g->P, 256), 256, 0, g->st>>>(g->theta, g->grad, g->m, g->v, g->P, lr, b1, b2, c1, c2, 1e-8f);
    return cudaStreamSynchronize(g->st) == cudaSuccess ? ADMM_OK : ADMM_ERR_CUDA;
}

}  // extern "C"
