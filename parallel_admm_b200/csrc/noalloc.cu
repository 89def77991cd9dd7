// noalloc.cu -- a Jacobi solve of the global system that allocates nothing.
//
// The handle API (admm_b200_create) allocates every device buffer it needs up
// front.  Some callers cannot do that: a host application whose device memory is
// entirely owned by its own pool allocator and that forbids any other cudaMalloc,
// a real-time loop that cannot afford cudaMalloc's latency and implicit device
// synchronisation, or a plug-in host that only hands out buffers it allocated
// itself.  admm_b200_jacobi_noalloc serves them: the caller passes the matrix,
// the right-hand side and the input/output positions in its own device memory,
// and the two ping-pong buffers the sweeps need live in a file-scope
// __device__ array of fixed size, g_jacobi_scratch, reserved in every GPU that
// loads the library until the process exits.
//
// Limits and contract:
//  * at most kNoAllocMaxRows rows (262144, i.e. 2 x 262144 x 3 floats = 6 MiB of
//    static device memory); larger systems are rejected with ADMM_ERR_INVALID;
//  * the scratch is shared by every call in the process: calls whose work
//    overlaps on the GPU (different streams, or different host threads on one
//    device) race on it and must be ordered by the caller;
//  * nothing in the scratch needs to start at zero: every sweep overwrites all
//    rows it later reads, so a call never sees the previous call's contents;
//  * the first call on a device looks up the device address of the scratch
//    (cudaGetSymbolAddress, with that device current) and keeps it for later
//    calls; that first call should come before any stream capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "admm_b200.h"

namespace {

constexpr int kNoAllocMaxRows = 262144;
constexpr int kNoAllocMaxDevices = 64;

// Two ping-pong buffers of row-major n x 3 floats.
static __device__ __align__(256) float g_jacobi_scratch[2][kNoAllocMaxRows * 3];

std::mutex g_mu;
float* g_scratch_dev[kNoAllocMaxDevices] = {nullptr};

// One Jacobi sweep on CSR (off-diagonal part, JacobiFunctor of the reference's
// jacobi_solver.cu:52-98): dst_i = (b_i - sum_{j != i} a_ij src_j) / a_ii,
// row-major n x 3 vectors.
__global__ void k_jacobi_csr(int n, const int32_t* __restrict__ start, const int32_t* __restrict__ cols,
                             const float* __restrict__ vals, const float* __restrict__ diag,
                             const float* __restrict__ b, const float* __restrict__ src, float* __restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float ax = 0.f, ay = 0.f, az = 0.f;
    const int e = start[i + 1];
    for (int k = start[i]; k < e; k++) {
        const int j = cols[k];
        const float a = vals[k];
        ax = fmaf(a, src[3 * j + 0], ax);
        ay = fmaf(a, src[3 * j + 1], ay);
        az = fmaf(a, src[3 * j + 2], az);
    }
    const float d = diag[i];
    dst[3 * i + 0] = (b[3 * i + 0] - ax) / d;
    dst[3 * i + 1] = (b[3 * i + 1] - ay) / d;
    dst[3 * i + 2] = (b[3 * i + 2] - az) / d;
}

// Device address of g_jacobi_scratch on the current device (looked up once).
int scratch_on_current_device(float** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return ADMM_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_jacobi_scratch);
        if (e != cudaSuccess) {
            fprintf(stderr, "admm_b200_jacobi_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return ADMM_ERR_CUDA;
        }
        g_scratch_dev[dev] = static_cast<float*>(p);
    }
    *out = g_scratch_dev[dev];
    return ADMM_OK;
}

}  // namespace

extern "C" int admm_b200_jacobi_noalloc(int n, const int32_t* row_start, const int32_t* cols, const float* vals,
                                        const float* diag, const float* b, const float* x_in, float* x_out, int sweeps,
                                        void* stream) {
    if (n <= 0 || n > kNoAllocMaxRows) {
        fprintf(stderr, "admm_b200_jacobi_noalloc: n = %d rows is outside 1..%d (the static scratch holds %d rows)\n",
                n, kNoAllocMaxRows, kNoAllocMaxRows);
        return ADMM_ERR_INVALID;
    }
    if (sweeps < 0 || !row_start || !cols || !vals || !diag || !b || !x_in || !x_out) {
        fprintf(stderr, "admm_b200_jacobi_noalloc: null pointer or negative sweep count\n");
        return ADMM_ERR_INVALID;
    }
    float* scratch = nullptr;
    const int rc = scratch_on_current_device(&scratch);
    if (rc != ADMM_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t bytes = sizeof(float) * 3 * (size_t)n;
    if (sweeps == 0) {
        if (x_out != x_in && cudaMemcpyAsync(x_out, x_in, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return ADMM_ERR_CUDA;
        return ADMM_OK;
    }
    float* buf[2] = {scratch, scratch + (size_t)kNoAllocMaxRows * 3};
    const int threads = 128, blocks = (n + threads - 1) / threads;
    for (int k = 0; k < sweeps; k++) {
        const float* src = k == 0 ? x_in : buf[(k - 1) & 1];
        // the last sweep writes x_out directly unless x_out is also its source
        float* dst = (k == sweeps - 1 && src != x_out) ? x_out : buf[k & 1];
        k_jacobi_csr<<<blocks, threads, 0, st>>>(n, row_start, cols, vals, diag, b, src, dst);
        if (k == sweeps - 1 && dst != x_out &&
            cudaMemcpyAsync(x_out, dst, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return ADMM_ERR_CUDA;
    }
    return cudaGetLastError() == cudaSuccess ? ADMM_OK : ADMM_ERR_CUDA;
}
