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
//  * the device address of the scratch is looked up (cudaGetSymbolAddress) in the
//    context that is current on the calling thread, on every call made outside
//    stream capture, and remembered per context; a call made while its stream is
//    being captured uses the address remembered for the current context, so a call
//    in that context must have run outside capture first (else ADMM_ERR_STATE).
//    Keying by context keeps the address right for callers that run in their own
//    driver-API contexts and across a cudaDeviceReset;
//  * an error already pending on the calling thread (from the caller's own work)
//    is left untouched and the call returns ADMM_ERR_CUDA without launching.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <vector>

#include "admm_b200.h"

namespace {

constexpr int kNoAllocMaxRows = 262144;
// Two ping-pong buffers of row-major n x 3 floats.
static __device__ __align__(256) float g_jacobi_scratch[2][kNoAllocMaxRows * 3];

// Address of g_jacobi_scratch per CUDA context (CUcontext as an opaque pointer).
struct ScratchEntry {
    void* ctx;
    float* ptr;
};
std::mutex g_mu;
std::vector<ScratchEntry> g_scratch;

typedef int (*CtxGetCurrentFn)(void**);

// The context current on this thread (the runtime's primary context unless the
// caller made its own current), through the driver's cuCtxGetCurrent.
void* current_context() {
    static CtxGetCurrentFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
    });
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) return nullptr;
    return ctx;
}

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

// Device address of g_jacobi_scratch in the current context: looked up again on
// every call outside capture (cheap), taken from the per-context record during
// capture.
int scratch_address(cudaStream_t st, float** out) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return ADMM_ERR_CUDA;  // also makes a context current
    void* ctx = current_context();
    if (!ctx) {
        fprintf(stderr, "admm_b200_jacobi_noalloc: no current CUDA context\n");
        return ADMM_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    ScratchEntry* e = nullptr;
    for (auto& x : g_scratch)
        if (x.ctx == ctx) e = &x;
    if (cs != cudaStreamCaptureStatusNone) {
        if (!e) {
            fprintf(stderr, "admm_b200_jacobi_noalloc: first call in this context made during stream capture; "
                            "call it once outside capture first\n");
            return ADMM_ERR_STATE;
        }
        *out = e->ptr;
        return ADMM_OK;
    }
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_jacobi_scratch);
    if (err != cudaSuccess) {
        fprintf(stderr, "admm_b200_jacobi_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(err));
        return ADMM_ERR_CUDA;
    }
    if (e)
        e->ptr = static_cast<float*>(p);
    else
        g_scratch.push_back({ctx, static_cast<float*>(p)});
    *out = static_cast<float*>(p);
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
    if (cudaPeekAtLastError() != cudaSuccess) {
        fprintf(stderr, "admm_b200_jacobi_noalloc: a CUDA error is already pending on this thread (%s); "
                        "nothing launched\n", cudaGetErrorString(cudaPeekAtLastError()));
        return ADMM_ERR_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    float* scratch = nullptr;
    const int rc = scratch_address(st, &scratch);
    if (rc != ADMM_OK) return rc;
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
        if (cudaGetLastError() != cudaSuccess) return ADMM_ERR_CUDA;
        if (k == sweeps - 1 && dst != x_out &&
            cudaMemcpyAsync(x_out, dst, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return ADMM_ERR_CUDA;
    }
    return ADMM_OK;
}
