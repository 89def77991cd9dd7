// common.cuh -- shared device helpers for the B200 ADMM substep.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#define ADMM_DEV __device__ __forceinline__

// Programmatic dependent launch: every kernel of a substep first lets the next
// kernel of the stream begin its launch, then waits until all preceding kernels
// have completed and their writes are visible.  Results are unchanged; the
// launch latency of a kernel overlaps the execution of its predecessor.  Both
// instructions are no-ops for a kernel launched without the PDL attribute.
// The two halves, for kernels that first load data which no kernel of a substep
// writes (matrices, constraint records) and only then wait: those loads overlap
// the tail of the preceding kernels.
#define ADMM_PDL_TRIGGER() asm volatile("griddepcontrol.launch_dependents;" ::: "memory")
#define ADMM_PDL_WAIT() asm volatile("griddepcontrol.wait;" ::: "memory")

// Wait first, then let the next kernel launch: the next kernel then starts only
// after this kernel's predecessor has completed, so before its own wait it may
// read (through L2) anything that the kernels before this one wrote.
#define ADMM_PDL_WAIT_THEN_TRIGGER()                                 \
    do {                                                             \
        asm volatile("griddepcontrol.wait;" ::: "memory");           \
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); \
    } while (0)

#define ADMM_PDL_PROLOGUE()                                          \
    do {                                                             \
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); \
        asm volatile("griddepcontrol.wait;" ::: "memory");           \
    } while (0)

namespace admm {

constexpr int kWarp = 32;

// Launches `k` on `st`; with pdl the launch carries the programmatic stream
// serialization attribute (the kernel must start with ADMM_PDL_PROLOGUE).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                            Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? attr : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

ADMM_DEV float4 f4(float x, float y, float z, float w = 0.f) { return make_float4(x, y, z, w); }
ADMM_DEV float4 add3(float4 a, float4 b) { return f4(a.x + b.x, a.y + b.y, a.z + b.z); }
ADMM_DEV float4 sub3(float4 a, float4 b) { return f4(a.x - b.x, a.y - b.y, a.z - b.z); }
ADMM_DEV float4 scale3(float4 a, float s) { return f4(a.x * s, a.y * s, a.z * s); }
ADMM_DEV float dot3(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Non-contracting operations: every call is one IEEE round-to-nearest float
// operation, in the order written (the narrow phase must match the oracle bit
// for bit, and the oracle is compiled with -ffp-contract=off).
ADMM_DEV float fadd(float a, float b) { return __fadd_rn(a, b); }
ADMM_DEV float fsub(float a, float b) { return __fsub_rn(a, b); }
ADMM_DEV float fmul(float a, float b) { return __fmul_rn(a, b); }
ADMM_DEV float fdiv(float a, float b) { return __fdiv_rn(a, b); }
ADMM_DEV float fsqrt(float a) { return __fsqrt_rn(a); }

// float <-> order-preserving uint32 for atomicMin/atomicMax on floats
ADMM_DEV uint32_t float_to_ordered(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
ADMM_DEV float ordered_to_float(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

template <class T>
ADMM_DEV T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of a double; result valid in thread 0.  Uses blockDim.x/32
// doubles of shared memory passed in by the caller.
ADMM_DEV double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        r = lane < nw ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

}  // namespace admm
