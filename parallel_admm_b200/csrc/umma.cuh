// umma.cuh -- the fifth-generation tensor cores (tcgen05) for the dense layers
// of the learned preconditioner: shared-memory operand descriptors of the
// canonical no-swizzle K-major layout, the instruction descriptor of
// kind::tf32 with FP32 accumulation, tensor-memory (TMEM) allocation, the MMA
// issued by one thread, its completion through an mbarrier, and the TMEM ->
// register load of the accumulator.  Field layouts follow the PTX ISA for
// sm_100a (the same bit positions as CUTLASS's UMMA::SmemDescriptor and
// UMMA::InstrDescriptor).
#pragma once
#include <cstdint>

namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major operand without swizzle: 8-row x 16-byte core matrices; core matrix
// (row group g, 16-byte K chunk c) starts at (g * chunks + c) * 128 bytes, so
// the next K chunk is 128 B further (leading byte offset) and the next row
// group chunks * 128 B further (stride byte offset).  Row r of a core matrix
// is its r-th 16 bytes.
__host__ __device__ constexpr uint32_t core_offset(int row, int chunk, int chunks) {
    return (uint32_t)(((row >> 3) * chunks + chunk) * 128 + (row & 7) * 16);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t chunks) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);            // start address >> 4, bits [0,14)
    d |= (uint64_t)(128u >> 4) << 16;                   // leading byte offset >> 4, bits [16,30)
    d |= (uint64_t)(((chunks * 128u) >> 4) & 0x3FFFu) << 32;  // stride byte offset >> 4, bits [32,46)
    d |= (uint64_t)1 << 46;                             // descriptor version 1, bits [46,48)
    return d;                                           // base offset 0, legacy LBO mode, no swizzle
}

// D format F32 (bits 4-5), A and B format TF32 (bits 7-9, 10-12), both
// K-major (bits 15, 16 clear), N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ float tf32_round(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
    return __uint_as_float(r);
}

__device__ __forceinline__ void fence_operands() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Whole warp: allocate `cols` TMEM columns (a power of two >= 32); the base
// address is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// One thread: D (+)= A B^T for one K step of the operands described by adesc, bdesc.
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;  // no output lane disabled
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3)
        : "memory");
}

// One thread: arrive on the mbarrier once all MMAs it issued have completed.
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

// Initialises the mbarrier and makes the initialisation visible to the
// asynchronous proxy that the MMA commit arrives through.
__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for phase `parity` of the mbarrier at most `limit` polls; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, int limit) {
    const uint32_t a = smem_u32(mbar);
    for (int i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t"
            ".reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// The warp's 32 TMEM lanes (its quarter of the 128 rows), 16 consecutive
// 32-bit columns.  The registers hold the values only after tmem_wait16.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

// Waits for this thread's outstanding TMEM loads; the registers pass through
// the instruction so that no use of them is scheduled before it.
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

}  // namespace umma
