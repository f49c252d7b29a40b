// tcgen05 building blocks for sm_100a (inline PTX): TMEM allocation, shared-memory matrix and instruction
// descriptors for kind::f16 (BF16 operands, FP32 accumulator), the MMA issue, its commit to an mbarrier,
// bounded mbarrier waits and the TMEM -> register load of an accumulator.
//
// Operand layout used throughout: K-major, no swizzle. A matrix of R rows x K bf16 is a grid of "core
// matrices" of 8 rows x 8 elements (8 x 16 bytes, rows 16 bytes apart, 128 contiguous bytes); core
// matrices adjacent along K are LBO bytes apart, groups of 8 rows SBO bytes apart. For a row-block of
// K = Kp elements stored K-chunk-minor: offset(r, k) = (r / 8) * (Kp / 8 * 128) + (k / 8) * 128 + (r % 8) * 16
// + (k % 8) * 2, so LBO = 128 and SBO = Kp / 8 * 128; one MMA consumes K = 16 (two K chunks), and the
// next K step starts 256 bytes further.
#pragma once
#include <cstdint>

namespace gam {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor (K-major, SWIZZLE_NONE, version 1)
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for tcgen05
    return d;                 // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor: kind::f16 with BF16 A and B (both K-major), FP32 D, dense, M x N
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4)                       // D format F32
         | (1u << 7)                       // A format BF16
         | (1u << 10)                      // B format BF16
         | ((uint32_t)(N >> 3) << 17)      // N / 8
         | ((uint32_t)(M >> 4) << 24);     // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool acc) {
    uint32_t scale = acc ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(scale));
}

// arrive on the mbarrier when every MMA issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(mbar)), "r"(count) : "memory");
}

// wait until the phase with the given parity has completed; gives up after maxIter polls (returns false)
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t maxIter) {
    uint32_t a = smem_u32(mbar);
    for (uint32_t it = 0; it < maxIter; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred q;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, q;\n\t}\n"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// TMEM allocation by one full warp; the column base is written to *dst (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(dst)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(base), "r"(ncols) : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// byte offset of element (r, k) in a K-major no-swizzle block whose rows hold Kp elements
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int Kp) {
    return (uint32_t)((r >> 3) * (Kp >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

}  // namespace tc
}  // namespace gam
