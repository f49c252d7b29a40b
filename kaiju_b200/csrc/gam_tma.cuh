// Tensor-memory-accelerator (TMA) staging of pencil planes into shared memory.
//
// Host side: a 3-D tiled tensor map over one plane of the pencil layout -- dimensions (Ni+1, Nj+1, Nk+1),
// i fastest, row pitch P and plane pitch P*Q elements -- with a box of (bx, by, bz) elements; elements of
// the box outside those dimensions arrive as zeros. The encoder is the driver's cuTensorMapEncodeTiled,
// reached through the runtime's driver entry point (no link against the driver library).
//
// Device side: one thread arms an mbarrier with the byte count of all the boxes of a tile and issues the
// copies (cp.async.bulk.tensor, tile mode, no multicast); every thread then waits on the mbarrier with a
// bounded number of polls. A copy's x coordinate times the element size must be a multiple of 16 bytes;
// the launch code checks that before it chooses this path.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "gam_common.cuh"
#include "gam_tc.cuh"

namespace gam {
namespace tma {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// the encoder, looked up once (a function-local static: initialised once even when several host threads
// create handles at the same time); null when the driver does not provide it
inline EncodeTiledFn encoder() {
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<EncodeTiledFn>(p);
        return nullptr;
    }();
    return fn;
}

// Tensor map of one plane (element size 4 or 8 bytes) with the given box; false if it cannot be made
inline bool plane_map(CUtensorMap* m, const void* plane, int esize, const Lay& L, int bx, int by, int bz) {
    EncodeTiledFn enc = encoder();
    if (!enc || !plane || (reinterpret_cast<uintptr_t>(plane) & 15)) return false;
    cuuint64_t dim[3] = {(cuuint64_t)L.Ni + 1, (cuuint64_t)L.Nj + 1, (cuuint64_t)L.Nk + 1};
    cuuint64_t stride[2] = {(cuuint64_t)L.P * esize, (cuuint64_t)L.P * L.Q * esize};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
    cuuint32_t es[3] = {1, 1, 1};
    CUtensorMapDataType dt = esize == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    return enc(m, dt, 3, const_cast<void*>(plane), dim, stride, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// make an mbarrier initialisation visible to the asynchronous proxy before any copy completes on it
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// this thread's arrival, announcing the bytes the copies of the phase will deliver
__device__ __forceinline__ void arrive_expect_tx(uint64_t* mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(tc::smem_u32(mbar)), "r"(bytes)
                 : "memory");
}
// box at (x, y, z) of the tensor map into shared memory at dst; completes its bytes on mbar
__device__ __forceinline__ void load3(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        :: "r"(tc::smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(tc::smem_u32(mbar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

}  // namespace tma
}  // namespace gam
