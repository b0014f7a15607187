// Tensor-memory-accelerator (TMA) tile loads for the transform passes.
//
// A pass whose input is one contiguous buffer of fields (the ZI buffer
// [f][z][kyc][kx] after the z transform) reads each block's whole input
// tile with one cp.async.bulk.tensor load issued by one thread: a 4-D
// tensor map over the buffer (kx as 2 scalars per complex value, the
// compact or full axis, the other axis, the field), the tile box (2 TX
// scalars, the axis, the block's rows of the other axis, 1 field), and an
// mbarrier in shared memory that counts the tile's bytes.  Loads start on
// 16-byte boundaries: the x coordinate is 2 TX bx scalars, a multiple of
// 16 bytes for TX >= 2.  Coordinates past a tensor edge (the last row
// block) read zeros.  Tensor maps cover this GPU's memory only and the
// loads use no cluster multicast.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace hydft {

// ------------------------------------------------------------------ host
// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library links the CUDA runtime statically and not libcuda)
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_tiled_fn()
{
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// A 4-D tensor map over `fields` buffers of complex values laid out
// [field][d2][d1][pkx] (pkx complex values per row), scalar type R, box
// {2 tx, b1, b2, 1}.  Returns false when the driver refuses it (the pass
// then loads from global memory directly).
template <typename R>
inline bool make_field_tmap(CUtensorMap *m, const void *base, int pkx, int d1, int d2, int fields, int tx, int b1,
                            int b2)
{
    EncodeTiledFn fn = encode_tiled_fn();
    if (!fn || tx < 2 || b1 < 1 || b1 > 256 || b2 < 1 || b2 > 256 || 2 * tx > 256) return false;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)2 * pkx, (cuuint64_t)d1, (cuuint64_t)d2, (cuuint64_t)fields};
    const cuuint64_t row = (cuuint64_t)2 * pkx * sizeof(R);
    const cuuint64_t strides[3] = {row, row * (cuuint64_t)d1, row * (cuuint64_t)d1 * (cuuint64_t)d2};
    if (row % 16 != 0) return false;
    const cuuint32_t box[4] = {(cuuint32_t)(2 * tx), (cuuint32_t)b1, (cuuint32_t)b2, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = sizeof(R) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const CUresult r = fn(m, dt, 4, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// ---------------------------------------------------------------- device
__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of the barrier; gives up after a bounded number
// of polls (each try_wait itself suspends for a hardware-defined time) and
// returns false then.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity)
{
    for (int i = 0; i < (1 << 22); ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// one 4-D tile load of tensor map *tm at scalar coordinates (c0, c1, c2, c3)
// into shared memory at dst, completing on bar; no multicast
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, int c3,
                                            unsigned long long *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// The block's tile at src (shared memory, 128-byte aligned) written to the
// tensor of map *tm at scalar coordinates (c0, c1, c2, c3), none negative
// and c0 a multiple of 16 bytes; elements past the tensor's edges are
// clipped.  Every thread's writes of the tile come first (proxy fence and
// barrier); thread 0 issues the store and waits until it has read the tile,
// so the block's shared memory outlives the read.  No multicast.
__device__ __forceinline__ void tma_store_tile_4d(const CUtensorMap *tm, const void *src, int c0, int c1, int c2, int c3)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(
                         reinterpret_cast<uint64_t>(tm)),
                     "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
}

// One untiled bulk copy of `bytes` (a multiple of 16) from global memory
// into this CTA's shared memory, completing on bar; both addresses 16-byte
// aligned; no multicast, and the source is this GPU's memory.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Orders this thread's earlier shared-memory accesses (and those ordered
// before them by a barrier) before later bulk copies into the same space.
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace hydft
