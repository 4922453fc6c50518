// tma.cuh -- Tensor Memory Accelerator tiles of the reference-layout fields.
//
// A 3-D field (n1, n2, nk) of doubles, column-major (i fastest), is described
// to the TMA unit as a tensor of dimensions {n1, n2, nk} with byte strides
// {8 n1, 8 n1 n2}; a box {W, 1, nk} is one j-row segment of W points over all
// layers, landing in shared memory as [nk][W].  The unit requires the strides
// to be multiples of 16 bytes (n1 even) and the innermost box extent in bytes
// to be a multiple of 16 (W even), and a load must start at an even x (an
// x offset times 8 bytes that is a multiple of 16): callers round x down to
// even and read the wider box.  Points outside the tensor read as zero.
//
// Loads complete on an mbarrier (transaction bytes); every wait is bounded by
// a clock64 budget so a load that never lands cannot hang the kernel.  No
// multicast form is used.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mom6b {

__device__ __forceinline__ uint32_t tma_smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void tma_bar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tma_smem_u32(bar)),
                 "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void tma_bar_expect(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                     tma_smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool tma_bar_try(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(tma_smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase of the given parity; false once `budget` cycles passed.
__device__ __forceinline__ bool tma_bar_wait(uint64_t* bar, uint32_t parity, long long budget)
{
    if (tma_bar_try(bar, parity)) return true;
    const long long t0 = clock64();
    while (!tma_bar_try(bar, parity))
        if (clock64() - t0 > budget) return false;
    return true;
}

// 3-D tiled load of the box at (x, y, z) into shared memory, completing on bar.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y,
                                           int z, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(tma_smem_u32(dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(tma_smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

// Host: the tensor map of a (n1, n2, nk) double field read in boxes of
// {box_w, 1, nk}.  cudaErrorNotSupported when the layout does not meet the
// unit's alignment rules (odd n1, misaligned base, box beyond 256).
cudaError_t tma_map_field3d(CUtensorMap* map, const double* base, int n1, int n2, int nk,
                            int box_w);
// The same field read in boxes of {box_w, box_h, box_d} (landing as
// [box_d][box_h][box_w]); tma_map_cached keeps one map per (address, shape,
// box) and returns false when the layout does not qualify.
cudaError_t tma_map_box3d(CUtensorMap* map, const double* base, int n1, int n2, int nk,
                          int box_w, int box_h, int box_d);
bool tma_map_cached(const double* base, int n1, int n2, int nk, int box_w, int box_h,
                    int box_d, CUtensorMap* out);

} // namespace mom6b
