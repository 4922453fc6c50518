// abi_common.cuh -- index-box launch helpers of the reference-compatible ABI.
//
// Every launch_* entry point covers one or more rectangular index ranges of
// the (n1, n2[, n3]) Fortran arrays.  run_box() launches a grid-stride kernel
// over the union of those ranges (i fastest, so a warp reads 32 consecutive
// doubles of a row) and calls a device lambda at each (i, j, k); the lambda
// tests the sub-ranges itself.  The caller's grid/block arguments are not
// used: the box is the contract, not the launch geometry.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>

namespace mom6b {
namespace abi {

// 1-based Fortran indexing with 64-bit offsets.
__device__ __forceinline__ size_t at2(int i, int j, int n1)
{
    return (size_t)(j - 1) * (size_t)n1 + (size_t)(i - 1);
}
__device__ __forceinline__ size_t at3(int i, int j, int k, int n1, int n2)
{
    return ((size_t)(k - 1) * (size_t)n2 + (size_t)(j - 1)) * (size_t)n1 + (size_t)(i - 1);
}
// f_4_u / f_4_v: (4, n1, n2), component c in 1..4
__device__ __forceinline__ size_t at4(int c, int i, int j, int n1)
{
    return ((size_t)(j - 1) * (size_t)n1 + (size_t)(i - 1)) * 4 + (size_t)(c - 1);
}

struct Box {
    int i0, i1, j0, j1;  // inclusive, 1-based
};

// Clip a box to the allocated array [1, n1] x [1, n2].
inline Box clip(Box b, int n1, int n2)
{
    return Box{std::max(b.i0, 1), std::min(b.i1, n1), std::max(b.j0, 1), std::min(b.j1, n2)};
}

template <class F>
__global__ void __launch_bounds__(256) k_box(Box b, F f)
{
    const int w = b.i1 - b.i0 + 1;
    const long long n = (long long)w * (long long)(b.j1 - b.j0 + 1);
    const int k = 1 + (int)blockIdx.y;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = b.i0 + (int)(t % w);
        const int j = b.j0 + (int)(t / w);
        f(i, j, k);
    }
}

// Launch f over box b (already clipped) for layers 1..nk (nk = 1 for 2-D).
template <class F>
inline void run_box(Box b, int nk, void* stream, F f)
{
    if (b.i1 < b.i0 || b.j1 < b.j0 || nk < 1) return;
    const long long n = (long long)(b.i1 - b.i0 + 1) * (long long)(b.j1 - b.j0 + 1);
    long long blocks = (n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    dim3 grid((unsigned)blocks, (unsigned)nk, 1);
    k_box<<<grid, 256, 0, (cudaStream_t)stream>>>(b, f);
}

// The barotropic deferral (abi_barotropic.cu): the launch_bt_* calls of one
// btstep_cuda_c are recorded from launch_bt_init_kernel on and run as one
// persistent loop at launch_bt_copy_output_kernel.  Every other entry point
// and every runtime helper first replays an open record call by call, so the
// device state any of them can observe is the reference sequence's.
void flush_deferred();

} // namespace abi
} // namespace mom6b
