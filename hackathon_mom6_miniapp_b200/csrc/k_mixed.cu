// k_mixed.cu -- the mixed-precision form of the split RK2 step.
//
// State (u, v, h and the intermediate up, vp, uh, h_u, PPM edges) is stored
// in FP32, which halves the bytes the bandwidth-bound kernels move, and the
// stencil arithmetic is FP32.  Double precision is kept where accumulation
// or conditioning needs it:
//   continuity  the per-face column sums (uh_tot, duhdu_tot, the BT_cont face
//               areas), the Newton scalars and the thickness update
//               h = max(hin - dt IareaT (uh(I) - uh(I-1)), 0);
//   vertvisc    the tridiagonal elimination (b1, d1, c1, the eliminated
//               velocity, the back substitution) and the bottom stress; the
//               coefficients are FP32.  An opt-in variant eliminates in FP32
//               too (the system is diagonally dominant);
//   btstep      runs in FP64 (its 2-D state is a few MB and its cost is the
//               latency of the substep loop, not bytes).
// This file is built with FMA contraction (the FP64 files are not), and the
// FP32 Newton iteration uses a tolerance suited to FP32 fluxes (below).
#include "mixed_impl.cuh"
#include "tendency_impl.cuh"
#include "vertvisc_impl.cuh"

namespace mom6b {

cudaError_t launch_tendency_f(const Dims& D, const Metrics& M, const UniMetrics& U,
                              const float* uin, const float* vin, const float* h,
                              const float* ubase, const float* vbase, float* uout,
                              float* vout, float coef, float h_neglect, cudaStream_t s)
{
    return launch_tendency_t<float>(D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef,
                                    h_neglect, s);
}

cudaError_t launch_vertvisc_f(const Dims& D, const Metrics& M, float* u, float* v,
                              const float* h, double dt, const VVParams& P, double* taux_bot,
                              double* tauy_bot, cudaStream_t s, bool f32_elim)
{
    if (f32_elim)
        return launch_vertvisc_pf_t<float, float>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
    return launch_vertvisc_pf_t<float, double>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
}

__global__ void __launch_bounds__(128)
k_ppm_edges_warp_f(Dims D, Metrics M, const float* __restrict__ hin, float* __restrict__ hW,
                   float* __restrict__ hE, float h_min)
{
    ppm_cells_warp_f(D, M, hin, hW, hE, h_min,
                     (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5),
                     D.js + (int)blockIdx.y, 1 + (int)blockIdx.z * kEdgeLayersF);
}

// AS: the column sweeps stage the next chunk in shared memory with cp.async.
template <int MINB, bool AS = false>
__global__ void __launch_bounds__(128, MINB)
k_cont_faces_f(Dims D, Metrics M, const float* __restrict__ u, const float* __restrict__ hin,
               const float* __restrict__ hW, const float* __restrict__ hE,
               const double* __restrict__ uhbt2d, ContOutF O, float* ovl_all, double dt)
{
    __shared__ float stage[AS ? 2 * kMixCH * 7 * 128 : 1];
    cont_faces_f(D, M, u, hin, hW, hE, uhbt2d, O, ovl_all, dt, (int)blockIdx.x,
                 (int)blockIdx.y, (int)gridDim.x, AS ? stage : nullptr);
}

cudaError_t launch_continuity_f(const Dims& D, const Metrics& M, const float* u,
                                const float* hin, float* hW, float* hE, const double* uhbt,
                                float* h, float* uh, float* h_u, const ContOut& O2,
                                double* uh_ovl, double dt, double h_min, cudaStream_t s)
{
    {
        const int n = (D.ie + 1) - (D.is - 1) + 1;
        const int warps = (n + kEdgeCellsPerWarpF - 1) / kEdgeCellsPerWarpF;
        dim3 grid((warps + 3) / 4, D.je - D.js + 1, (D.nk + kEdgeLayersF - 1) / kEdgeLayersF);
        k_ppm_edges_warp_f<<<grid, 128, 0, s>>>(D, M, hin, hW, hE, (float)h_min);
    }
    ContOutF O{h, uh, h_u, O2.FA_u_W0, O2.FA_u_WW, O2.FA_u_E0, O2.FA_u_EE, O2.uBT_WW,
               O2.uBT_EE, O2.du_cor};
    const int nb = 128, step = nb - 1;
    const int nfaces = D.ie - (D.is - 1) + 1;
    dim3 grid((nfaces - 1 + step - 1) / step, D.je - D.js + 1, 1);
    // 6 CTAs per SM, chunks loaded into registers: 2.19 ms per step at
    // 720x720x75 (5 CTAs: 2.23, 4: 2.38; staging the sweeps in shared memory
    // with cp.async: 2.30 and 2.38)
    k_cont_faces_f<6><<<grid, nb, 0, s>>>(D, M, u, hin, hW, hE, uhbt, O, (float*)uh_ovl, dt);
    return cudaGetLastError();
}

} // namespace mom6b
