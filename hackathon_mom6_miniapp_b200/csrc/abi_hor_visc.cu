// abi_hor_visc.cu -- launch_stress_kernel / launch_divergence_kernel.
//
// Laplacian horizontal viscosity as the reference's CUDA C backend splits it
// (mom6_hor_visc_kernels.cu:30-150, launchers :157-204): stresses at h and q
// points, then their divergence.  Same ranges and operation order as the
// reference kernels.
#include "../../include/mom6_cuda_c.h"
#include "abi_common.cuh"

using namespace mom6b::abi;

extern "C" void launch_stress_kernel(double* str_xx, double* str_xy, double* u, double* v,
                                     double* h, double* DY_dxT, double* DX_dyT, double* DY_dxBu,
                                     double* DX_dyBu, double* IdyCu, double* IdxCu,
                                     double* IdyCv, double* IdxCv, double* mask2dBu,
                                     double* reduction_xx, double* reduction_xy, double Kh_bg,
                                     int n1, int n2, int n3, int is_l, int ie_l, int js_l,
                                     int je_l, int, int, int, int, int, int, void* stream)
{
    flush_deferred();
    // str_xx on [is-1, ie+1] x [js-1, je+1], str_xy on [is-1, ie] x [js-1, je]
    const int Isq = is_l - 1, Ieq = ie_l, Jsq = js_l - 1, Jeq = je_l;
    run_box(clip(Box{Isq, Ieq + 1, Jsq, Jeq + 1}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const size_t p2 = at2(i, j, n1), p = at3(i, j, k, n1, n2);
                {
                    const size_t w2 = at2(i - 1, j, n1), s2 = at2(i, j - 1, n1);
                    const double dudx = DY_dxT[p2] * (IdyCu[p2] * u[p] -
                                                      IdyCu[w2] * u[at3(i - 1, j, k, n1, n2)]);
                    const double dvdy = DX_dyT[p2] * (IdxCv[p2] * v[p] -
                                                      IdxCv[s2] * v[at3(i, j - 1, k, n1, n2)]);
                    const double sh_xx = dudx - dvdy;
                    str_xx[p] = -Kh_bg * sh_xx * h[p] * reduction_xx[p2];
                }
                if (i <= Ieq && j <= Jeq) {
                    const size_t e2 = at2(i + 1, j, n1), n2_ = at2(i, j + 1, n1);
                    const size_t pe = at3(i + 1, j, k, n1, n2), pn = at3(i, j + 1, k, n1, n2);
                    const double dvdx = DY_dxBu[p2] * (v[pe] * IdyCv[e2] - v[p] * IdyCv[p2]);
                    const double dudy = DX_dyBu[p2] * (u[pn] * IdxCu[n2_] - u[p] * IdxCu[p2]);
                    const double sh_xy = mask2dBu[p2] * (dvdx + dudy);
                    const double hq = 0.25 * ((h[p] + h[at3(i + 1, j + 1, k, n1, n2)]) +
                                              (h[pe] + h[pn]));
                    str_xy[p] = -Kh_bg * sh_xy * hq * mask2dBu[p2] * reduction_xy[p2];
                }
            });
}

extern "C" void launch_divergence_kernel(double* diffu, double* diffv, double* str_xx,
                                         double* str_xy, double* h, double* mask2dT,
                                         double* IdyCu, double* IdxCu, double* IdyCv,
                                         double* IdxCv, double* IareaCu, double* IareaCv,
                                         double* dy2h, double* dx2h, double* dy2q, double* dx2q,
                                         double h_neglect, int n1, int n2, int n3, int is_l,
                                         int ie_l, int js_l, int je_l, int, int, int, int, int,
                                         int, void* stream)
{
    flush_deferred();
    // diffu on [is-1, ie] x [js, je], diffv on [is, ie] x [js-1, je]
    run_box(clip(Box{is_l - 1, ie_l, js_l - 1, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const size_t p2 = at2(i, j, n1), p = at3(i, j, k, n1, n2);
                if (j >= js_l) {
                    const size_t e2 = at2(i + 1, j, n1), pe = at3(i + 1, j, k, n1, n2);
                    const double h_u = 0.5 * (mask2dT[p2] * h[p] + mask2dT[e2] * h[pe]);
                    const double by_xy = dx2q[at2(i, j - 1, n1)] * str_xy[at3(i, j - 1, k, n1, n2)] -
                                         dx2q[p2] * str_xy[p];
                    const double by_xx = dy2h[p2] * str_xx[p] - dy2h[e2] * str_xx[pe];
                    diffu[p] = ((IdxCu[p2] * by_xy + IdyCu[p2] * by_xx) * IareaCu[p2]) /
                               (h_u + h_neglect);
                }
                if (i >= is_l) {
                    const size_t n2_ = at2(i, j + 1, n1), pn = at3(i, j + 1, k, n1, n2);
                    const double h_v = 0.5 * (mask2dT[p2] * h[p] + mask2dT[n2_] * h[pn]);
                    const double by_xy = dy2q[at2(i - 1, j, n1)] * str_xy[at3(i - 1, j, k, n1, n2)] -
                                         dy2q[p2] * str_xy[p];
                    const double by_xx = dx2h[p2] * str_xx[p] - dx2h[n2_] * str_xx[pn];
                    diffv[p] = ((IdyCv[p2] * by_xy - IdxCv[p2] * by_xx) * IareaCv[p2]) /
                               (h_v + h_neglect);
                }
            });
}
