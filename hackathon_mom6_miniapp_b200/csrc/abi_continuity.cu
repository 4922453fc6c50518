// abi_continuity.cu -- continuity PPM entry points of the reference ABI.
//
// The reference's CUDA C continuity (mom6_continuity_kernels.cu:23-1098,
// launchers :1108-1305) splits continuity_PPM into PPM edges, layer fluxes,
// column reductions, CFL limits, the Newton flux adjustment, BT_cont face
// areas, the flux thickness and the convergence.  The entry points below
// keep that split, its index ranges, its flags and its arithmetic order;
// they differ from the serial code the high-level API follows in the
// limiter (CW84 when monotonic = 1), in the double-precision tolerance
// literals, and in writing the adjusted transports once after the Newton
// loop.  A pointer whose flag is 0 is never dereferenced.
#include "../../include/mom6_cuda_c.h"
#include "abi_common.cuh"

#include <cmath>

using namespace mom6b::abi;

namespace {

struct FaceFlags {
    int vol_CFL, visc_rem, por_face;
};

// The column of one u face (i, j): pointers at layer 1, layer stride plane.
struct FaceView {
    const double *u, *hc, *hW, *hE, *vr, *por;   // hc/hW/hE at cell i; cell i+1 is +1
    size_t plane;
    double dy_Cu, IareaT_i, IareaT_ip1, IdxT_i, IdxT_ip1;
    FaceFlags f;

    __device__ double visc_rem(int k) const
    {
        return f.visc_rem ? vr[(size_t)(k - 1) * plane] : 1.0;
    }
    __device__ double dy_pfa(int k) const
    {
        return f.por_face ? dy_Cu * por[(size_t)(k - 1) * plane] : dy_Cu;
    }
};

__device__ __forceinline__ FaceView face_view(const double* u, const double* h_in,
                                              const double* h_W, const double* h_E,
                                              const double* visc_rem_u,
                                              const double* por_face_areaU,
                                              const double* dy_Cu, const double* IareaT,
                                              const double* IdxT, FaceFlags f, int i, int j,
                                              int n1, int n2)
{
    const size_t p2 = at2(i, j, n1), e2 = at2(i + 1, j, n1);
    FaceView F;
    F.u = u + p2; F.hc = h_in + p2; F.hW = h_W + p2; F.hE = h_E + p2;
    F.vr = f.visc_rem ? visc_rem_u + p2 : nullptr;
    F.por = f.por_face ? por_face_areaU + p2 : nullptr;
    F.plane = (size_t)n1 * (size_t)n2;
    F.dy_Cu = dy_Cu[p2];
    F.IareaT_i = f.vol_CFL ? IareaT[p2] : 0.0;
    F.IareaT_ip1 = f.vol_CFL ? IareaT[e2] : 0.0;
    F.IdxT_i = f.vol_CFL ? 0.0 : IdxT[p2];
    F.IdxT_ip1 = f.vol_CFL ? 0.0 : IdxT[e2];
    F.f = f;
    return F;
}

// Upwind PPM flux of layer k at face velocity ua (:218-238): returns the
// transport and sets the marginal (h_marg) and average (h_avg) thickness.
__device__ __forceinline__ double ppm_flux(const FaceView& F, int k, double ua, double dt,
                                           double dy_pfa, double& h_marg, double& h_avg)
{
    const size_t o = (size_t)(k - 1) * F.plane;
    if (ua > 0.0) {
        const double CFL = F.f.vol_CFL ? (ua * dt) * (F.dy_Cu * F.IareaT_i)
                                       : ua * dt * F.IdxT_i;
        const double hW = F.hW[o], hE = F.hE[o];
        const double curv_3 = (hW + hE) - 2.0 * F.hc[o];
        h_avg = hE + CFL * (0.5 * (hW - hE) + curv_3 * (CFL - 1.5));
        h_marg = hE + CFL * ((hW - hE) + 3.0 * curv_3 * (CFL - 1.0));
        return dy_pfa * ua * h_avg;
    }
    if (ua < 0.0) {
        const double CFL = F.f.vol_CFL ? (-ua * dt) * (F.dy_Cu * F.IareaT_ip1)
                                       : -ua * dt * F.IdxT_ip1;
        const double hW = F.hW[o + 1], hE = F.hE[o + 1];
        const double curv_3 = (hW + hE) - 2.0 * F.hc[o + 1];
        h_avg = hW + CFL * (0.5 * (hE - hW) + curv_3 * (CFL - 1.5));
        h_marg = hW + CFL * ((hE - hW) + 3.0 * curv_3 * (CFL - 1.0));
        return dy_pfa * ua * h_avg;
    }
    h_marg = 0.5 * (F.hW[o + 1] + F.hE[o]);
    h_avg = h_marg;
    return 0.0;
}

// The Newton iteration of zonal_flux_adjust_kernel_c / set_zonal_BT_cont (:505-604):
// starts from the column sums at du = 0 and returns the converged du.
__device__ double newton_du(const FaceView& F, int nz, double dt, double target,
                            double uh_err0, double duhdu_tot0, double du_max, double du_min,
                            double fac, double tol_eta_base, double tol_vel, int better_iter)
{
    const int max_itts = 20;
    double du = 0.0;
    double uh_err = uh_err0, duhdu_tot = duhdu_tot0;
    double uh_err_best = fabs(uh_err);
    bool more = true;
    for (int itt = 1; itt <= max_itts; ++itt) {
        const double tol_eta = itt <= 1   ? 1.0e-6 * tol_eta_base
                               : itt == 2 ? 1.0e-4 * tol_eta_base
                               : itt == 3 ? 1.0e-2 * tol_eta_base
                                          : tol_eta_base;
        if (uh_err > 0.0) du_max = du;
        else if (uh_err < 0.0) du_min = du;
        else more = false;
        if (more) {
            const double ae = fabs(uh_err);
            if ((fac * ae > tol_eta) ||
                (better_iter == 1 && ((ae > tol_vel * duhdu_tot) || (ae > uh_err_best)))) {
                const double ddu = -uh_err / duhdu_tot;
                const double du_prev = du;
                du = du + ddu;
                if (fabs(ddu) < 1.0e-15 * fabs(du)) {
                    more = false;
                } else if (ddu > 0.0) {
                    if (du >= du_max) {
                        du = 0.5 * (du_prev + du_max);
                        if (du_max - du_prev < 1.0e-15 * fabs(du)) more = false;
                    }
                } else if (du <= du_min) {
                    du = 0.5 * (du_prev + du_min);
                    if (du_prev - du_min < 1.0e-15 * fabs(du)) more = false;
                }
            } else {
                more = false;
            }
        }
        if (!more) break;
        uh_err = target;
        duhdu_tot = 0.0;
        for (int k = 1; k <= nz; ++k) {
            const double vr = F.visc_rem(k), dyp = F.dy_pfa(k);
            const double ua = F.u[(size_t)(k - 1) * F.plane] + du * vr;
            double hm, ha;
            const double uhk = ppm_flux(F, k, ua, dt, dyp, hm, ha);
            uh_err += uhk;
            duhdu_tot += dyp * hm * vr;
        }
        uh_err_best = fmin(uh_err_best, fabs(uh_err));
    }
    return du;
}

// Slope of the cell centred on hc with neighbours hl, hr, limited (:70-113)
__device__ __forceinline__ double ppm_slope_abi(double hl, double hc, double hr)
{
    double s = 0.5 * (hr - hl);
    const double dMx = fmax(fmax(hr, hl), hc) - hc;
    const double dMn = hc - fmin(fmin(hr, hl), hc);
    return copysign(1.0, s) * fmin(fabs(s), 2.0 * fmin(dMx, dMn));
}

} // namespace

// PPM edges with the CW84 (monotonic = 1) or positive-definite limiter;
// cells [is-1, ie+1] x [js, je], every layer (:23-161)
extern "C" void launch_ppm_reconstruction_3d_kernel(double* h_W, double* h_E, double* h_in,
                                                    double* mask2dT, int n1, int n2, int n3,
                                                    int is_l, int ie_l, int js_l, int je_l,
                                                    double h_min, int monotonic,
                                                    int upwind_1st_flag, int simple_2nd_flag,
                                                    int, int, int, int, int, int, void* stream)
{
    flush_deferred();
    run_box(clip(Box{is_l - 1, ie_l + 1, js_l, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const size_t p = at3(i, j, k, n1, n2);
                const double hi = h_in[p];
                if (upwind_1st_flag == 1) {
                    h_W[p] = hi;
                    h_E[p] = hi;
                    return;
                }
                auto H = [&](int ii) { return h_in[at3(ii, j, k, n1, n2)]; };
                auto Mk = [&](int ii) { return mask2dT[at2(ii, j, n1)]; };
                const int im1 = i - 1 >= 1 ? i - 1 : 1;
                const int ip1 = i + 1 <= n1 ? i + 1 : n1;
                const double h_l = Mk(im1) * H(im1) + (1.0 - Mk(im1)) * hi;
                const double h_r = Mk(ip1) * H(ip1) + (1.0 - Mk(ip1)) * hi;
                double hW, hE;
                if (simple_2nd_flag == 1) {
                    hW = 0.5 * (h_l + hi);
                    hE = 0.5 * (h_r + hi);
                } else {
                    double s_m = 0.0, s_c = 0.0, s_p = 0.0;
                    if (i - 2 >= 1 && (Mk(i - 2) * Mk(i - 1) * Mk(i)) != 0.0)
                        s_m = ppm_slope_abi(H(i - 2), H(i - 1), hi);
                    if (i - 1 >= 1 && i + 1 <= n1 && (Mk(i - 1) * Mk(i) * Mk(i + 1)) != 0.0)
                        s_c = ppm_slope_abi(H(i - 1), hi, H(i + 1));
                    if (i + 2 <= n1 && (Mk(i) * Mk(i + 1) * Mk(i + 2)) != 0.0)
                        s_p = ppm_slope_abi(hi, H(i + 1), H(i + 2));
                    const double oneSixth = 1.0 / 6.0;
                    hW = 0.5 * (h_l + hi) + oneSixth * (s_m - s_c);
                    hE = 0.5 * (h_r + hi) + oneSixth * (s_c - s_p);
                }
                if (monotonic == 1) {
                    if ((hE - hi) * (hi - hW) <= 0.0) {
                        hW = hi;
                        hE = hi;
                    } else {
                        const double RLdiff = hE - hW;
                        const double RLmean = 0.5 * (hE + hW);
                        const double FunFac = 6.0 * RLdiff * (hi - RLmean);
                        const double RLdiff2 = RLdiff * RLdiff;
                        if (FunFac > RLdiff2) hW = 3.0 * hi - 2.0 * hE;
                        if (FunFac < -RLdiff2) hE = 3.0 * hi - 2.0 * hW;
                    }
                } else {
                    const double curv = 3.0 * ((hW + hE) - 2.0 * hi);
                    if (curv > 0.0) {
                        const double dh = hE - hW;
                        if (fabs(dh) < curv) {
                            if (hi <= h_min) {
                                hW = hi;
                                hE = hi;
                            } else if (12.0 * curv * (hi - h_min) < (curv * curv + 3.0 * dh * dh)) {
                                const double scale =
                                    12.0 * curv * (hi - h_min) / (curv * curv + 3.0 * dh * dh);
                                hW = hi + scale * (hW - hi);
                                hE = hi + scale * (hE - hi);
                            }
                        }
                    }
                }
                h_W[p] = hW;
                h_E[p] = hE;
            });
}

// uh and duhdu per layer on faces [is-1, ie] x [js, je] (:167-239)
extern "C" void launch_zonal_flux_layer_3d_kernel(
    double* uh, double* duhdu, double* u, double* h_in, double* h_W, double* h_E, double* dy_Cu,
    double* IdxT, double* IareaT, double* por_face_areaU, double* visc_rem_u, int n1, int n2,
    int n3, int is_l, int ie_l, int js_l, int je_l, double dt, int vol_CFL_flag,
    int use_visc_rem_flag, int use_por_face_flag, int, int, int, int, int, int, void* stream)
{
    flush_deferred();
    const FaceFlags fl{vol_CFL_flag == 1, use_visc_rem_flag == 1, use_por_face_flag == 1};
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const FaceView F = face_view(u, h_in, h_W, h_E, visc_rem_u, por_face_areaU,
                                             dy_Cu, IareaT, IdxT, fl, i, j, n1, n2);
                const size_t p = at3(i, j, k, n1, n2);
                const double dyp = F.dy_pfa(k);
                double hm, ha;
                uh[p] = ppm_flux(F, k, u[p], dt, dyp, hm, ha);
                duhdu[p] = dyp * hm * F.visc_rem(k);
            });
}

// h = max(hin - dt IareaT (uh - uh(i-1)), 0) on [is, ie] x [js, je] (:245-266)
extern "C" void launch_zonal_convergence_kernel(double* h, double* hin, double* uh,
                                                double* IareaT, int n1, int n2, int n3,
                                                int is_l, int ie_l, int js_l, int je_l,
                                                double dt, int, int, int, int, int, int,
                                                void* stream)
{
    flush_deferred();
    run_box(clip(Box{is_l, ie_l, js_l, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const size_t p = at3(i, j, k, n1, n2);
                h[p] = fmax(hin[p] - dt * IareaT[at2(i, j, n1)] * (uh[p] - uh[p - 1]), 0.0);
            });
}

extern "C" void launch_visc_rem_max_kernel(double* visc_rem_max_out, double* visc_rem_u, int n1,
                                           int n2, int n3, int is_l, int ie_l, int js_l,
                                           int je_l, int use_vrm_max_flag, int, int, int, int,
                                           int, int, void* stream)
{
    flush_deferred();
    const size_t plane = (size_t)n1 * (size_t)n2;
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p2 = at2(i, j, n1);
                double vmax = 1.0;
                if (use_vrm_max_flag == 1) {
                    vmax = 0.0;
                    for (int k = 1; k <= n3; ++k)
                        vmax = fmax(vmax, visc_rem_u[p2 + (size_t)(k - 1) * plane]);
                }
                visc_rem_max_out[p2] = vmax;
            });
}

extern "C" void launch_uh_duhdu_tot_kernel(double* uh_tot_0, double* duhdu_tot_0, double* uh,
                                           double* duhdu, int n1, int n2, int n3, int is_l,
                                           int ie_l, int js_l, int je_l, int, int, int, int,
                                           int, int, void* stream)
{
    flush_deferred();
    const size_t plane = (size_t)n1 * (size_t)n2;
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p2 = at2(i, j, n1);
                double a = 0.0, b = 0.0;
                for (int k = 1; k <= n3; ++k) {
                    a += uh[p2 + (size_t)(k - 1) * plane];
                    b += duhdu[p2 + (size_t)(k - 1) * plane];
                }
                uh_tot_0[p2] = a;
                duhdu_tot_0[p2] = b;
            });
}

// Bounds on the barotropic velocity correction (:326-448)
extern "C" void launch_zonal_CFL_limits_kernel(
    double* du_max_CFL_out, double* du_min_CFL_out, double* u, double* visc_rem_u,
    double* visc_rem_max_in, double* dxT, double* areaT, double* dy_Cu, double* mask2dCu, int n1,
    int n2, int n3, int is_l, int ie_l, int js_l, int je_l, double CFL_dt, double I_dt,
    int vol_CFL_flag, int use_visc_rem_flag, int aggress_flag, int, int, int, int, int, int,
    void* stream)
{
    flush_deferred();
    const size_t plane = (size_t)n1 * (size_t)n2;
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p2 = at2(i, j, n1), e2 = at2(i + 1, j, n1);
                const double vrm = visc_rem_max_in[p2];
                const double I_vrm = vrm > 0.0 ? 1.0 / vrm : 0.0;
                double dx_W, dx_E;
                if (vol_CFL_flag == 1) {
                    dx_W = areaT[p2] / (dy_Cu[p2] + 1.0e-30);
                    if (fabs(dx_W) > 1000.0 * dxT[p2]) dx_W = 1000.0 * dxT[p2];
                    dx_E = areaT[e2] / (dy_Cu[p2] + 1.0e-30);
                    if (fabs(dx_E) > 1000.0 * dxT[e2]) dx_E = 1000.0 * dxT[e2];
                } else {
                    dx_W = dxT[p2];
                    dx_E = dxT[e2];
                }
                double du_max = 2.0 * (CFL_dt * dx_W) * I_vrm;
                double du_min = -2.0 * (CFL_dt * dx_E) * I_vrm;
                const double mCu = mask2dCu[p2];
                for (int k = 1; k <= n3; ++k) {
                    const size_t o = p2 + (size_t)(k - 1) * plane;
                    const double uk = u[o];
                    if (use_visc_rem_flag == 1) {
                        const double vr = visc_rem_u[o];
                        if (aggress_flag == 1) {
                            double lim = 0.499 * ((dx_W * I_dt - uk) + fmin(0.0, u[o - 1]));
                            if (du_max * vr > lim) du_max = lim / vr;
                            lim = 0.499 * ((-dx_E * I_dt - uk) + fmax(0.0, u[o + 1]));
                            if (du_min * vr < lim) du_min = lim / vr;
                        } else {
                            if (du_max * vr > dx_W * CFL_dt - uk * mCu)
                                du_max = (dx_W * CFL_dt - uk) / vr;
                            if (du_min * vr < -dx_E * CFL_dt - uk * mCu)
                                du_min = -(dx_E * CFL_dt + uk) / vr;
                        }
                    } else if (aggress_flag == 1) {
                        du_max = fmin(du_max, 0.499 * ((dx_W * I_dt - uk) + fmin(0.0, u[o - 1])));
                        du_min = fmax(du_min, 0.499 * ((-dx_E * I_dt - uk) + fmax(0.0, u[o + 1])));
                    } else {
                        du_max = fmin(du_max, dx_W * CFL_dt - uk);
                        du_min = fmax(du_min, -(dx_E * CFL_dt + uk));
                    }
                }
                du_max_CFL_out[p2] = fmax(du_max, 0.0);
                du_min_CFL_out[p2] = fmin(du_min, 0.0);
            });
}

// Newton adjustment of the layer transports to uhbt, then the transports at
// the converged du (:454-650)
extern "C" void launch_zonal_flux_adjust_kernel(
    double* uh, double* du_out, double* u, double* h_in, double* h_W, double* h_E, double* uhbt,
    double* visc_rem_u, double* por_face_areaU, double* IareaT, double* dy_Cu, double* IdxT,
    double* du_max_CFL_in, double* du_min_CFL_in, double* uh_tot_0_in, double* duhdu_tot_0_in,
    int n1, int n2, int n3, int is_l, int ie_l, int js_l, int je_l, double dt,
    double tol_eta_base, double tol_vel_val, int vol_CFL_flag, int use_visc_rem_flag,
    int better_iter_flag, int use_por_face_flag, int, int, int, int, int, int, void* stream)
{
    flush_deferred();
    const FaceFlags fl{vol_CFL_flag == 1, use_visc_rem_flag == 1, use_por_face_flag == 1};
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p2 = at2(i, j, n1);
                const FaceView F = face_view(u, h_in, h_W, h_E, visc_rem_u, por_face_areaU,
                                             dy_Cu, IareaT, IdxT, fl, i, j, n1, n2);
                const double fac = dt * fmin(IareaT[p2], IareaT[at2(i + 1, j, n1)]);
                const double du = newton_du(F, n3, dt, -uhbt[p2], uh_tot_0_in[p2] - uhbt[p2],
                                            duhdu_tot_0_in[p2], du_max_CFL_in[p2],
                                            du_min_CFL_in[p2], fac, tol_eta_base, tol_vel_val,
                                            better_iter_flag);
                for (int k = 1; k <= n3; ++k) {
                    const double vr = F.visc_rem(k);
                    const size_t o = p2 + (size_t)(k - 1) * F.plane;
                    double hm, ha;
                    uh[o] = ppm_flux(F, k, u[o] + du * vr, dt, F.dy_pfa(k), hm, ha);
                }
                du_out[p2] = du;
            });
}

// BT_cont face areas from a zero-transport solve and two test velocities
// (:656-992)
extern "C" void launch_set_zonal_BT_cont_kernel(
    double* FA_u_W0, double* FA_u_WW, double* uBT_WW, double* FA_u_E0, double* FA_u_EE,
    double* uBT_EE, double* u, double* h_in, double* h_W, double* h_E, double* visc_rem_u,
    double* por_face_areaU, double* IareaT, double* dy_Cu, double* IdxT, double* dxCu,
    double* visc_rem_max_in, double* du_max_CFL_in, double* du_min_CFL_in, double* uh_tot_0_in,
    double* duhdu_tot_0_in, int n1, int n2, int n3, int is_l, int ie_l, int js_l, int je_l,
    double dt, double tol_eta_base, double tol_vel_val, int vol_CFL_flag, int use_visc_rem_flag,
    int better_iter_flag, int use_por_face_flag, int, int, int, int, int, int, void* stream)
{
    flush_deferred();
    const FaceFlags fl{vol_CFL_flag == 1, use_visc_rem_flag == 1, use_por_face_flag == 1};
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p2 = at2(i, j, n1);
                const FaceView F = face_view(u, h_in, h_W, h_E, visc_rem_u, por_face_areaU,
                                             dy_Cu, IareaT, IdxT, fl, i, j, n1, n2);
                const double fac = dt * fmin(IareaT[p2], IareaT[at2(i + 1, j, n1)]);
                const double du0 = newton_du(F, n3, dt, 0.0, uh_tot_0_in[p2],
                                             duhdu_tot_0_in[p2], du_max_CFL_in[p2],
                                             du_min_CFL_in[p2], fac, tol_eta_base, tol_vel_val,
                                             better_iter_flag);
                const double Idt = 1.0 / dt;
                const double du_CFL = (1.0e-6 * Idt) * dxCu[p2];
                double duR = fmin(0.0, du0 - du_CFL);
                double duL = fmax(0.0, du0 + du_CFL);
                const double vrm = visc_rem_max_in[p2];
                for (int k = 1; k <= n3; ++k) {
                    const double vr = F.visc_rem(k);
                    const double lim = fmax(vr, 0.1 * vrm);
                    if (lim > 0.0) {
                        const double uk = u[p2 + (size_t)(k - 1) * F.plane];
                        if (uk + duR * lim > -du_CFL * vr) duR = -(uk + du_CFL * vr) / lim;
                        if (uk + duL * lim < du_CFL * vr) duL = -(uk - du_CFL * vr) / lim;
                    }
                }
                double FAmt_0 = 0.0, FAmt_L = 0.0, FAmt_R = 0.0, uhtot_L = 0.0, uhtot_R = 0.0;
                for (int k = 1; k <= n3; ++k) {
                    const double vr = F.visc_rem(k), dyp = F.dy_pfa(k);
                    const double uk = u[p2 + (size_t)(k - 1) * F.plane];
                    double hm, ha;
                    ppm_flux(F, k, uk + du0 * vr, dt, dyp, hm, ha);
                    FAmt_0 += dyp * hm * vr;
                    const double uL = ppm_flux(F, k, uk + duL * vr, dt, dyp, hm, ha);
                    FAmt_L += dyp * hm * vr;
                    uhtot_L += uL;
                    const double uR = ppm_flux(F, k, uk + duR * vr, dt, dyp, hm, ha);
                    FAmt_R += dyp * hm * vr;
                    uhtot_R += uR;
                }
                double FA_0 = FAmt_0, FA_avg = FAmt_0;
                if ((duL - du0) != 0.0) FA_avg = uhtot_L / (duL - du0);
                if (FA_avg > fmax(FA_0, FAmt_L)) FA_avg = fmax(FA_0, FAmt_L);
                else if (FA_avg < fmin(FA_0, FAmt_L)) FA_0 = FA_avg;
                FA_u_W0[p2] = FA_0;
                FA_u_WW[p2] = FAmt_L;
                uBT_WW[p2] = (fabs(FA_0 - FAmt_L) <= 1.0e-12 * FA_0)
                                 ? 0.0
                                 : (1.5 * (duL - du0)) * ((FAmt_L - FA_avg) / (FAmt_L - FA_0));
                FA_0 = FAmt_0;
                FA_avg = FAmt_0;
                if ((duR - du0) != 0.0) FA_avg = uhtot_R / (duR - du0);
                if (FA_avg > fmax(FA_0, FAmt_R)) FA_avg = fmax(FA_0, FAmt_R);
                else if (FA_avg < fmin(FA_0, FAmt_R)) FA_0 = FA_avg;
                FA_u_E0[p2] = FA_0;
                FA_u_EE[p2] = FAmt_R;
                uBT_EE[p2] = (fabs(FAmt_R - FA_0) <= 1.0e-12 * FA_0)
                                 ? 0.0
                                 : (1.5 * (duR - du0)) * ((FAmt_R - FA_avg) / (FAmt_R - FA_0));
            });
}

// h_u: marginal or average face thickness per layer (:998-1066)
extern "C" void launch_zonal_flux_thickness_kernel(
    double* h_u, double* u, double* h, double* h_W, double* h_E, double* por_face_areaU,
    double* visc_rem_u, double* IareaT, double* IdxT, double* dy_Cu, int n1, int n2, int n3,
    int is_l, int ie_l, int js_l, int je_l, double dt, int vol_CFL_flag, int marginal_flag,
    int has_visc_rem_flag, int use_por_face_flag, int, int, int, int, int, int, void* stream)
{
    flush_deferred();
    const FaceFlags fl{vol_CFL_flag == 1, has_visc_rem_flag == 1, use_por_face_flag == 1};
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const FaceView F = face_view(u, h, h_W, h_E, visc_rem_u, por_face_areaU, dy_Cu,
                                             IareaT, IdxT, fl, i, j, n1, n2);
                const size_t p = at3(i, j, k, n1, n2);
                double hm, ha;
                ppm_flux(F, k, u[p], dt, F.dy_Cu, hm, ha);
                double r = marginal_flag == 1 ? hm : ha;
                if (fl.visc_rem && fl.por_face) r *= visc_rem_u[p] * por_face_areaU[p];
                else if (fl.visc_rem) r *= visc_rem_u[p];
                else if (fl.por_face) r *= por_face_areaU[p];
                h_u[p] = r;
            });
}

extern "C" void launch_u_cor_kernel(double* u_cor, double* u, double* du, double* visc_rem_u,
                                    int n1, int n2, int n3, int is_l, int ie_l, int js_l,
                                    int je_l, int use_visc_rem_flag, int, int, int, int, int,
                                    int, void* stream)
{
    flush_deferred();
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const size_t p = at3(i, j, k, n1, n2);
                if (use_visc_rem_flag == 1) u_cor[p] = u[p] + du[at2(i, j, n1)] * visc_rem_u[p];
                else u_cor[p] = u[p] + du[at2(i, j, n1)];
            });
}
