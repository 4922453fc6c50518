// cont_impl.cuh -- pieces of continuity_PPM shared by the exact and the fast
// FP64 continuity kernels (k_continuity.cu, k_cont_fast.cu): the PPM edge
// values of a cell and one iteration of zonal_flux_adjust's Newton solve.
//
// The FP32 quirks of the serial source are kept: the real(4) locals of
// PPM_limit_pos (mom6_continuity_serial.F90:1266-1268) and the default-real
// literals 1e-6, 1e-4, 1e-2, 1e-15, 1e-12 and 0.1 (F32(x) is the double
// value of the single-precision literal).
#pragma once

#include "kernels.h"

namespace mom6b {

#define F32(x) ((double)(x##f))

// The PPM slope of a cell from h of its two neighbours (ppm_slope's
// operations; ok = the product of the three masks is nonzero).
__device__ __forceinline__ double ppm_slope3(double hm, double hc, double hp, bool ok)
{
    if (!ok) return 0.0;
    const double s = 0.5 * (hp - hm);
    const double dMx = dmax(dmax(hp, hm), hc) - hc;
    const double dMn = hc - dmin(dmin(hp, hm), hc);
    return copysign(1.0, s) * dmin(fabs(s), 2.0 * dmin(dMx, dMn));
}

// Edge values of a cell from h of the cell and its neighbours, their masks
// (ml, mr; oml = 1 - ml, omr = 1 - mr) and the slopes of cells i-1, i, i+1:
// the rest of PPM_reconstruction_x and PPM_limit_pos (ppm_cell's operations).
// FAST: the limiter's quotient (rounded to single precision) by div_nr.
template <bool FAST = false>
__device__ __forceinline__ void ppm_edges_limited(double hm1, double hc, double hp1, double ml,
                                                  double oml, double mr, double omr, double slm,
                                                  double slc, double slp, double h_min,
                                                  double& hL, double& hR)
{
    const double oneSixth = 1.0 / 6.0;
    const double h_im1 = ml * hm1 + oml * hc;
    const double h_ip1 = mr * hp1 + omr * hc;
    hL = 0.5 * (h_im1 + hc) + oneSixth * (slm - slc);
    hR = 0.5 * (h_ip1 + hc) + oneSixth * (slc - slp);
    float curv = (float)(3.0 * ((hL + hR) - 2.0 * hc));
    if ((double)curv > 0.0) {
        float dh = (float)(hR - hL);
        if (fabsf(dh) < curv) {
            if (hc <= h_min) {
                hL = hc; hR = hc;
            } else {
                float c12 = __fmul_rn(12.0f, curv);
                float den = __fadd_rn(__fmul_rn(curv, curv), __fmul_rn(3.0f, __fmul_rn(dh, dh)));
                double lhs = (double)c12 * (hc - h_min);
                if (lhs < (double)den) {
                    float scale;
                    if constexpr (FAST) scale = (float)div_nr(lhs, (double)den);
                    else scale = (float)(lhs / (double)den);
                    hL = hc + (double)scale * (hL - hc);
                    hR = hc + (double)scale * (hR - hc);
                }
            }
        }
    }
}

// PPM_reconstruction_x + PPM_limit_pos for one cell from its 5-cell stencil
// (h[0..4] = cells i-2..i+2, m[0..4] their masks); same operations as ppm_cell.
__device__ __forceinline__ void ppm_stencil(const double* h, const double* m, double h_min,
                                            double& hL, double& hR)
{
    const double slm = ppm_slope3(h[0], h[1], h[2], (m[0] * m[1] * m[2]) != 0.0);
    const double slc = ppm_slope3(h[1], h[2], h[3], (m[1] * m[2] * m[3]) != 0.0);
    const double slp = ppm_slope3(h[2], h[3], h[4], (m[2] * m[3] * m[4]) != 0.0);
    ppm_edges_limited(h[1], h[2], h[3], m[1], 1.0 - m[1], m[3], 1.0 - m[3], slm, slc, slp,
                      h_min, hL, hR);
}


// State of one zonal_flux_adjust iteration (:813-903) for one face.
struct Newton {
    double du, du_max, du_min, uh_err, duhdu_tot, uh_err_best;
    bool live;  // the iteration loop has not exited yet
};

__device__ __forceinline__ Newton newton_start(double uh_err, double duhdu_tot,
                                               double du_max_CFL, double du_min_CFL, bool live)
{
    return Newton{0.0, du_max_CFL, du_min_CFL, uh_err, duhdu_tot, fabs(uh_err), live};
}

// Iteration itt of zonal_flux_adjust up to its exit test (:829-883): bounds
// the root, takes the Newton (or bisection) step; returns do_I.  FAST: the
// Newton step's quotient by div_nr.
template <bool FAST = false>
__device__ __forceinline__ bool newton_iter(Newton& S, int itt, double tol_eta_dt_fac)
{
    const double tol_eta_cs = 1.0e-12, tol_vel = 3.0e8;
    double tol_eta;
    if (itt <= 1) tol_eta = F32(1e-6) * tol_eta_cs;
    else if (itt == 2) tol_eta = F32(1e-4) * tol_eta_cs;
    else if (itt == 3) tol_eta = F32(1e-2) * tol_eta_cs;
    else tol_eta = tol_eta_cs;
    bool do_I = true;
    if (S.uh_err > 0.0) S.du_max = S.du;
    else if (S.uh_err < 0.0) S.du_min = S.du;
    else do_I = false;
    if (do_I) {
        double ae = fabs(S.uh_err);
        if ((tol_eta_dt_fac * ae > tol_eta) ||
            ((ae > tol_vel * S.duhdu_tot) || (ae > S.uh_err_best))) {
            double ddu;
            // (div_nr wants a normal divisor; a column without thickness keeps
            // the IEEE quotient's infinity, which the bounds then catch)
            if (FAST && fabs(S.duhdu_tot) > 1.0e-300) ddu = -div_nr(S.uh_err, S.duhdu_tot);
            else ddu = -(S.uh_err / S.duhdu_tot);
            double du_prev = S.du;
            S.du = S.du + ddu;
            if (fabs(ddu) < F32(1.0e-15) * fabs(S.du)) {
                do_I = false;
            } else if (ddu > 0.0) {
                if (S.du >= S.du_max) {
                    S.du = 0.5 * (du_prev + S.du_max);
                    if (S.du_max - du_prev < F32(1.0e-15) * fabs(S.du)) do_I = false;
                }
            } else {
                if (S.du <= S.du_min) {
                    S.du = 0.5 * (du_prev + S.du_min);
                    if (du_prev - S.du_min < F32(1.0e-15) * fabs(S.du)) do_I = false;
                }
            }
        } else {
            do_I = false;
        }
    }
    return do_I;
}

} // namespace mom6b
