// k_continuity.cu -- zonal PPM continuity (FP64), serial-driver semantics.
//
// Restates continuity_PPM of mom6_continuity_serial.F90:100-1294 as
// rk2_serial_driver calls it (:293, :380):
//   k_ppm_edges   PPM_reconstruction_x + PPM_limit_pos (:1124-1294), one
//                 thread per cell, h_W/h_E to a scratch pair;
//   k_cont_faces  one thread per u face (I, j): zonal_flux_layer (:516-598),
//                 the CFL limits of zonal_mass_flux (:322-433),
//                 zonal_flux_adjust (:739-916), u_cor/du_cor, set_zonal_BT_cont
//                 (:920-1121), zonal_flux_thickness (:602-735), and finally
//                 continuity_zonal_convergence (:148-176) for the cells whose
//                 two faces belong to the CTA (CTAs overlap by one face).
//
// The serial code iterates a whole row with a shared do_I mask and exits when
// no face of the row needs more work; a face whose do_I is false is never
// touched again, so each face's iteration is independent of its neighbours
// and a per-face loop gives the same result.
//
// visc_rem_u and por_face_areaU are identically 1 in the driver
// (continuity_init, :63-64); every multiplication and division by them is
// exact and is omitted.  With uhbt = 0 on a face, set_zonal_BT_cont's
// zero-transport Newton solve repeats zonal_flux_adjust's iteration exactly,
// so du0 = du there and the second solve is skipped; u_0 then equals u_cor,
// and h_u is the marginal thickness already evaluated for FA_u_0.
//
// The FP32 quirks of the serial source are kept: the real(4) locals of
// PPM_limit_pos and the default-real literals 1e-6, 1e-4, 1e-2, 1e-15, 1e-12
// and 0.1.
#include <cstdlib>

#include "kernels.h"

namespace mom6b {

#define F32(x) ((double)(x##f))

// ---------------------------------------------------------------------------
// PPM edge values
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ppm_slope(const double* __restrict__ hrow,
                                            const double* __restrict__ mrow, int i)
{
    // hrow/mrow point at element i=1 of the row (1-based access below)
    if ((mrow[i - 2] * mrow[i - 1] * mrow[i]) == 0.0) return 0.0;
    double hp = hrow[i], hm = hrow[i - 2], hc = hrow[i - 1];
    double s = 0.5 * (hp - hm);
    double dMx = dmax(dmax(hp, hm), hc) - hc;
    double dMn = hc - dmin(dmin(hp, hm), hc);
    return copysign(1.0, s) * dmin(fabs(s), 2.0 * dmin(dMx, dMn));
}

__global__ void __launch_bounds__(128)
k_ppm_edges(Dims D, Metrics M, const double* __restrict__ hin,
            double* __restrict__ hW, double* __restrict__ hE, double h_min)
{
    const int i = D.is - 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = D.js + (int)blockIdx.y;
    const int k = 1 + (int)blockIdx.z;
    if (i > D.ie + 1) return;
    const size_t rowoff = (size_t)(k - 1) * D.plane + (size_t)(j - 1) * D.n1;
    const double* hrow = hin + rowoff;                    // hrow[i-1] = h(i)
    const double* mrow = M.mask2dT + (size_t)(j - 1) * D.n1;
    const double oneSixth = 1.0 / 6.0;
    double slm = ppm_slope(hrow, mrow, i - 1);
    double slc = ppm_slope(hrow, mrow, i);
    double slp = ppm_slope(hrow, mrow, i + 1);
    double hc = hrow[i - 1];
    double h_im1 = mrow[i - 2] * hrow[i - 2] + (1.0 - mrow[i - 2]) * hc;
    double h_ip1 = mrow[i] * hrow[i] + (1.0 - mrow[i]) * hc;
    double hL = 0.5 * (h_im1 + hc) + oneSixth * (slm - slc);
    double hR = 0.5 * (h_ip1 + hc) + oneSixth * (slc - slp);
    // PPM_limit_pos with real(4) curv, dh, scale (:1266-1268)
    float curv = (float)(3.0 * ((hL + hR) - 2.0 * hc));
    if ((double)curv > 0.0) {
        float dh = (float)(hR - hL);
        if (fabsf(dh) < curv) {
            if (hc <= h_min) {
                hL = hc; hR = hc;
            } else {
                float c12 = __fmul_rn(12.0f, curv);
                float den = __fadd_rn(__fmul_rn(curv, curv),
                                      __fmul_rn(3.0f, __fmul_rn(dh, dh)));
                double lhs = (double)c12 * (hc - h_min);
                if (lhs < (double)den) {
                    float scale = (float)(lhs / (double)den);
                    hL = hc + (double)scale * (hL - hc);
                    hR = hc + (double)scale * (hR - hc);
                }
            }
        }
    }
    hW[rowoff + (i - 1)] = hL;
    hE[rowoff + (i - 1)] = hR;
}

// ---------------------------------------------------------------------------
// face column work
// ---------------------------------------------------------------------------
struct FaceCol {
    const double* u;     // u(I, j, 1), layer stride = plane
    const double* hc;    // h(I, j, 1)   (cell i = I)
    const double* hWc;   // h_W(I, j, 1)
    const double* hEc;   // h_E(I, j, 1)
    size_t plane;
    double dy;           // dy_Cu(I, j) (times por_face_areaU = 1)
    double IdxT_i, IdxT_ip1;
};

// zonal_flux_layer (:554-583) for one layer; returns uh and sets h_marg.
// The two upwind cases are one operation sequence on (base, other, h) =
// (h_E(i), h_W(i), h(i)) for u > 0 or (h_W(i+1), h_E(i+1), h(i+1)) for u < 0,
// and CFL = (|u| dt) Idx equals the reference's -(u dt Idx) for u < 0 exactly,
// so the evaluation is written without a divergent branch.
__device__ __forceinline__ double flux_eval(const FaceCol& F, int k, double uI,
                                            double dt, double& h_marg)
{
    const size_t o = (size_t)(k - 1) * F.plane;
    const double hWi = F.hWc[o], hEi = F.hEc[o], hi = F.hc[o];
    const double hWp = F.hWc[o + 1], hEp = F.hEc[o + 1], hp = F.hc[o + 1];
    const bool pos = uI > 0.0;
    const double base = pos ? hEi : hWp;
    const double oth = pos ? hWi : hEp;
    const double hc = pos ? hi : hp;
    const double Idx = pos ? F.IdxT_i : F.IdxT_ip1;
    const double CFL = fabs(uI) * dt * Idx;
    const double curv_3 = (oth + base) - 2.0 * hc;
    const double uh = F.dy * uI * (base + CFL * (0.5 * (oth - base) + curv_3 * (CFL - 1.5)));
    const double hm = base + CFL * ((oth - base) + 3.0 * curv_3 * (CFL - 1.0));
    const bool zero = !(uI > 0.0) && !(uI < 0.0);
    h_marg = zero ? 0.5 * (hWp + hEi) : hm;
    return zero ? 0.0 : uh;
}

// zonal_flux_adjust for one face (:813-903).  When uh_out is given the flux of
// every evaluated iteration is stored (the present(uh_3d) call).
__device__ double flux_adjust_face(const FaceCol& F, int nz, double dt,
                                   double uhbt, double uh_tot_0,
                                   double duhdu_tot_0, double du_max_CFL,
                                   double du_min_CFL, double tol_eta_dt_fac,
                                   double* uh_out, size_t uh_stride)
{
    const int max_itts = 20;
    const double tol_eta_cs = 1.0e-12, tol_vel = 3.0e8;
    double du = 0.0;
    bool do_I = true;
    double du_max = du_max_CFL, du_min = du_min_CFL;
    double uh_err = uh_tot_0 - uhbt;
    double duhdu_tot = duhdu_tot_0;
    double uh_err_best = fabs(uh_err);
    for (int itt = 1; itt <= max_itts; ++itt) {
        double tol_eta;
        if (itt <= 1) tol_eta = F32(1e-6) * tol_eta_cs;
        else if (itt == 2) tol_eta = F32(1e-4) * tol_eta_cs;
        else if (itt == 3) tol_eta = F32(1e-2) * tol_eta_cs;
        else tol_eta = tol_eta_cs;
        if (uh_err > 0.0) du_max = du;
        else if (uh_err < 0.0) du_min = du;
        else do_I = false;
        if (do_I) {
            double ae = fabs(uh_err);
            if ((tol_eta_dt_fac * ae > tol_eta) ||
                ((ae > tol_vel * duhdu_tot) || (ae > uh_err_best))) {
                double ddu = -(uh_err / duhdu_tot);
                double du_prev = du;
                du = du + ddu;
                if (fabs(ddu) < F32(1.0e-15) * fabs(du)) {
                    do_I = false;
                } else if (ddu > 0.0) {
                    if (du >= du_max) {
                        du = 0.5 * (du_prev + du_max);
                        if (du_max - du_prev < F32(1.0e-15) * fabs(du)) do_I = false;
                    }
                } else {
                    if (du <= du_min) {
                        du = 0.5 * (du_prev + du_min);
                        if (du_prev - du_min < F32(1.0e-15) * fabs(du)) do_I = false;
                    }
                }
            } else {
                do_I = false;
            }
        }
        if (!do_I) break;
        const bool update = itt < max_itts;
        if (update || uh_out) {
            double e = -uhbt, dt_sum = 0.0;
            for (int k = 1; k <= nz; ++k) {
                const size_t o = (size_t)(k - 1) * F.plane;
                double u_new = F.u[o] + du;
                double hm;
                double uhk = flux_eval(F, k, u_new, dt, hm);
                double duhdu = F.dy * hm;
                if (uh_out) uh_out[(size_t)(k - 1) * uh_stride] = uhk;
                e = e + uhk;
                dt_sum = dt_sum + duhdu;
            }
            if (update) {
                uh_err = e;
                duhdu_tot = dt_sum;
                uh_err_best = dmin(uh_err_best, fabs(uh_err));
            }
        }
    }
    return du;
}


// blockDim.x faces per CTA along I; consecutive CTAs overlap by one face.
// Face ownership: thread 0 recomputes the last face of the CTA to its left
// (it owns face is-1 only in the first CTA) and keeps that face's transport
// column in shared memory, so no CTA ever reads a global transport another
// CTA may still be iterating on.
__global__ void __launch_bounds__(128)
k_cont_faces(Dims D, Metrics M, const double* __restrict__ u,
             const double* __restrict__ hin, const double* __restrict__ hW,
             const double* __restrict__ hE, const double* __restrict__ uhbt2d,
             ContOut O, double dt)
{
    extern __shared__ double s_uh_left[];  // [nk], transports of thread 0's face
    const int nz = D.nk;
    const int step = (int)blockDim.x - 1;
    const int I = D.is - 1 + (int)blockIdx.x * step + (int)threadIdx.x;
    const int j = D.js + (int)blockIdx.y;
    const bool face_ok = I <= D.ie;
    const bool owner = threadIdx.x >= 1 || blockIdx.x == 0;
    if (face_ok) {
        const size_t f0 = (size_t)(j - 1) * D.n1 + (I - 1);
        FaceCol F;
        F.u = u + f0; F.hc = hin + f0; F.hWc = hW + f0; F.hEc = hE + f0;
        F.plane = (size_t)D.plane;
        F.dy = MOM6B_A2(M.dy_Cu, I, j, D);
        F.IdxT_i = MOM6B_A2(M.IdxT, I, j, D);
        F.IdxT_ip1 = MOM6B_A2(M.IdxT, I + 1, j, D);
        double* uh = (threadIdx.x == 0) ? s_uh_left : O.uh + f0;
        const size_t ust = (threadIdx.x == 0) ? 1 : F.plane;

        // initial fluxes and their column sums (:305-355)
        double uh_tot_0 = 0.0, duhdu_tot_0 = 0.0;
        for (int k = 1; k <= nz; ++k) {
            const size_t o = (size_t)(k - 1) * F.plane;
            double hm;
            double uhk = flux_eval(F, k, F.u[o], dt, hm);
            uh[(size_t)(k - 1) * ust] = uhk;
            duhdu_tot_0 = duhdu_tot_0 + F.dy * hm;
            uh_tot_0 = uh_tot_0 + uhk;
        }
        // CFL limits (:335-433), vol_CFL = aggress_adjust = .false.
        const double CFL_dt = 0.5 / dt;
        const double dx_W = MOM6B_A2(M.dxT, I, j, D), dx_E = MOM6B_A2(M.dxT, I + 1, j, D);
        const double mCu = MOM6B_A2(M.mask2dCu, I, j, D);
        double du_max_CFL = 2.0 * (CFL_dt * dx_W);
        double du_min_CFL = -(2.0 * (CFL_dt * dx_E));
        for (int k = 1; k <= nz; ++k) {
            double uk = F.u[(size_t)(k - 1) * F.plane];
            if (du_max_CFL > dx_W * CFL_dt - uk * mCu) du_max_CFL = dx_W * CFL_dt - uk;
            if (du_min_CFL < -(dx_E * CFL_dt) - uk * mCu) du_min_CFL = -(dx_E * CFL_dt + uk);
        }
        du_max_CFL = dmax(du_max_CFL, 0.0);
        du_min_CFL = dmin(du_min_CFL, 0.0);

        const double fac = dt * dmin(MOM6B_A2(M.IareaT, I, j, D), MOM6B_A2(M.IareaT, I + 1, j, D));
        const double uhbt = MOM6B_A2(uhbt2d, I, j, D);
        double du = flux_adjust_face(F, nz, dt, uhbt, uh_tot_0, duhdu_tot_0,
                                     du_max_CFL, du_min_CFL, fac, uh, ust);
        if (owner) {
            if (threadIdx.x == 0)  // face is-1 of the first CTA: publish its column
                for (int k = 1; k <= nz; ++k)
                    O.uh[f0 + (size_t)(k - 1) * F.plane] = s_uh_left[k - 1];
            O.du_cor[f0] = du;

            // set_zonal_BT_cont (:991-1121)
            double du0 = (uhbt == 0.0)
                             ? du
                             : flux_adjust_face(F, nz, dt, 0.0, uh_tot_0, duhdu_tot_0,
                                                du_max_CFL, du_min_CFL, fac, nullptr, 0);
            const double Idt = 1.0 / dt;
            const double du_CFL = (F32(1e-6) * Idt) * MOM6B_A2(M.dxCu, I, j, D);
            double duR = dmin(0.0, du0 - du_CFL);
            double duL = dmax(0.0, du0 + du_CFL);
            // visc_rem_lim = max(1, 0.1 * 1) = 1 > 0 on every layer
            for (int k = 1; k <= nz; ++k) {
                double uk = F.u[(size_t)(k - 1) * F.plane];
                if (uk + duR > -du_CFL) duR = -(uk + du_CFL);
                if (uk + duL < du_CFL) duL = -(uk - du_CFL);
            }
            double FAmt_0 = 0.0, FAmt_L = 0.0, FAmt_R = 0.0, uhtot_L = 0.0, uhtot_R = 0.0;
            double* h_u = O.h_u + f0;
            const bool same = (du0 == du);
            for (int k = 1; k <= nz; ++k) {
                const size_t o = (size_t)(k - 1) * F.plane;
                double uk = F.u[o];
                double hm0, hmL, hmR;
                flux_eval(F, k, uk + du0, dt, hm0);
                double uhL = flux_eval(F, k, uk + duL, dt, hmL);
                double uhR = flux_eval(F, k, uk + duR, dt, hmR);
                FAmt_0 = FAmt_0 + F.dy * hm0;
                FAmt_L = FAmt_L + F.dy * hmL;
                FAmt_R = FAmt_R + F.dy * hmR;
                uhtot_L = uhtot_L + uhL;
                uhtot_R = uhtot_R + uhR;
                // zonal_flux_thickness with u_cor = u + du (marginal faces)
                double hmc = hm0;
                if (!same) flux_eval(F, k, uk + du, dt, hmc);
                h_u[o] = hmc;
            }
            double FA_0 = FAmt_0, FA_avg = FAmt_0;
            if ((duL - du0) != 0.0) FA_avg = uhtot_L / (duL - du0);
            if (FA_avg > dmax(FA_0, FAmt_L)) FA_avg = dmax(FA_0, FAmt_L);
            else if (FA_avg < dmin(FA_0, FAmt_L)) FA_0 = FA_avg;
            O.FA_u_W0[f0] = FA_0;
            O.FA_u_WW[f0] = FAmt_L;
            O.uBT_WW[f0] = (fabs(FA_0 - FAmt_L) <= F32(1e-12) * FA_0)
                               ? 0.0
                               : (1.5 * (duL - du0)) * ((FAmt_L - FA_avg) / (FAmt_L - FA_0));
            FA_0 = FAmt_0; FA_avg = FAmt_0;
            if ((duR - du0) != 0.0) FA_avg = uhtot_R / (duR - du0);
            if (FA_avg > dmax(FA_0, FAmt_R)) FA_avg = dmax(FA_0, FAmt_R);
            else if (FA_avg < dmin(FA_0, FAmt_R)) FA_0 = FA_avg;
            O.FA_u_E0[f0] = FA_0;
            O.FA_u_EE[f0] = FAmt_R;
            O.uBT_EE[f0] = (fabs(FAmt_R - FA_0) <= F32(1e-12) * FA_0)
                               ? 0.0
                               : (1.5 * (duR - du0)) * ((FAmt_R - FA_avg) / (FAmt_R - FA_0));
        }
    }
    __syncthreads();  // the CTA's transport columns are complete and visible
    // continuity_zonal_convergence for cell i = I (faces I-1 and I in this CTA)
    const int i = I;
    if (threadIdx.x >= 1 && i >= D.is && i <= D.ie) {
        const size_t c0 = (size_t)(j - 1) * D.n1 + (i - 1);
        const double fac = dt * MOM6B_A2(M.IareaT, i, j, D);
        for (int k = 1; k <= nz; ++k) {
            const size_t o = (size_t)(k - 1) * D.plane + c0;
            double uh_left = (threadIdx.x == 1) ? s_uh_left[k - 1] : O.uh[o - 1];
            O.h[o] = dmax(hin[o] - fac * (O.uh[o] - uh_left), 0.0);
        }
    }
}

// CTAs per SM for k_cont_faces; 0 lets the hardware fill the SM.
constexpr int kContCtasPerSM = 0;

cudaError_t launch_continuity(const Dims& D, const Metrics& M, const double* u,
                              const double* hin, double* hW, double* hE,
                              const double* uhbt, const ContOut& O, double dt,
                              double h_min, cudaStream_t s)
{
    {
        int n = (D.ie + 1) - (D.is - 1) + 1;
        dim3 grid((n + 127) / 128, D.je - D.js + 1, D.nk);
        k_ppm_edges<<<grid, 128, 0, s>>>(D, M, hin, hW, hE, h_min);
    }
    {
        // Residency: each face re-reads its column on every Newton pass, so
        // the resident CTAs' columns should stay in L2.  The dynamic shared
        // memory request is padded to cap the CTAs per SM (kContCtasPerSM).
        const int nb = 128, step = nb - 1;
        int nfaces = D.ie - (D.is - 1) + 1;
        dim3 grid((nfaces - 1 + step - 1) / step, D.je - D.js + 1, 1);
        size_t smem = (size_t)D.nk * sizeof(double);
        static int ctas = -1;
        if (ctas < 0) {
            const char* e = getenv("MOM6B_CONT_CTAS_PER_SM");
            ctas = e ? atoi(e) : kContCtasPerSM;
        }
        if (ctas > 0) {
            size_t pad = (size_t)(227 * 1024) / (size_t)ctas - 1024;
            if (pad > smem) smem = pad;
        }
        cudaError_t e = cudaFuncSetAttribute(k_cont_faces,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        k_cont_faces<<<grid, nb, smem, s>>>(D, M, u, hin, hW, hE, uhbt, O, dt);
    }
    return cudaGetLastError();
}

} // namespace mom6b
