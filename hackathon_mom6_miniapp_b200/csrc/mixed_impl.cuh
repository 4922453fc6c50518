// mixed_impl.cuh -- device code of the mixed-precision continuity: FP32 PPM
// edges and upwind fluxes with FP64 column sums, Newton scalars and thickness
// update.  Shared by the single-domain launchers (k_mixed.cu) and the batched
// ensemble kernels (k_ensemble.cu); both are built with FMA contraction, so
// a domain gets the same arithmetic either way.
//
// Restates continuity_PPM of mom6_continuity_serial.F90:100-1294 (zonal):
// PPM_reconstruction_x + PPM_limit_pos (:1124-1294), zonal_flux_layer
// (:516-598), zonal_flux_adjust (:739-916), set_zonal_BT_cont (:920-1121),
// zonal_flux_thickness (:602-735) and continuity_zonal_convergence (:148-176).
#pragma once

#include "kernels.h"

namespace mom6b {

// ---------------------------------------------------------------------------
// FP32 continuity
// ---------------------------------------------------------------------------
// Newton tolerance of the FP32 form: the adjustment stops when the implied
// sea-surface change dt * IareaT * |uh_err| is below kMixedTolEta metres (the
// FP64 form follows the serial schedule 1e-18 .. 1e-12 m, below what FP32
// fluxes resolve), or when the step is below kMixedRelStep of |du|.
constexpr double kMixedTolEta = 1.0e-6;
constexpr double kMixedRelStep = 1.0e-6;

// The FP32 PPM slope of a cell from h of its neighbours (ok = the product of
// the three masks is nonzero).
__device__ __forceinline__ float ppm_slope3_f(float hm, float hc, float hp, bool ok)
{
    if (!ok) return 0.0f;
    const float s = 0.5f * (hp - hm);
    const float dMx = fmaxf(fmaxf(hp, hm), hc) - hc;
    const float dMn = hc - fminf(fminf(hp, hm), hc);
    return copysignf(1.0f, s) * fminf(fabsf(s), 2.0f * fminf(dMx, dMn));
}

// FP32 edge values of a cell from h of the cell and its neighbours, their
// masks and the slopes of cells i-1, i, i+1 (PPM_reconstruction_x and
// PPM_limit_pos).
__device__ __forceinline__ void ppm_edges_f(float hm1, float hc, float hp1, float ml, float mr,
                                            float slm, float slc, float slp, float h_min,
                                            float& hL, float& hR)
{
    const float oneSixth = 1.0f / 6.0f;
    const float h_im1 = ml * hm1 + (1.0f - ml) * hc;
    const float h_ip1 = mr * hp1 + (1.0f - mr) * hc;
    hL = 0.5f * (h_im1 + hc) + oneSixth * (slm - slc);
    hR = 0.5f * (h_ip1 + hc) + oneSixth * (slc - slp);
    const float curv = 3.0f * ((hL + hR) - 2.0f * hc);
    if (curv > 0.0f) {
        const float dh = hR - hL;
        if (fabsf(dh) < curv) {
            if (hc <= h_min) {
                hL = hc; hR = hc;
            } else if (12.0f * curv * (hc - h_min) < curv * curv + 3.0f * dh * dh) {
                const float scale = 12.0f * curv * (hc - h_min) / (curv * curv + 3.0f * dh * dh);
                hL = hc + scale * (hL - hc);
                hR = hc + scale * (hR - hc);
            }
        }
    }
}

// PPM_reconstruction_x + PPM_limit_pos in FP32 for one cell of a row: cell
// i = is-1 + bx * blockDim.x + tx of row j = js + by, layer k = 1 + bz.
__device__ __forceinline__ void ppm_cell_f(const Dims& D, const Metrics& M,
                                           const float* __restrict__ hin,
                                           float* __restrict__ hW, float* __restrict__ hE,
                                           float h_min, int bx, int by, int bz)
{
    const int i = D.is - 1 + bx * (int)blockDim.x + (int)threadIdx.x;
    const int j = D.js + by;
    const int k = 1 + bz;
    if (i > D.ie + 1) return;
    const size_t row = (size_t)(k - 1) * D.plane + (size_t)(j - 1) * D.n1;
    float h[5], m[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        h[c] = hin[row + (i - 3 + c)];
        m[c] = (float)M.mask2dT[(size_t)(j - 1) * D.n1 + (i - 3 + c)];
    }
    const float slm = ppm_slope3_f(h[0], h[1], h[2], (m[0] * m[1] * m[2]) != 0.0f);
    const float slc = ppm_slope3_f(h[1], h[2], h[3], (m[1] * m[2] * m[3]) != 0.0f);
    const float slp = ppm_slope3_f(h[2], h[3], h[4], (m[2] * m[3] * m[4]) != 0.0f);
    float hL, hR;
    ppm_edges_f(h[1], h[2], h[3], m[1], m[3], slm, slc, slp, h_min, hL, hR);
    hW[row + (i - 1)] = hL;
    hE[row + (i - 1)] = hR;
}

// The same edges with each cell's slope formed once (the warp layout of the
// FP64 k_ppm_edges_warp): lane l takes cell c = is - 2 + 30 w + l, lanes
// 1..30 write their cells' edges, kEdgeLayersF layers per thread.
constexpr int kEdgeCellsPerWarpF = 30;
constexpr int kEdgeLayersF = 5;

__device__ __forceinline__ void ppm_cells_warp_f(const Dims& D, const Metrics& M,
                                                 const float* __restrict__ hin,
                                                 float* __restrict__ hW, float* __restrict__ hE,
                                                 float h_min, int wrow, int j, int k0)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = (int)threadIdx.x & 31;
    const int c = D.is - 2 + kEdgeCellsPerWarpF * wrow + lane;
    const bool load_ok = c <= D.ie + 2;
    const bool write_ok = lane >= 1 && lane <= kEdgeCellsPerWarpF && c <= D.ie + 1;
    const size_t r = (size_t)(j - 1) * D.n1 + (size_t)(c - 1);
    const double* mrow = M.mask2dT + r;
    const float m0 = load_ok ? (float)mrow[-1] : 0.0f;
    const float m1 = load_ok ? (float)mrow[0] : 0.0f;
    const float m2 = load_ok ? (float)mrow[1] : 0.0f;
    const bool slope_ok = (m0 * m1 * m2) != 0.0f;
    const int kn = min(kEdgeLayersF, D.nk - k0 + 1);
    const float* hp0 = hin + (size_t)(k0 - 1) * D.plane + r;
    float hm[kEdgeLayersF], hc[kEdgeLayersF], hp[kEdgeLayersF];
#pragma unroll
    for (int q = 0; q < kEdgeLayersF; ++q) {
        const float* p = hp0 + (size_t)q * D.plane;
        const bool ok = load_ok && q < kn;
        hm[q] = ok ? p[-1] : 0.0f;
        hc[q] = ok ? p[0] : 0.0f;
        hp[q] = ok ? p[1] : 0.0f;
    }
#pragma unroll
    for (int q = 0; q < kEdgeLayersF; ++q) {
        if (q < kn) {
            const float slc = ppm_slope3_f(hm[q], hc[q], hp[q], slope_ok);
            const float slm = __shfl_up_sync(FULL, slc, 1);
            const float slp = __shfl_down_sync(FULL, slc, 1);
            float hL, hR;
            ppm_edges_f(hm[q], hc[q], hp[q], m0, m2, slm, slc, slp, h_min, hL, hR);
            if (write_ok) {
                const size_t o = (size_t)(k0 - 1 + q) * D.plane + r;
                hW[o] = hL;
                hE[o] = hR;
            }
        }
    }
}

struct LayerF {
    float u, hWi, hEi, hi, hWp, hEp, hp;
};

struct FaceF {
    const float *u, *hc, *hW, *hE;
    size_t plane;
    float dy, Idx_i, Idx_p, dt;
    // this thread's staging slots (nullptr: chunks are loaded into registers);
    // slot (b, c, f) at st[((b * kMixCH + c) * 7 + f) * sts]
    float* st = nullptr;
    int sts = 0;
    __device__ LayerF load(int k) const
    {
        const size_t o = (size_t)(k - 1) * plane;
        return LayerF{u[o], hW[o], hE[o], hc[o], hW[o + 1], hE[o + 1], hc[o + 1]};
    }
    // the face's last pass: u and the edges with the evict-first hint
    __device__ LayerF load_last(int k) const
    {
        const size_t o = (size_t)(k - 1) * plane;
        return LayerF{__ldcs(u + o), __ldcs(hW + o), __ldcs(hE + o), hc[o],
                      __ldcs(hW + o + 1), __ldcs(hE + o + 1), hc[o + 1]};
    }
    // upwind PPM transport and marginal thickness at face velocity uI
    __device__ float eval(const LayerF& L, float uI, float& hm) const
    {
        const bool pos = uI > 0.0f;
        const float base = pos ? L.hEi : L.hWp, oth = pos ? L.hWi : L.hEp;
        const float hcl = pos ? L.hi : L.hp, Idx = pos ? Idx_i : Idx_p;
        const float CFL = fabsf(uI) * dt * Idx;
        const float curv_3 = (oth + base) - 2.0f * hcl;
        const float uh = dy * uI * (base + CFL * (0.5f * (oth - base) + curv_3 * (CFL - 1.5f)));
        const float hmm = base + CFL * ((oth - base) + 3.0f * curv_3 * (CFL - 1.0f));
        const bool zero = !(uI > 0.0f) && !(uI < 0.0f);
        hm = zero ? 0.5f * (L.hWp + L.hEi) : hmm;
        return zero ? 0.0f : uh;
    }
};

constexpr int kMixCH = 4;

template <bool LAST = false, typename Fn>
__device__ __forceinline__ void mix_layers(const FaceF& F, int nz, Fn&& fn)
{
    if (F.st) {
        // the next chunk's seven values copied with cp.async while the
        // current chunk is evaluated
        auto slot = [&](int b, int c, int f) -> float& {
            return F.st[(size_t)((b * kMixCH + c) * 7 + f) * F.sts];
        };
        auto stage = [&](int kt, int b) {
#pragma unroll
            for (int c = 0; c < kMixCH; ++c) {
                const int k = kt + c;
                const bool ok = k <= nz;
                const size_t o = ok ? (size_t)(k - 1) * F.plane : 0;
                cp_async_elem(&slot(b, c, 0), F.u + o, ok);
                cp_async_elem(&slot(b, c, 1), F.hW + o, ok);
                cp_async_elem(&slot(b, c, 2), F.hE + o, ok);
                cp_async_elem(&slot(b, c, 3), F.hc + o, ok);
                cp_async_elem(&slot(b, c, 4), F.hW + o + 1, ok);
                cp_async_elem(&slot(b, c, 5), F.hE + o + 1, ok);
                cp_async_elem(&slot(b, c, 6), F.hc + o + 1, ok);
            }
            cp_async_commit();
        };
        stage(1, 0);
        for (int kt = 1, it = 0; kt <= nz; kt += kMixCH, ++it) {
            const int b = it & 1;
            if (kt + kMixCH <= nz) {
                stage(kt + kMixCH, b ^ 1);
                cp_async_wait_prior();
            } else {
                cp_async_wait_all();
            }
            LayerF L[kMixCH];
#pragma unroll
            for (int c = 0; c < kMixCH; ++c)
                L[c] = LayerF{slot(b, c, 0), slot(b, c, 1), slot(b, c, 2), slot(b, c, 3),
                              slot(b, c, 4), slot(b, c, 5), slot(b, c, 6)};
#pragma unroll
            for (int c = 0; c < kMixCH; ++c)
                if (kt + c <= nz) fn(kt + c, L[c]);
        }
        return;
    }
    for (int kt = 1; kt <= nz; kt += kMixCH) {
        LayerF L[kMixCH];
#pragma unroll
        for (int c = 0; c < kMixCH; ++c)
            if (kt + c <= nz) L[c] = LAST ? F.load_last(kt + c) : F.load(kt + c);
#pragma unroll
        for (int c = 0; c < kMixCH; ++c)
            if (kt + c <= nz) fn(kt + c, L[c]);
    }
}

// One zonal_flux_adjust iteration on FP32 fluxes with FP64 sums.
struct NewtonF {
    double du, du_max, du_min, uh_err, duhdu_tot, best;
    bool live;
};

__device__ __forceinline__ bool mix_iter(NewtonF& S, double fac)
{
    bool more = true;
    if (S.uh_err > 0.0) S.du_max = S.du;
    else if (S.uh_err < 0.0) S.du_min = S.du;
    else more = false;
    if (more) {
        const double ae = fabs(S.uh_err);
        if (fac * ae > kMixedTolEta || ae > S.best) {
            const double ddu = -(S.uh_err / S.duhdu_tot);
            const double du_prev = S.du;
            S.du = S.du + ddu;
            if (fabs(ddu) < kMixedRelStep * fabs(S.du)) {
                more = false;
            } else if (ddu > 0.0) {
                if (S.du >= S.du_max) {
                    S.du = 0.5 * (du_prev + S.du_max);
                    if (S.du_max - du_prev < kMixedRelStep * fabs(S.du)) more = false;
                }
            } else if (S.du <= S.du_min) {
                S.du = 0.5 * (du_prev + S.du_min);
                if (du_prev - S.du_min < kMixedRelStep * fabs(S.du)) more = false;
            }
        } else {
            more = false;
        }
    }
    return more;
}

// The face's two solves in lockstep, one column pass per iteration: A toward
// uhbt, keeping its last evaluated transports in uh (stride ust); B toward
// zero transport (set_zonal_BT_cont), when live.
static __device__ void mix_adjust_pair(const FaceF& F, int nz, double uhbt, double fac, NewtonF& A,
                                NewtonF& B, float* uh, size_t ust)
{
    for (int itt = 1; itt <= 20; ++itt) {
        if (A.live) A.live = mix_iter(A, fac);
        if (B.live) B.live = mix_iter(B, fac);
        const bool pa = A.live, pb = B.live;
        if (!pa && !pb) break;
        double eA = -uhbt, sA = 0.0, eB = 0.0, sB = 0.0;
        const float fA = (float)A.du, fB = (float)B.du;
        mix_layers(F, nz, [&](int k, const LayerF& L) {
            if (pa) {
                float hm;
                const float t = F.eval(L, L.u + fA, hm);
                uh[(size_t)(k - 1) * ust] = t;
                eA += (double)t;
                sA += (double)(F.dy * hm);
            }
            if (pb) {
                float hm;
                const float t = F.eval(L, L.u + fB, hm);
                eB += (double)t;
                sB += (double)(F.dy * hm);
            }
        });
        if (pa) {
            A.uh_err = eA; A.duhdu_tot = sA; A.best = fmin(A.best, fabs(eA));
        }
        if (pb) {
            B.uh_err = eB; B.duhdu_tot = sB; B.best = fmin(B.best, fabs(eB));
        }
    }
}

struct ContOutF {
    float *h, *uh, *h_u;
    double *FA_u_W0, *FA_u_WW, *FA_u_E0, *FA_u_EE, *uBT_WW, *uBT_EE, *du_cor;
};

// One thread per u face, blockDim.x - 1 faces per CTA, consecutive CTAs
// overlapping by one face whose transports thread 0 keeps in its CTA's slot of
// ovl.  (bx, by) are the CTA's block coordinates, gx the CTAs per row.
__device__ __forceinline__ void cont_faces_f(const Dims& D, const Metrics& M,
                                             const float* __restrict__ u,
                                             const float* __restrict__ hin,
                                             const float* __restrict__ hW,
                                             const float* __restrict__ hE,
                                             const double* __restrict__ uhbt2d,
                                             const ContOutF& O, float* ovl_all, double dt,
                                             int bx, int by, int gx, float* stage = nullptr)
{
    const int nz = D.nk;
    const int I = D.is - 1 + bx * ((int)blockDim.x - 1) + (int)threadIdx.x;
    const int j = D.js + by;
    const bool face_ok = I <= D.ie;
    const bool owner = threadIdx.x >= 1 || bx == 0;
    float* ovl = ovl_all + ((size_t)by * gx + bx) * (size_t)nz;
    const size_t plane = (size_t)D.plane;
    if (face_ok) {
        const size_t f0 = (size_t)(j - 1) * D.n1 + (I - 1);
        FaceF F{u + f0, hin + f0, hW + f0, hE + f0, plane,
                (float)MOM6B_A2(M.dy_Cu, I, j, D), (float)MOM6B_A2(M.IdxT, I, j, D),
                (float)MOM6B_A2(M.IdxT, I + 1, j, D), (float)dt};
        if (stage) {
            F.st = stage + threadIdx.x;
            F.sts = (int)blockDim.x;
        }
        float* uh = owner ? O.uh + f0 : ovl;
        const size_t ust = owner ? plane : 1;
        // initial fluxes, column sums, CFL limits
        double uh_tot_0 = 0.0, duhdu_tot_0 = 0.0;
        const double CFL_dt = 0.5 / dt;
        const double dx_W = MOM6B_A2(M.dxT, I, j, D), dx_E = MOM6B_A2(M.dxT, I + 1, j, D);
        const double mCu = MOM6B_A2(M.mask2dCu, I, j, D);
        double du_max_CFL = 2.0 * (CFL_dt * dx_W), du_min_CFL = -(2.0 * (CFL_dt * dx_E));
        mix_layers(F, nz, [&](int k, const LayerF& L) {
            float hm;
            const float t = F.eval(L, L.u, hm);
            uh[(size_t)(k - 1) * ust] = t;
            uh_tot_0 += (double)t;
            duhdu_tot_0 += (double)(F.dy * hm);
            const double uk = (double)L.u;
            if (du_max_CFL > dx_W * CFL_dt - uk * mCu) du_max_CFL = dx_W * CFL_dt - uk;
            if (du_min_CFL < -(dx_E * CFL_dt) - uk * mCu) du_min_CFL = -(dx_E * CFL_dt + uk);
        });
        du_max_CFL = fmax(du_max_CFL, 0.0);
        du_min_CFL = fmin(du_min_CFL, 0.0);
        const double fac = dt * fmin(MOM6B_A2(M.IareaT, I, j, D), MOM6B_A2(M.IareaT, I + 1, j, D));
        const double uhbt = MOM6B_A2(uhbt2d, I, j, D);
        const bool solve0 = owner && uhbt != 0.0;
        const double e0 = uh_tot_0 - uhbt;
        NewtonF A{0.0, du_max_CFL, du_min_CFL, e0, duhdu_tot_0, fabs(e0), true};
        NewtonF B{0.0, du_max_CFL, du_min_CFL, uh_tot_0, duhdu_tot_0, fabs(uh_tot_0), solve0};
        mix_adjust_pair(F, nz, uhbt, fac, A, B, uh, ust);
        const double du = A.du;
        if (owner) {
            O.du_cor[f0] = du;
            const double du0 = solve0 ? B.du : du;
            const double du_CFL = (1.0e-6 / dt) * MOM6B_A2(M.dxCu, I, j, D);
            double duR = fmin(0.0, du0 - du_CFL), duL = fmax(0.0, du0 + du_CFL);
            for (int k = 1; k <= nz; ++k) {
                const double uk = (double)u[f0 + (size_t)(k - 1) * plane];
                if (uk + duR > -du_CFL) duR = -(uk + du_CFL);
                if (uk + duL < du_CFL) duL = -(uk - du_CFL);
            }
            double FAmt_0 = 0.0, FAmt_L = 0.0, FAmt_R = 0.0, uhtot_L = 0.0, uhtot_R = 0.0;
            const float d0 = (float)du0, dL = (float)duL, dR = (float)duR, dc = (float)du;
            const bool same = du0 == du;
            mix_layers<true>(F, nz, [&](int k, const LayerF& L) {
                float hm0, hmL, hmR;
                F.eval(L, L.u + d0, hm0);
                const float uL = F.eval(L, L.u + dL, hmL);
                const float uR = F.eval(L, L.u + dR, hmR);
                FAmt_0 += (double)(F.dy * hm0);
                FAmt_L += (double)(F.dy * hmL);
                FAmt_R += (double)(F.dy * hmR);
                uhtot_L += (double)uL;
                uhtot_R += (double)uR;
                float hmc = hm0;
                if (!same) F.eval(L, L.u + dc, hmc);
                __stcs(O.h_u + f0 + (size_t)(k - 1) * plane, hmc);
            });
            double FA_0 = FAmt_0, FA_avg = FAmt_0;
            if ((duL - du0) != 0.0) FA_avg = uhtot_L / (duL - du0);
            if (FA_avg > fmax(FA_0, FAmt_L)) FA_avg = fmax(FA_0, FAmt_L);
            else if (FA_avg < fmin(FA_0, FAmt_L)) FA_0 = FA_avg;
            O.FA_u_W0[f0] = FA_0;
            O.FA_u_WW[f0] = FAmt_L;
            O.uBT_WW[f0] = (fabs(FA_0 - FAmt_L) <= 1e-12 * FA_0)
                               ? 0.0
                               : (1.5 * (duL - du0)) * ((FAmt_L - FA_avg) / (FAmt_L - FA_0));
            FA_0 = FAmt_0; FA_avg = FAmt_0;
            if ((duR - du0) != 0.0) FA_avg = uhtot_R / (duR - du0);
            if (FA_avg > fmax(FA_0, FAmt_R)) FA_avg = fmax(FA_0, FAmt_R);
            else if (FA_avg < fmin(FA_0, FAmt_R)) FA_0 = FA_avg;
            O.FA_u_E0[f0] = FA_0;
            O.FA_u_EE[f0] = FAmt_R;
            O.uBT_EE[f0] = (fabs(FAmt_R - FA_0) <= 1e-12 * FA_0)
                               ? 0.0
                               : (1.5 * (duR - du0)) * ((FAmt_R - FA_avg) / (FAmt_R - FA_0));
        }
    }
    __syncthreads();  // the CTA's transports are complete and visible
    // thickness update in FP64 for cell i = I (faces I-1 and I in this CTA)
    const int i = I;
    if (threadIdx.x >= 1 && i >= D.is && i <= D.ie) {
        const size_t c0 = (size_t)(j - 1) * D.n1 + (i - 1);
        const double fac = dt * MOM6B_A2(M.IareaT, i, j, D);
        const bool from_ovl = threadIdx.x == 1 && bx > 0;
        for (int k = 1; k <= nz; ++k) {
            const size_t o = (size_t)(k - 1) * plane + c0;
            const double left = from_ovl ? (double)ovl[k - 1] : (double)O.uh[o - 1];
            __stcs(O.h + o, (float)fmax((double)hin[o] - fac * ((double)O.uh[o] - left), 0.0));
        }
    }
}

} // namespace mom6b
