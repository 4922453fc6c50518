// k_cont_fast.cu -- zonal continuity_PPM, the fast FP64 form.
//
// The algorithm of k_continuity.cu (continuity_PPM of
// mom6_continuity_serial.F90:100-1294 as rk2_serial_driver calls it: PPM
// edges and PPM_limit_pos, the initial fluxes and CFL limits of
// zonal_mass_flux, zonal_flux_adjust's Newton solve, set_zonal_BT_cont,
// zonal_flux_thickness and continuity_zonal_convergence), with a data path in
// which every input crosses HBM once:
//   * one CTA per segment of 28 u faces of one row j and all layers; the first
//     face is the last face of the CTA to its left, recomputed, so that both
//     faces of every cell the CTA updates are its own;
//   * h of the cells I0-2 .. I0+31 and u of the faces (all layers) come into
//     shared memory with two TMA tile loads (a plain cooperative copy when the
//     field layout does not meet the TMA alignment rules);
//   * the PPM edge values and the curvature term (h_W + h_E) - 2 h of every
//     cell are formed in shared memory once: a warp takes a layer, a lane a
//     cell's slope, the neighbours' slopes come by shuffle (the 32 slopes of
//     cells I0-1 .. I0+30 give the edges of the CTA's 29 cells);
//   * each face is worked by 8 lanes of a warp, lane g taking the layers
//     g, g + 8, ...; a column sum is the lanes' partial sums combined by a
//     butterfly of shuffles, which leaves the same bits in all 8 lanes, so
//     the Newton scalars of a face are formed identically in its 8 lanes;
//   * a face's velocities stay in registers across its column passes, and
//     the transports, face thicknesses and new thicknesses leave in rows.
// Arithmetic differences from the exact form: column sums in another order,
// multiply-adds contracted (this file is built with FMA), the flux and the
// marginal thickness evaluated as base + CFL (...) in FMA form from the cell's
// edge values and curvature, and the CFL and BT_cont velocity bounds taken as
// minima / maxima over the column.  Every prognostic field stays within a
// relative L2 of 1e-12 of the exact form (tested after 10 steps).
#include <map>
#include <mutex>
#include <tuple>

#include "cont_impl.cuh"
#include "tma.cuh"

namespace mom6b {

constexpr int kCfFaces = 28;                    // faces per CTA, the first recomputed
constexpr int kCfG = 8;                         // lanes per face
constexpr int kCfWarps = kCfFaces * kCfG / 32;  // 7
constexpr int kCfThreads = kCfFaces * kCfG;     // 224
constexpr int kCfHW = 36;                       // h tile width (cells I0-2 .. I0+31 and more)
constexpr int kCfUW = 30;                       // u tile width (faces)
constexpr int kCfAB = 31;                       // (a, b) row stride in 16-byte units (odd)
constexpr int kCfC3 = 30;                       // curvature row stride in doubles (2 x odd)
constexpr int kCfOwned = kCfFaces - 1;          // cells (and faces) a CTA owns
constexpr unsigned kFull = 0xffffffffu;

// shared-memory regions in doubles, each starting on a 128-byte boundary
__host__ __device__ constexpr size_t cf_align(size_t n) { return (n + 15) & ~(size_t)15; }
__host__ __device__ constexpr size_t cf_off_u(int nk) { return cf_align((size_t)nk * kCfHW); }
__host__ __device__ constexpr size_t cf_off_ab(int nk)
{
    return cf_off_u(nk) + cf_align((size_t)nk * kCfUW);
}
__host__ __device__ constexpr size_t cf_off_c3(int nk)
{
    return cf_off_ab(nk) + cf_align((size_t)nk * kCfAB * 2);
}
__host__ __device__ constexpr size_t cf_off_m(int nk)
{
    return cf_off_c3(nk) + cf_align((size_t)nk * kCfC3);
}
__host__ __device__ constexpr size_t cf_off_bar(int nk) { return cf_off_m(nk) + cf_align(kCfHW); }
// + 16 doubles for the barrier, + 16 for aligning the base
__host__ __device__ constexpr size_t cf_smem_bytes(int nk)
{
    return (cf_off_bar(nk) + 32) * sizeof(double);
}

// Sum / min / max over the 8 lanes of a face (aligned groups of 8 lanes);
// a butterfly, so every lane of the group ends with the same value.
__device__ __forceinline__ double face_sum(double v)
{
    v += __shfl_xor_sync(kFull, v, 1);
    v += __shfl_xor_sync(kFull, v, 2);
    v += __shfl_xor_sync(kFull, v, 4);
    return v;
}
__device__ __forceinline__ double face_min(double v)
{
    v = fmin(v, __shfl_xor_sync(kFull, v, 1));
    v = fmin(v, __shfl_xor_sync(kFull, v, 2));
    return fmin(v, __shfl_xor_sync(kFull, v, 4));
}
__device__ __forceinline__ double face_max(double v)
{
    v = fmax(v, __shfl_xor_sync(kFull, v, 1));
    v = fmax(v, __shfl_xor_sync(kFull, v, 2));
    return fmax(v, __shfl_xor_sync(kFull, v, 4));
}

// One face's view of the cell data in shared memory.  A cell's PPM edges
// are kept as a = (h_W + h_E)/2 and b = (h_W - h_E)/2, so that the upwind
// cell's edge at the face is base = a - s b and the other minus it is 2 s b,
// with s = +1 for a flow out of cell i (u > 0) and -1 into it; c3 is the
// curvature (h_W + h_E) - 2 h.
struct CfFace {
    const double2* ab;      // (a, b) of cell i at layer 0 of this lane; cell i + 1 follows
    const double* c3;       // c3 of cell i at layer 0 of this lane
    double dy, dtIdx_i, dtIdx_p;
};

// zonal_flux_layer (:554-583) for the lane's t-th layer at velocity u1: the
// transport, and the marginal thickness in hm.  DIR: 0 selects the upwind
// cell by the sign of u1; +1 / -1 is a flow known to leave / enter cell i
// (u1 > 0 / u1 < 0).  ZERO (DIR 0): also the serial code's zero-velocity case
// (no transport, the mean of the two edges at the face); without it a zero
// u1 is evaluated as a flow into cell i and the caller repeats the pass with
// ZERO when any lane met a zero.
template <int DIR, bool ZERO>
__device__ __forceinline__ double cf_flux(const CfFace& F, int t, double u1, double& hm)
{
    const bool pos = DIR > 0 ? true : (DIR < 0 ? false : u1 > 0.0);
    const int c = pos ? 0 : 1;
    const double2 ab = F.ab[t * kCfG * kCfAB + c];
    const double c3 = F.c3[t * kCfG * kCfC3 + c];
    const double sb = pos ? ab.y : -ab.y;
    const double base = ab.x - sb;
    const double CFL = DIR > 0 ? u1 * F.dtIdx_i
                               : (DIR < 0 ? -u1 * F.dtIdx_p
                                          : fabs(u1) * (pos ? F.dtIdx_i : F.dtIdx_p));
    const double uh = (F.dy * u1) * fma(CFL, fma(c3, CFL - 1.5, sb), base);
    hm = fma(CFL, fma(3.0 * c3, CFL - 1.0, sb + sb), base);
    if constexpr (DIR == 0 && ZERO) {
        if (!(u1 > 0.0) && !(u1 < 0.0)) {
            const double2 abi = F.ab[t * kCfG * kCfAB], abp = F.ab[t * kCfG * kCfAB + 1];
            hm = 0.5 * ((abp.x + abp.y) + (abi.x - abi.y));    // (h_W(i+1) + h_E(i)) / 2
            return 0.0;
        }
    }
    return uh;
}

// Where a pass leaves the transports and face thicknesses of its layers
// (the face's last evaluated iterate is its uh, and its marginal thickness
// is the face thickness whenever u_cor is that iterate): uh into the lane's
// slots of the u tile (the velocities are in registers by then), the
// thickness into the global h_u of an owned face.
struct CfSink {
    double* uh;             // u-tile slot of layer 0 of this lane (stride kCfG * kCfUW)
    double* hu;             // h_u of layer 0 of this lane (stride kCfG * plane), or null
    size_t hu_stride;
};

// One pass over the lane's layers at velocities u + du: partial sums of the
// transports and of dy * the marginal thicknesses; with keep, the layers'
// transports and thicknesses also go to the sink.
template <int KPL>
__device__ __forceinline__ void cf_pass(const CfFace& F, const double (&ur)[KPL], int g, int nk,
                                        double du, double& su, double& sd, bool keep,
                                        const CfSink& S)
{
    su = 0.0;
    sd = 0.0;
    bool zero = false;
#pragma unroll
    for (int t = 0; t < KPL; ++t) {
        if (g + kCfG * t < nk) {
            const double u1 = ur[t] + du;
            zero |= u1 == 0.0;
            double hm;
            const double uh = cf_flux<0, false>(F, t, u1, hm);
            su += uh;
            sd = fma(F.dy, hm, sd);
            if (keep) {
                S.uh[t * kCfG * kCfUW] = uh;
                if (S.hu) __stcs(S.hu + (size_t)t * S.hu_stride, hm);
            }
        }
    }
    if (__any_sync(kFull, zero)) {
        su = 0.0;
        sd = 0.0;
#pragma unroll
        for (int t = 0; t < KPL; ++t) {
            if (g + kCfG * t < nk) {
                double hm;
                const double uh = cf_flux<0, true>(F, t, ur[t] + du, hm);
                su += uh;
                sd = fma(F.dy, hm, sd);
                if (keep) {
                    S.uh[t * kCfG * kCfUW] = uh;
                    if (S.hu) __stcs(S.hu + (size_t)t * S.hu_stride, hm);
                }
            }
        }
    }
}

// KPL: layers per lane (nk <= 8 KPL).  TMA: tiles by tensor maps, else by a
// cooperative copy.
template <int KPL, bool TMA>
__global__ void __launch_bounds__(kCfThreads, 2)
k_cont_fast(Dims D, Metrics M, const __grid_constant__ CUtensorMap map_u,
            const __grid_constant__ CUtensorMap map_h, const double* __restrict__ u,
            const double* __restrict__ hin, const double* __restrict__ uhbt2d, ContOut O,
            double dt, double h_min, int* status)
{
    extern __shared__ __align__(16) double smem_raw[];
    // the regions start on 128-byte boundaries of the shared window
    const int pad = (int)(((128u - ((uint32_t)__cvta_generic_to_shared(smem_raw) & 127u)) & 127u) >> 3);
    double* sm = smem_raw + pad;
    const int nk = D.nk;
    const int tid = (int)threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int j = D.js + (int)blockIdx.y;
    const int I0 = D.is - 1 + (int)blockIdx.x * kCfOwned;
    const int x0h = (I0 - 3) & ~1;      // 0-based i of h-tile column 0 (even)
    const int x0u = (I0 - 1) & ~1;      // 0-based i of u-tile column 0 (even)
    const size_t row = (size_t)(j - 1) * D.n1;
    double* sh_h = sm;                                   // [nk][kCfHW]
    double* sh_u = sm + cf_off_u(nk);                    // [nk][kCfUW]
    double2* sh_ab = (double2*)(sm + cf_off_ab(nk));     // [nk][kCfAB] (a, b)
    double* sh_c3 = sm + cf_off_c3(nk);                  // [nk][kCfC3] slope, then curvature
    double* sh_m = sm + cf_off_m(nk);                    // [kCfHW] mask2dT of the h tile
    uint64_t* bar = (uint64_t*)(sm + cf_off_bar(nk));

    // ---- the tiles --------------------------------------------------------
    if constexpr (TMA) {
        if (tid == 0) {
            tma_prefetch_map(&map_h);
            tma_prefetch_map(&map_u);
            tma_bar_init(bar, 1);
        }
        __syncthreads();
        if (tid == 0) {
            tma_bar_expect(bar, (uint32_t)((size_t)nk * (kCfHW + kCfUW) * sizeof(double)));
            tma_load_3d(sh_h, &map_h, x0h, j - 1, 0, bar);
            tma_load_3d(sh_u, &map_u, x0u, j - 1, 0, bar);
        }
    } else {
        for (int k = warp; k < nk; k += kCfWarps) {
            const size_t o = (size_t)k * D.plane + row;
            for (int c = lane; c < kCfHW; c += 32) {
                const int x = x0h + c;
                sh_h[k * kCfHW + c] = x < D.n1 ? hin[o + x] : 0.0;
            }
            for (int c = lane; c < kCfUW; c += 32) {
                const int x = x0u + c;
                sh_u[k * kCfUW + c] = x < D.n1 ? u[o + x] : 0.0;
            }
        }
    }
    for (int c = tid; c < kCfHW; c += kCfThreads) {
        const int x = x0h + c;
        sh_m[c] = x < D.n1 ? M.mask2dT[row + x] : 0.0;
    }

    // per-face quantities while the tiles land
    const int f = tid >> 3, g = tid & 7;
    const int I = I0 + f;
    const bool face_ok = I <= D.ie;
    const bool owner = face_ok && (f >= 1 || blockIdx.x == 0);
    const int Ic = face_ok ? I : D.ie;
    const int ucol = I - 1 - x0u;
    CfFace F;
    F.dy = MOM6B_A2(M.dy_Cu, Ic, j, D);
    F.dtIdx_i = dt * MOM6B_A2(M.IdxT, Ic, j, D);
    F.dtIdx_p = dt * MOM6B_A2(M.IdxT, Ic + 1, j, D);
    F.ab = sh_ab + g * kCfAB + (f + 1);
    F.c3 = sh_c3 + g * kCfC3 + (f + 1);
    const double CFL_dt = 0.5 / dt;
    const double dx_W = MOM6B_A2(M.dxT, Ic, j, D), dx_E = MOM6B_A2(M.dxT, Ic + 1, j, D);
    const double mCu = MOM6B_A2(M.mask2dCu, Ic, j, D);
    const double fac = dt * fmin(MOM6B_A2(M.IareaT, Ic, j, D), MOM6B_A2(M.IareaT, Ic + 1, j, D));
    const double uhbt = MOM6B_A2(uhbt2d, Ic, j, D);
    const double du_CFL = (F32(1e-6) * (1.0 / dt)) * MOM6B_A2(M.dxCu, Ic, j, D);

    int timed_out = 0;
    if constexpr (TMA) timed_out = !tma_bar_wait(bar, 0, kBtDefaultWait);
    if (__syncthreads_or(timed_out)) {
        if (tid == 0) atomicExch(status, kDevTimeout);
        return;
    }

    // ---- PPM edges: warp w takes layers w, w + 7, ..., four at a time; in a
    // layer lane l forms the slope of cell I0 - 1 + l, takes its neighbours'
    // slopes by shuffle, and lanes 1 .. 29 form the edges and the curvature
    // of cells I0 .. I0 + 28 (local index lc = l).
    {
        const int hb = I0 - 2 - x0h;        // h-tile column of cell I0 - 1
        const double* hr0 = sh_h + hb + lane;
        const double ml = sh_m[hb + lane - 1], mc = sh_m[hb + lane], mr = sh_m[hb + lane + 1];
        const bool slope_ok = (ml * mc * mr) != 0.0;
        const double oml = 1.0 - ml, omr = 1.0 - mr;
        const bool write = lane >= 1 && lane <= kCfFaces + 1;
        auto edges = [&](int k) {
            const double* hr = hr0 + k * kCfHW;
            const double hm = hr[-1], hc = hr[0], hp = hr[1];
            const double slc = ppm_slope3(hm, hc, hp, slope_ok);
            const double slm = __shfl_up_sync(kFull, slc, 1);
            const double slp = __shfl_down_sync(kFull, slc, 1);
            double hL, hR;
            ppm_edges_limited<true>(hm, hc, hp, ml, oml, mr, omr, slm, slc, slp, h_min, hL,
                                    hR);
            if (write) {
                sh_ab[k * kCfAB + lane] = make_double2(0.5 * (hL + hR), 0.5 * (hL - hR));
                sh_c3[k * kCfC3 + lane] = (hL + hR) - 2.0 * hc;
            }
        };
        int k = warp;
        for (; k + 3 * kCfWarps < nk; k += 4 * kCfWarps) {
            edges(k);
            edges(k + kCfWarps);
            edges(k + 2 * kCfWarps);
            edges(k + 3 * kCfWarps);
        }
        for (; k < nk; k += kCfWarps) edges(k);
    }
    __syncthreads();

    // ---- the faces ----------------------------------------------------------
    double ur[KPL];
#pragma unroll
    for (int t = 0; t < KPL; ++t) {
        const int k = g + kCfG * t;
        ur[t] = k < nk ? sh_u[k * kCfUW + ucol] : 0.0;
    }
    // the CFL limits (:335-433): minima / maxima over the column where the
    // face mask is 1; elsewhere the serial test u*mask in layer order
    double dmx = 2.0 * (CFL_dt * dx_W), dmn = -(2.0 * (CFL_dt * dx_E));
    if (mCu != 1.0) {
        for (int k = 0; k < nk; ++k) {
            const double uk = sh_u[k * kCfUW + ucol];
            if (dmx > dx_W * CFL_dt - uk * mCu) dmx = dx_W * CFL_dt - uk;
            if (dmn < -(dx_E * CFL_dt) - uk * mCu) dmn = -(dx_E * CFL_dt + uk);
        }
    } else {
#pragma unroll
        for (int t = 0; t < KPL; ++t) {
            if (g + kCfG * t < nk) {
                dmx = fmin(dmx, dx_W * CFL_dt - ur[t]);
                dmn = fmax(dmn, -(dx_E * CFL_dt + ur[t]));
            }
        }
    }
    dmx = face_min(dmx);
    dmn = face_max(dmn);
    const double du_max_CFL = fmax(dmx, 0.0), du_min_CFL = fmin(dmn, 0.0);
    __syncwarp();   // every lane of the warp has read its u from the tile

    CfSink S;
    S.uh = sh_u + g * kCfUW + ucol;
    S.hu = owner ? O.h_u + (size_t)g * D.plane + row + (size_t)(I - 1) : nullptr;
    S.hu_stride = (size_t)kCfG * D.plane;

    // initial fluxes and their column sums (:305-355)
    double s_uh, s_da;
    cf_pass<KPL>(F, ur, g, nk, 0.0, s_uh, s_da, face_ok, S);
    const double uh_tot_0 = face_sum(s_uh), duhdu_tot_0 = face_sum(s_da);

    // zonal_flux_adjust toward uhbt (:813-903); the transports of the last
    // evaluated iterate are the face's uh, its thicknesses kept beside them
    constexpr int max_itts = 20;
    Newton A = newton_start(uh_tot_0 - uhbt, duhdu_tot_0, du_max_CFL, du_min_CFL, face_ok);
    double du_eval = 0.0, sd_eval = duhdu_tot_0;
    for (int itt = 1; itt <= max_itts; ++itt) {
        if (A.live) A.live = newton_iter<true>(A, itt, fac);
        const bool pa = A.live;
        if (!__any_sync(kFull, pa)) break;
        double su = 0.0, sd = 0.0;
        cf_pass<KPL>(F, ur, g, nk, A.du, su, sd, pa, S);
        su = face_sum(su);
        sd = face_sum(sd);
        if (pa) {
            du_eval = A.du;
            sd_eval = sd;
            if (itt < max_itts) {
                A.uh_err = su - uhbt;
                A.duhdu_tot = sd;
                A.uh_err_best = fmin(A.uh_err_best, fabs(A.uh_err));
            }
        }
    }
    const double du = A.du;
    // set_zonal_BT_cont's zero-transport solve (:991-1002), needed only where
    // uhbt /= 0 (with uhbt = 0 it repeats the solve above exactly)
    double du0 = du;
    const bool solve0 = owner && uhbt != 0.0;
    if (__any_sync(kFull, solve0)) {
        Newton B = newton_start(uh_tot_0, duhdu_tot_0, du_max_CFL, du_min_CFL, solve0);
        for (int itt = 1; itt <= max_itts; ++itt) {
            if (B.live) B.live = newton_iter<true>(B, itt, fac);
            const bool pb = B.live && itt < max_itts;
            if (!__any_sync(kFull, pb)) break;
            double su = 0.0, sd = 0.0;
            cf_pass<KPL>(F, ur, g, nk, B.du, su, sd, false, S);
            su = face_sum(su);
            sd = face_sum(sd);
            if (pb) {
                B.uh_err = su;
                B.duhdu_tot = sd;
                B.uh_err_best = fmin(B.uh_err_best, fabs(B.uh_err));
            }
        }
        if (solve0) du0 = B.du;
    }

    // set_zonal_BT_cont (:991-1121): the bounding velocities, then the face
    // areas at du0, duL, duR and the transports at duL, duR.  Where du0 and
    // u_cor's du are the last evaluated iterate (the rule: uhbt = 0) its sums
    // and thicknesses are reused, and the flows at duL / duR are of known
    // sign (u + duL >= du_CFL > 0, u + duR <= -du_CFL < 0).
    double duR = fmin(0.0, du0 - du_CFL), duL = fmax(0.0, du0 + du_CFL);
#pragma unroll
    for (int t = 0; t < KPL; ++t) {
        if (g + kCfG * t < nk) {
            duR = fmin(duR, -(ur[t] + du_CFL));
            duL = fmax(duL, -(ur[t] - du_CFL));
        }
    }
    duR = face_min(duR);
    duL = face_max(duL);
    double F0, FL = 0.0, FR = 0.0, UL = 0.0, UR = 0.0;
    const bool reuse = __all_sync(kFull, (du0 == du_eval && du == du_eval && du_CFL > 0.0) ||
                                             !face_ok);
    if (reuse) {
        F0 = sd_eval;
#pragma unroll
        for (int t = 0; t < KPL; ++t) {
            if (g + kCfG * t < nk) {
                double hmL, hmR;
                UL += cf_flux<1, false>(F, t, ur[t] + duL, hmL);
                UR += cf_flux<-1, false>(F, t, ur[t] + duR, hmR);
                FL = fma(F.dy, hmL, FL);
                FR = fma(F.dy, hmR, FR);
            }
        }
    } else {
        // the general pass: every evaluation with the zero-velocity case
        F0 = 0.0;
#pragma unroll
        for (int t = 0; t < KPL; ++t) {
            if (g + kCfG * t < nk) {
                double hm0, hmL, hmR, hmc, tmp;
                cf_flux<0, true>(F, t, ur[t] + du0, hm0);
                UL += cf_flux<0, true>(F, t, ur[t] + duL, hmL);
                UR += cf_flux<0, true>(F, t, ur[t] + duR, hmR);
                cf_flux<0, true>(F, t, ur[t] + du, hmc);
                const double uhf = cf_flux<0, true>(F, t, ur[t] + du_eval, tmp);
                F0 = fma(F.dy, hm0, F0);
                FL = fma(F.dy, hmL, FL);
                FR = fma(F.dy, hmR, FR);
                if (face_ok) {
                    S.uh[t * kCfG * kCfUW] = uhf;
                    if (S.hu) __stcs(S.hu + (size_t)t * S.hu_stride, hmc);
                }
            }
        }
        F0 = face_sum(F0);
    }
    FL = face_sum(FL);
    FR = face_sum(FR);
    UL = face_sum(UL);
    UR = face_sum(UR);
    if (owner) {
        const size_t f0 = row + (size_t)(I - 1);
        // the west (lane 0) and east (lane 1) sides of the face in parallel
        if (g < 2) {
            const bool west = g == 0;
            const double dub = west ? duL : duR, FAmt = west ? FL : FR;
            const double uhtot = west ? UL : UR;
            double FA_0 = F0, FA_avg = F0;
            if ((dub - du0) != 0.0) FA_avg = uhtot / (dub - du0);
            if (FA_avg > fmax(FA_0, FAmt)) FA_avg = fmax(FA_0, FAmt);
            else if (FA_avg < fmin(FA_0, FAmt)) FA_0 = FA_avg;
            const double uBT = (fabs(FAmt - FA_0) <= F32(1e-12) * FA_0)
                                   ? 0.0
                                   : (1.5 * (dub - du0)) * ((FAmt - FA_avg) / (FAmt - FA_0));
            (west ? O.FA_u_W0 : O.FA_u_E0)[f0] = FA_0;
            (west ? O.FA_u_WW : O.FA_u_EE)[f0] = FAmt;
            (west ? O.uBT_WW : O.uBT_EE)[f0] = uBT;
        } else if (g == 2) {
            O.du_cor[f0] = du;
        }
    }
    __syncthreads();

    // ---- transports of the owned faces, and continuity_zonal_convergence
    // (:148-176) of the cells I0+1 .. I0+27: warp w takes layers w, w + 7, ...,
    // lane l face I0 + l and cell I0 + l
    {
        const int Iw = I0 + lane;
        const bool out_uh = lane < kCfFaces && Iw <= D.ie && (lane >= 1 || blockIdx.x == 0);
        const int c = Iw;
        const bool out_h = lane >= 1 && lane < kCfFaces && c >= D.is && c <= D.ie;
        const double fc = out_h ? dt * MOM6B_A2(M.IareaT, c, j, D) : 0.0;
        for (int k = warp; k < nk; k += kCfWarps) {
            const double* ue = sh_u + k * kCfUW + (Iw - 1 - x0u);
            const size_t o = (size_t)k * D.plane + row + (size_t)(Iw - 1);
            if (out_uh) __stcs(O.uh + o, ue[0]);
            if (out_h) {
                const double hn = fmax(sh_h[k * kCfHW + (c - 1 - x0h)] - fc * (ue[0] - ue[-1]), 0.0);
                __stcs(O.h + o, hn);
            }
        }
    }
}

// ---- host ----------------------------------------------------------------

typedef CUresult (*CfEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                               const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                               const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                               CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

cudaError_t tma_map_box3d(CUtensorMap* map, const double* base, int n1, int n2, int nk,
                          int box_w, int box_h, int box_d)
{
    static CfEncodeFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return cudaErrorNotSupported;
        fn = (CfEncodeFn)p;
    }
    if (((uintptr_t)base & 15u) || (n1 & 1) || (box_w & 1) || box_w > 256 || box_h > 256 ||
        box_d > 256 || box_w < 2 || box_h < 1 || box_d < 1 || nk < 1)
        return cudaErrorNotSupported;
    cuuint64_t gdim[3] = {(cuuint64_t)n1, (cuuint64_t)n2, (cuuint64_t)nk};
    cuuint64_t gstride[2] = {(cuuint64_t)n1 * 8, (cuuint64_t)n1 * (cuuint64_t)n2 * 8};
    cuuint32_t box[3] = {(cuuint32_t)box_w, (cuuint32_t)box_h, (cuuint32_t)box_d};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), gdim,
                    gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorNotSupported;
}

cudaError_t tma_map_field3d(CUtensorMap* map, const double* base, int n1, int n2, int nk,
                            int box_w)
{
    return tma_map_box3d(map, base, n1, n2, nk, box_w, 1, nk);
}

// Tensor maps are encoded once per (field address, shape, box) and kept.
bool tma_map_cached(const double* base, int n1, int n2, int nk, int box_w, int box_h,
                    int box_d, CUtensorMap* out)
{
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, int, int, int, int>, CUtensorMap> maps;
    const auto key = std::make_tuple((const void*)base, n1, n2, nk, box_w, box_h, box_d);
    std::lock_guard<std::mutex> lock(mu);
    auto it = maps.find(key);
    if (it == maps.end()) {
        CUtensorMap m;
        if (tma_map_box3d(&m, base, n1, n2, nk, box_w, box_h, box_d) != cudaSuccess)
            return false;
        it = maps.emplace(key, m).first;
    }
    *out = it->second;
    return true;
}

static bool cf_map(const double* base, const Dims& D, int box_w, CUtensorMap* out)
{
    return tma_map_cached(base, D.n1, D.n2, D.nk, box_w, 1, D.nk, out);
}

bool continuity_fast_fits(const Dims& D) { return D.nk >= 1 && D.nk <= 128; }

template <int KPL>
static cudaError_t launch_cf(const Dims& D, const Metrics& M, const double* u, const double* hin,
                             const double* uhbt, const ContOut& O, double dt, double h_min,
                             int* status, cudaStream_t s)
{
    const int nfaces = D.ie - (D.is - 1) + 1;
    dim3 grid((nfaces - 1 + kCfOwned - 1) / kCfOwned, D.je - D.js + 1, 1);
    const size_t smem = cf_smem_bytes(D.nk);
    CUtensorMap mu{}, mh{};
    const bool tma = cf_map(u, D, kCfUW, &mu) && cf_map(hin, D, kCfHW, &mh);
    auto kern = tma ? k_cont_fast<KPL, true> : k_cont_fast<KPL, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kCfThreads, smem, s>>>(D, M, mu, mh, u, hin, uhbt, O, dt, h_min, status);
    return cudaGetLastError();
}

cudaError_t launch_continuity_fast(const Dims& D, const Metrics& M, const double* u,
                                   const double* hin, const double* uhbt, const ContOut& O,
                                   double dt, double h_min, int* status, cudaStream_t s)
{
    if (!continuity_fast_fits(D)) return cudaErrorInvalidValue;
    if (D.nk <= 8 * 10) return launch_cf<10>(D, M, u, hin, uhbt, O, dt, h_min, status, s);
    return launch_cf<16>(D, M, u, hin, uhbt, O, dt, h_min, status, s);
}

} // namespace mom6b
