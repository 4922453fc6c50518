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

// PPM_reconstruction_x + PPM_limit_pos for cell i of one row (hrow/mrow point
// at element i = 1 of the row).
__device__ __forceinline__ void ppm_cell(const double* __restrict__ hrow,
                                         const double* __restrict__ mrow, int i,
                                         double h_min, double& hL, double& hR)
{
    const double oneSixth = 1.0 / 6.0;
    double slm = ppm_slope(hrow, mrow, i - 1);
    double slc = ppm_slope(hrow, mrow, i);
    double slp = ppm_slope(hrow, mrow, i + 1);
    double hc = hrow[i - 1];
    double h_im1 = mrow[i - 2] * hrow[i - 2] + (1.0 - mrow[i - 2]) * hc;
    double h_ip1 = mrow[i] * hrow[i] + (1.0 - mrow[i]) * hc;
    hL = 0.5 * (h_im1 + hc) + oneSixth * (slm - slc);
    hR = 0.5 * (h_ip1 + hc) + oneSixth * (slc - slp);
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
}

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
                    float scale = (float)(lhs / (double)den);
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

__global__ void __launch_bounds__(128)
k_ppm_edges(Dims D, Metrics M, const double* __restrict__ hin,
            double* __restrict__ hW, double* __restrict__ hE, double h_min)
{
    const int i = D.is - 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = D.js + (int)blockIdx.y;
    const int k = 1 + (int)blockIdx.z;
    if (i > D.ie + 1) return;
    const size_t rowoff = (size_t)(k - 1) * D.plane + (size_t)(j - 1) * D.n1;
    double hL, hR;
    ppm_cell(hin + rowoff, M.mask2dT + (size_t)(j - 1) * D.n1, i, h_min, hL, hR);
    hW[rowoff + (i - 1)] = hL;
    hE[rowoff + (i - 1)] = hR;
}

// The same edges with each cell's slope formed once: lane l of a warp takes
// cell c = is - 2 + 30 w + l (w = the warp's index along the row), forms the
// slope of c, takes the slopes of c - 1 and c + 1 from lanes l - 1 and l + 1,
// and lanes 1..30 write the edges of their cells.  The masks are read once
// and each thread walks kEdgeLayers layers.
constexpr int kEdgeCellsPerWarp = 30;
constexpr int kEdgeLayers = 5;

__global__ void __launch_bounds__(128)
k_ppm_edges_warp(Dims D, Metrics M, const double* __restrict__ hin,
                 double* __restrict__ hW, double* __restrict__ hE, double h_min)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = (int)threadIdx.x & 31;
    const int wrow = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int c = D.is - 2 + kEdgeCellsPerWarp * wrow + lane;
    const int j = D.js + (int)blockIdx.y;
    const int k0 = 1 + (int)blockIdx.z * kEdgeLayers;
    const bool load_ok = c <= D.ie + 2;
    const bool write_ok = lane >= 1 && lane <= kEdgeCellsPerWarp && c <= D.ie + 1;
    const size_t r = (size_t)(j - 1) * D.n1 + (size_t)(c - 1);
    const double* mrow = M.mask2dT + r;
    const double m0 = load_ok ? mrow[-1] : 0.0;
    const double m1 = load_ok ? mrow[0] : 0.0;
    const double m2 = load_ok ? mrow[1] : 0.0;
    const bool slope_ok = (m0 * m1 * m2) != 0.0;
    const double om0 = 1.0 - m0, om2 = 1.0 - m2;
    const int kn = min(kEdgeLayers, D.nk - k0 + 1);   // uniform over the CTA
    const double* hp0 = hin + (size_t)(k0 - 1) * D.plane + r;
    double hm[kEdgeLayers], hc[kEdgeLayers], hp[kEdgeLayers];
#pragma unroll
    for (int q = 0; q < kEdgeLayers; ++q) {
        const double* p = hp0 + (size_t)q * D.plane;
        const bool ok = load_ok && q < kn;
        hm[q] = ok ? p[-1] : 0.0;
        hc[q] = ok ? p[0] : 0.0;
        hp[q] = ok ? p[1] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < kEdgeLayers; ++q) {
        if (q < kn) {
            const double slc = ppm_slope3(hm[q], hc[q], hp[q], slope_ok);
            const double slm = __shfl_up_sync(FULL, slc, 1);
            const double slp = __shfl_down_sync(FULL, slc, 1);
            double hL, hR;
            ppm_edges_limited(hm[q], hc[q], hp[q], m0, om0, m2, om2, slm, slc, slp, h_min, hL, hR);
            if (write_ok) {
                const size_t o = (size_t)(k0 - 1 + q) * D.plane + r;
                hW[o] = hL;
                hE[o] = hR;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// face column work
// ---------------------------------------------------------------------------
// EI is the index type of the edge arrays: size_t for the global scratch
// pair, int for the shared-memory copies (shared memory is always indexed
// with 32-bit offsets here).
template <typename EI>
struct FaceCol {
    const double* u;     // u(I, j, 1), layer stride = plane
    const double* hc;    // h(I, j, 1)   (cell i = I)
    const double* hWc;   // h_W of cell I at layer 1, layer stride = estride
    const double* hEc;   // h_E of cell I at layer 1
    size_t plane;
    EI estride;          // layer stride of hWc/hEc (plane, or the smem row length)
    double dy;           // dy_Cu(I, j) (times por_face_areaU = 1)
    double IdxT_i, IdxT_ip1;
    // meridional faces (Y): offsets of the next cell (J + 1) in the h and
    // edge arrays; zonal faces use the next element
    size_t nbh = 1;
    EI nbe = 1;
    // the vertical-viscosity remnant of the face column (VREM), stride plane
    const double* vr = nullptr;
    // AS: this thread's staging slots in shared memory, slot (b, c, f) at
    // st[((b * CH + c) * 7 + f) * sts]
    double* st = nullptr;
    int sts = 0;
};

// The inputs of one layer of one face: u(I) and the cell values of the two
// cells either side (h_W, h_E, h of i = I and of i + 1).
struct LayerVals {
    double u, hWi, hEi, hi, hWp, hEp, hp;
    double vr;   // visc_rem of the layer (the remnant form only)
};

// Layers whose inputs one prefetch brings into registers (CH).  Each pass
// over a face column is a chain of dependent sums, so the loads of CH layers
// are issued together and their latency is paid once per chunk.
constexpr int kContChunk = 4;
// Cache hints in the face kernel: evict-first loads in the last column pass,
// streaming stores of h_u and h.
#ifndef MOM6B_CONT_HINTS
#define MOM6B_CONT_HINTS 1
#endif
constexpr bool kContHints = MOM6B_CONT_HINTS != 0;

// LAST: the face's last pass over its column; u and the global edge arrays
// are then read with the evict-first hint (nothing reads them again), which
// leaves L2 to the columns whose Newton passes are still to come.
// Y: a meridional face (i, J) whose cells are (i, J) and (i, J + 1); the
// "W"/"E" edges are then the south/north edges.
template <bool LAST = false, bool Y = false, bool VREM = false, typename EI>
__device__ __forceinline__ LayerVals load_layer(const FaceCol<EI>& F, int k)
{
    const size_t o = (size_t)(k - 1) * F.plane;
    const EI oe = (EI)(k - 1) * F.estride;
    const size_t nh = Y ? F.nbh : (size_t)1;
    const EI ne = Y ? F.nbe : (EI)1;
    LayerVals L;
    if constexpr (LAST && sizeof(EI) == sizeof(size_t)) {
        L.u = __ldcs(F.u + o);
        L.hWi = __ldcs(F.hWc + oe); L.hEi = __ldcs(F.hEc + oe);
        L.hWp = __ldcs(F.hWc + oe + ne); L.hEp = __ldcs(F.hEc + oe + ne);
    } else {
        L.u = F.u[o];
        L.hWi = F.hWc[oe]; L.hEi = F.hEc[oe];
        L.hWp = F.hWc[oe + ne]; L.hEp = F.hEc[oe + ne];
    }
    L.hi = F.hc[o]; L.hp = F.hc[o + nh];
    if constexpr (VREM) L.vr = LAST ? __ldcs(F.vr + o) : F.vr[o];
    return L;
}

// VREM: the velocity a face evaluates at is u + du visc_rem, and its
// marginal areas (duhdu) carry the factor visc_rem (zonal_flux_layer :581,
// zonal_flux_adjust :880); without it visc_rem = 1 and both factors are
// exact, so they are omitted.
template <bool VREM>
__device__ __forceinline__ double u_at(const LayerVals& L, double du)
{
    if constexpr (VREM) return L.u + du * L.vr;
    else return L.u + du;
}
template <bool VREM, typename EI>
__device__ __forceinline__ double darea(const FaceCol<EI>& F, const LayerVals& L, double hm)
{
    if constexpr (VREM) return (F.dy * hm) * L.vr;
    else return F.dy * hm;
}

// Visit layers 1..nz in order, fn(k, LayerVals).
// AS: the next chunk's seven values per layer are copied into shared memory
// with cp.async while the current chunk is evaluated (zonal, without the
// remnant); otherwise each chunk is loaded into registers before it is
// evaluated.
template <int CH, bool LAST = false, bool Y = false, bool VREM = false, bool AS = false,
          typename EI, typename Fn>
__device__ __forceinline__ void for_layers(const FaceCol<EI>& F, int nz, Fn&& fn)
{
    if constexpr (AS && !Y && !VREM) {
        auto slot = [&](int b, int c, int f) -> double& {
            return F.st[(size_t)((b * CH + c) * 7 + f) * F.sts];
        };
        auto stage = [&](int kt, int b) {
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const int k = kt + c;
                const bool ok = k <= nz;
                const size_t o = ok ? (size_t)(k - 1) * F.plane : 0;
                const EI oe = ok ? (EI)(k - 1) * F.estride : (EI)0;
                cp_async_elem(&slot(b, c, 0), F.u + o, ok);
                cp_async_elem(&slot(b, c, 1), F.hWc + oe, ok);
                cp_async_elem(&slot(b, c, 2), F.hEc + oe, ok);
                cp_async_elem(&slot(b, c, 3), F.hc + o, ok);
                cp_async_elem(&slot(b, c, 4), F.hWc + oe + 1, ok);
                cp_async_elem(&slot(b, c, 5), F.hEc + oe + 1, ok);
                cp_async_elem(&slot(b, c, 6), F.hc + o + 1, ok);
            }
            cp_async_commit();
        };
        stage(1, 0);
        for (int kt = 1, it = 0; kt <= nz; kt += CH, ++it) {
            const int b = it & 1;
            if (kt + CH <= nz) {
                stage(kt + CH, b ^ 1);
                cp_async_wait_prior();
            } else {
                cp_async_wait_all();
            }
            LayerVals L[CH];
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                L[c].u = slot(b, c, 0);
                L[c].hWi = slot(b, c, 1); L[c].hEi = slot(b, c, 2); L[c].hi = slot(b, c, 3);
                L[c].hWp = slot(b, c, 4); L[c].hEp = slot(b, c, 5); L[c].hp = slot(b, c, 6);
            }
#pragma unroll
            for (int c = 0; c < CH; ++c)
                if (kt + c <= nz) fn(kt + c, L[c]);
        }
    } else {
    for (int kt = 1; kt <= nz; kt += CH) {
        LayerVals L[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c)
            if (kt + c <= nz) L[c] = load_layer<LAST, Y, VREM>(F, kt + c);
#pragma unroll
        for (int c = 0; c < CH; ++c)
            if (kt + c <= nz) fn(kt + c, L[c]);
    }
    }
}

// Visit u(I, k) for k = 1..nz in order, fn(k, u).
template <int CH, typename EI, typename Fn>
__device__ __forceinline__ void for_u(const FaceCol<EI>& F, int nz, Fn&& fn)
{
    constexpr int CU = 2 * CH;
    for (int kt = 1; kt <= nz; kt += CU) {
        double uk[CU];
#pragma unroll
        for (int c = 0; c < CU; ++c)
            if (kt + c <= nz) uk[c] = F.u[(size_t)(kt + c - 1) * F.plane];
#pragma unroll
        for (int c = 0; c < CU; ++c)
            if (kt + c <= nz) fn(kt + c, uk[c]);
    }
}

// zonal_flux_layer (:554-583) for one layer; returns uh and sets h_marg.
// The two upwind cases are one operation sequence on (base, other, h) =
// (h_E(i), h_W(i), h(i)) for u > 0 or (h_W(i+1), h_E(i+1), h(i+1)) for u < 0,
// and CFL = (|u| dt) Idx equals the reference's -(u dt Idx) for u < 0 exactly,
// so the evaluation is written without a divergent branch.
template <typename EI>
__device__ __forceinline__ double flux_eval(const FaceCol<EI>& F, const LayerVals& L,
                                            double uI, double dt, double& h_marg)
{
    const bool pos = uI > 0.0;
    const double base = pos ? L.hEi : L.hWp;
    const double oth = pos ? L.hWi : L.hEp;
    const double hc = pos ? L.hi : L.hp;
    const double Idx = pos ? F.IdxT_i : F.IdxT_ip1;
    const double CFL = fabs(uI) * dt * Idx;
    const double curv_3 = (oth + base) - 2.0 * hc;
    const double uh = F.dy * uI * (base + CFL * (0.5 * (oth - base) + curv_3 * (CFL - 1.5)));
    const double hm = base + CFL * ((oth - base) + 3.0 * curv_3 * (CFL - 1.0));
    const bool zero = !(uI > 0.0) && !(uI < 0.0);
    h_marg = zero ? 0.5 * (L.hWp + L.hEi) : hm;
    return zero ? 0.0 : uh;
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
// the root, takes the Newton (or bisection) step; returns do_I.
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
            double ddu = -(S.uh_err / S.duhdu_tot);
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

// The two zonal_flux_adjust solves of one face run in lockstep: A drives the
// face transport toward uhbt and stores the transports of every evaluated
// iteration in uh (the present(uh_3d) call, :307); B is set_zonal_BT_cont's
// zero-transport solve (:1002), live only when it is needed.  The two are
// independent iterations, each with its own operation sequence; sharing the
// column passes only halves how often the column is read.
template <int CH, typename EI, bool Y = false, bool VREM = false, bool AS = false>
__device__ void flux_adjust_pair(const FaceCol<EI>& F, int nz, double dt, double uhbt,
                                 double tol_eta_dt_fac, Newton& A, Newton& B,
                                 double* uh_out, size_t uh_stride)
{
    const int max_itts = 20;
    for (int itt = 1; itt <= max_itts; ++itt) {
        if (A.live) A.live = newton_iter(A, itt, tol_eta_dt_fac);
        if (B.live) B.live = newton_iter(B, itt, tol_eta_dt_fac);
        const bool update = itt < max_itts;
        const bool pa = A.live;            // A always stores, so it evaluates
        const bool pb = B.live && update;  // B evaluates only to update
        if (!pa && !pb) break;
        const double duA = A.du, duB = B.du;
        double eA = -uhbt, sA = 0.0, eB = -0.0, sB = 0.0;
        for_layers<CH, false, Y, VREM, AS>(F, nz, [&](int k, const LayerVals& L) {
            if (pa) {
                double hm;
                double uhk = flux_eval(F, L, u_at<VREM>(L, duA), dt, hm);
                uh_out[(size_t)(k - 1) * uh_stride] = uhk;
                eA = eA + uhk;
                sA = sA + darea<VREM>(F, L, hm);
            }
            if (pb) {
                double hm;
                double uhk = flux_eval(F, L, u_at<VREM>(L, duB), dt, hm);
                eB = eB + uhk;
                sB = sB + darea<VREM>(F, L, hm);
            }
        });
        if (pa && update) {
            A.uh_err = eA;
            A.duhdu_tot = sA;
            A.uh_err_best = dmin(A.uh_err_best, fabs(A.uh_err));
        }
        if (pb) {
            B.uh_err = eB;
            B.duhdu_tot = sB;
            B.uh_err_best = dmin(B.uh_err_best, fabs(B.uh_err));
        }
    }
}

// One zonal_flux_adjust solve on its own (:813-903): the transports of every
// evaluated iterate go to uh_out when it is given (then the last iterate is
// evaluated even at max_itts), otherwise passes run only to update.
template <int CH, typename EI, bool Y = false, bool VREM = false, bool AS = false>
__device__ void flux_adjust_one(const FaceCol<EI>& F, int nz, double dt, double target,
                                double tol_eta_dt_fac, Newton& S, double* uh_out,
                                size_t uh_stride)
{
    const int max_itts = 20;
    for (int itt = 1; itt <= max_itts; ++itt) {
        if (!newton_iter(S, itt, tol_eta_dt_fac)) break;
        const bool update = itt < max_itts;
        if (!update && !uh_out) break;
        const double du = S.du;
        double e = -target, sm = 0.0;
        for_layers<CH, false, Y, VREM, AS>(F, nz, [&](int k, const LayerVals& L) {
            double hm;
            double uhk = flux_eval(F, L, u_at<VREM>(L, du), dt, hm);
            if (uh_out) uh_out[(size_t)(k - 1) * uh_stride] = uhk;
            e = e + uhk;
            sm = sm + darea<VREM>(F, L, hm);
        });
        if (update) {
            S.uh_err = e;
            S.duhdu_tot = sm;
            S.uh_err_best = dmin(S.uh_err_best, fabs(S.uh_err));
        }
    }
}

// The work of one face (I, j) after its column views are set up: initial
// fluxes, CFL limits, zonal_flux_adjust, du_cor and, for the owner,
// set_zonal_BT_cont and zonal_flux_thickness.  uh/ust receive the face's
// transports (the output array, or the CTA's overlap column).
// LOCK: the two solves in lockstep (one column pass serves both) or one
// after the other (fewer live registers; the second runs only for uhbt /= 0).
// Y: the face is the meridional face (I, j) = (i, J) and every metric is
// its meridional counterpart (dyT, mask2dCv, dyCv; the cell beyond is
// (i, J + 1)); the operations are the zonal ones.
// VREM: the face's layers carry the vertical-viscosity remnant (F.vr).  The
// CFL limits are scaled by 1/max_k visc_rem and bound u + du visc_rem
// (zonal_mass_flux :335-433 with use_visc_rem_max), the bounding velocities
// of set_zonal_BT_cont use visc_rem_lim = max(visc_rem, 0.1 max_k visc_rem)
// (:1001-1018) and the face thickness is h_marg(u + du visc_rem) visc_rem
// (zonal_flux_thickness :730).  Without it every visc_rem is 1 and these
// reduce exactly to the forms below.
template <int CH, typename EI, bool LOCK = true, bool Y = false, bool VREM = false,
          bool AS = false>
__device__ __forceinline__ void face_work(const Dims& D, const Metrics& M, FaceCol<EI>& F,
                                          int I, int j, size_t f0, double* uh, size_t ust,
                                          bool owner, const double* uhbt2d, const ContOut& O,
                                          double dt)
{
    const int nz = D.nk;
    auto at = [&](const double* a) { return MOM6B_A2(a, I, j, D); };
    auto beyond = [&](const double* a) {
        return Y ? MOM6B_A2(a, I, j + 1, D) : MOM6B_A2(a, I + 1, j, D);
    };
    // initial fluxes and their column sums (:305-355), and the CFL limits
    // (:335-433, vol_CFL = aggress_adjust = .false.) from the same u values
    const double CFL_dt = 0.5 / dt;
    const double dx_W = at(Y ? M.dyT : M.dxT), dx_E = beyond(Y ? M.dyT : M.dxT);
    const double mCu = at(Y ? M.mask2dCv : M.mask2dCu);
    double du_max_CFL, du_min_CFL;
    double vr_max = 1.0;
    if constexpr (VREM) {
        vr_max = 0.0;
        for (int k = 1; k <= nz; ++k) vr_max = dmax(vr_max, F.vr[(size_t)(k - 1) * F.plane]);
        const double I_vrm = vr_max > 0.0 ? 1.0 / vr_max : 0.0;
        du_max_CFL = 2.0 * (CFL_dt * dx_W) * I_vrm;
        du_min_CFL = -(2.0 * (CFL_dt * dx_E) * I_vrm);
    } else {
        du_max_CFL = 2.0 * (CFL_dt * dx_W);
        du_min_CFL = -(2.0 * (CFL_dt * dx_E));
    }
    double uh_tot_0 = 0.0, duhdu_tot_0 = 0.0;
    for_layers<CH, false, Y, VREM, AS>(F, nz, [&](int k, const LayerVals& L) {
        double hm;
        double uhk = flux_eval(F, L, L.u, dt, hm);
        uh[(size_t)(k - 1) * ust] = uhk;
        duhdu_tot_0 = duhdu_tot_0 + darea<VREM>(F, L, hm);
        uh_tot_0 = uh_tot_0 + uhk;
        const double uk = L.u;
        if constexpr (VREM) {
            const double vrk = L.vr;
            if (du_max_CFL * vrk > dx_W * CFL_dt - uk * mCu)
                du_max_CFL = (dx_W * CFL_dt - uk) / vrk;
            if (du_min_CFL * vrk < -(dx_E * CFL_dt) - uk * mCu)
                du_min_CFL = -(dx_E * CFL_dt + uk) / vrk;
        } else {
            if (du_max_CFL > dx_W * CFL_dt - uk * mCu) du_max_CFL = dx_W * CFL_dt - uk;
            if (du_min_CFL < -(dx_E * CFL_dt) - uk * mCu) du_min_CFL = -(dx_E * CFL_dt + uk);
        }
    });
    du_max_CFL = dmax(du_max_CFL, 0.0);
    du_min_CFL = dmin(du_min_CFL, 0.0);

    const double fac = dt * dmin(at(M.IareaT), beyond(M.IareaT));
    const double uhbt = at(uhbt2d);
    // zonal_flux_adjust (A) and, for the owner with uhbt /= 0, the
    // zero-transport solve of set_zonal_BT_cont (B, :991-1002); with uhbt = 0
    // B would repeat A exactly, so du0 = du.
    const bool solve0 = owner && uhbt != 0.0;
    double du, du0;
    if (LOCK) {
        Newton A = newton_start(uh_tot_0 - uhbt, duhdu_tot_0, du_max_CFL, du_min_CFL, true);
        Newton B = newton_start(uh_tot_0 - 0.0, duhdu_tot_0, du_max_CFL, du_min_CFL, solve0);
        flux_adjust_pair<CH, EI, Y, VREM, AS>(F, nz, dt, uhbt, fac, A, B, uh, ust);
        du = A.du;
        du0 = solve0 ? B.du : du;
    } else {
        Newton A = newton_start(uh_tot_0 - uhbt, duhdu_tot_0, du_max_CFL, du_min_CFL, true);
        flux_adjust_one<CH, EI, Y, VREM, AS>(F, nz, dt, uhbt, fac, A, uh, ust);
        du = A.du;
        du0 = du;
        if (solve0) {
            Newton B = newton_start(uh_tot_0 - 0.0, duhdu_tot_0, du_max_CFL, du_min_CFL, true);
            flux_adjust_one<CH, EI, Y, VREM, AS>(F, nz, dt, 0.0, fac, B, (double*)nullptr, 0);
            du0 = B.du;
        }
    }
    if (!owner) return;
    O.du_cor[f0] = du;

    // set_zonal_BT_cont (:991-1121)
    const double Idt = 1.0 / dt;
    const double du_CFL = (F32(1e-6) * Idt) * at(Y ? M.dyCv : M.dxCu);
    double duR = dmin(0.0, du0 - du_CFL);
    double duL = dmax(0.0, du0 + du_CFL);
    if constexpr (VREM) {
        const double lim_min = F32(0.1) * vr_max;
        for (int k = 1; k <= nz; ++k) {
            const size_t o = (size_t)(k - 1) * F.plane;
            const double uk = F.u[o], vrk = F.vr[o];
            const double lim = dmax(vrk, lim_min);
            if (lim > 0.0) {
                if (uk + duR * lim > -(du_CFL * vrk)) duR = -(uk + du_CFL * vrk) / lim;
                if (uk + duL * lim < du_CFL * vrk) duL = -(uk - du_CFL * vrk) / lim;
            }
        }
    } else {
        // visc_rem_lim = max(1, 0.1 * 1) = 1 > 0 on every layer
        for_u<CH>(F, nz, [&](int, double uk) {
            if (uk + duR > -du_CFL) duR = -(uk + du_CFL);
            if (uk + duL < du_CFL) duL = -(uk - du_CFL);
        });
    }
    double FAmt_0 = 0.0, FAmt_L = 0.0, FAmt_R = 0.0, uhtot_L = 0.0, uhtot_R = 0.0;
    double* h_u = O.h_u + f0;
    const bool same = (du0 == du);
    for_layers<CH, kContHints, Y, VREM, AS>(F, nz, [&](int k, const LayerVals& L) {
        double hm0, hmL, hmR;
        flux_eval(F, L, u_at<VREM>(L, du0), dt, hm0);
        double uhL = flux_eval(F, L, u_at<VREM>(L, duL), dt, hmL);
        double uhR = flux_eval(F, L, u_at<VREM>(L, duR), dt, hmR);
        FAmt_0 = FAmt_0 + darea<VREM>(F, L, hm0);
        FAmt_L = FAmt_L + darea<VREM>(F, L, hmL);
        FAmt_R = FAmt_R + darea<VREM>(F, L, hmR);
        uhtot_L = uhtot_L + uhL;
        uhtot_R = uhtot_R + uhR;
        // zonal_flux_thickness with u_cor = u + du visc_rem (marginal faces)
        double hmc = hm0;
        if (!same) flux_eval(F, L, u_at<VREM>(L, du), dt, hmc);
        if constexpr (VREM) hmc = hmc * L.vr;
        if (kContHints) __stcs(h_u + (size_t)(k - 1) * F.plane, hmc);
        else h_u[(size_t)(k - 1) * F.plane] = hmc;
    });
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

// blockDim.x faces per CTA along I; consecutive CTAs overlap by one face.
// Face ownership: thread 0 recomputes the last face of the CTA to its left
// (it owns face is-1 only in the first CTA) and keeps that face's transport
// column in the CTA's own slot of uh_ovl ([CTA][nk]), so no CTA ever reads a
// global transport another CTA may still be iterating on.
__device__ __forceinline__ double* overlap_column(double* uh_ovl, int nz)
{
    return uh_ovl + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * (size_t)nz;
}

// continuity_zonal_convergence (:148-176) for cell i = I, whose faces I-1 and
// I both belong to this CTA.
__device__ __forceinline__ void cell_convergence(const Dims& D, const Metrics& M, int i, int j,
                                                 const double* __restrict__ hin,
                                                 const double* uh_left_col, const ContOut& O,
                                                 double dt)
{
    if (threadIdx.x >= 1 && i >= D.is && i <= D.ie) {
        const size_t c0 = (size_t)(j - 1) * D.n1 + (i - 1);
        const double fac = dt * MOM6B_A2(M.IareaT, i, j, D);
        const bool from_ovl = threadIdx.x == 1 && blockIdx.x > 0;
        for (int k = 1; k <= D.nk; ++k) {
            const size_t o = (size_t)(k - 1) * D.plane + c0;
            double uh_left = from_ovl ? uh_left_col[k - 1] : O.uh[o - 1];
            const double hn = dmax(hin[o] - fac * (O.uh[o] - uh_left), 0.0);
            if (kContHints) __stcs(O.h + o, hn);
            else O.h[o] = hn;
        }
    }
}

// MINB: the CTAs per SM the register allocation is held to (launch bounds).
template <int CH, int MINB = 1, bool LOCK = true, bool VREM = false, bool AS = false>
__global__ void __launch_bounds__(128, MINB)
k_cont_faces(Dims D, Metrics M, const double* __restrict__ u,
             const double* __restrict__ hin, const double* __restrict__ hW,
             const double* __restrict__ hE, const double* __restrict__ uhbt2d,
             ContOut O, double* uh_ovl, double dt, const double* __restrict__ visc_rem = nullptr)
{
    const int nz = D.nk;
    const int step = (int)blockDim.x - 1;
    const int I = D.is - 1 + (int)blockIdx.x * step + (int)threadIdx.x;
    const int j = D.js + (int)blockIdx.y;
    const bool face_ok = I <= D.ie;
    const bool owner = threadIdx.x >= 1 || blockIdx.x == 0;
    double* ovl = overlap_column(uh_ovl, nz);
    if (face_ok) {
        const size_t f0 = (size_t)(j - 1) * D.n1 + (I - 1);
        FaceCol<size_t> F;
        F.u = u + f0; F.hc = hin + f0; F.hWc = hW + f0; F.hEc = hE + f0;
        F.plane = (size_t)D.plane;
        F.estride = (size_t)D.plane;
        F.dy = MOM6B_A2(M.dy_Cu, I, j, D);
        F.IdxT_i = MOM6B_A2(M.IdxT, I, j, D);
        F.IdxT_ip1 = MOM6B_A2(M.IdxT, I + 1, j, D);
        if constexpr (VREM) F.vr = visc_rem + f0;
        if constexpr (AS) {
            extern __shared__ double cont_stage[];
            F.st = cont_stage + threadIdx.x;
            F.sts = (int)blockDim.x;
        }
        const bool to_ovl = !owner;
        double* uh = to_ovl ? ovl : O.uh + f0;
        const size_t ust = to_ovl ? 1 : F.plane;
        face_work<CH, size_t, LOCK, false, VREM, AS>(D, M, F, I, j, f0, uh, ust, owner, uhbt2d,
                                                     O, dt);
    }
    __syncthreads();  // the CTA's transport columns are complete and visible
    cell_convergence(D, M, I, j, hin, ovl, O, dt);
}

// ---------------------------------------------------------------------------
// Meridional continuity: the zonal algorithm on the v faces (i, J), J in
// [js-1, je], i in [is, ie] -- the same operations with y in place of x
// (continuity_PPM of MOM6 runs this pass after the zonal one; the reference
// mini-app is zonal only, mom6_continuity_serial.F90:143).
// ---------------------------------------------------------------------------
// PPM edges along y of cell (i, j), j in [js-1, je+1]: ppm_stencil over
// h(i, j-2 .. j+2); hS / hN take the places of h_W / h_E.
__global__ void __launch_bounds__(128)
k_ppm_edges_y(Dims D, Metrics M, const double* __restrict__ hin, double* __restrict__ hS,
              double* __restrict__ hN, double h_min)
{
    const int i = D.is + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = D.js - 1 + (int)blockIdx.y;
    const int k = 1 + (int)blockIdx.z;
    if (i > D.ie) return;
    const ptrdiff_t cm = (ptrdiff_t)(j - 1) * D.n1 + (i - 1);
    const ptrdiff_t c = (ptrdiff_t)(k - 1) * D.plane + cm;
    double h[5], m[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        h[q] = hin[c + (ptrdiff_t)(q - 2) * D.n1];
        m[q] = M.mask2dT[cm + (ptrdiff_t)(q - 2) * D.n1];
    }
    double hL, hR;
    ppm_stencil(h, m, h_min, hL, hR);
    hS[c] = hL;
    hN[c] = hR;
}

// kYTX columns x kYTY face rows per CTA; consecutive CTAs in y overlap by one
// face row, whose transports the upper CTA keeps in its overlap columns
// ([CTA][column][nk]) -- the zonal kernel's scheme along y.
constexpr int kYTX = 32, kYTY = 8;

size_t continuity_overlap_doubles_y(const Dims& D)
{
    const int nfaces = D.je - (D.js - 1) + 1;
    const size_t nbx = (size_t)(D.ie - D.is + 1 + kYTX - 1) / kYTX;
    const size_t nby = (size_t)(nfaces - 1 + kYTY - 2) / (kYTY - 1);
    return nbx * nby * kYTX * (size_t)D.nk;
}

template <int CH, int MINB, bool VREM = false>
__global__ void __launch_bounds__(kYTX * kYTY, MINB)
k_cont_faces_y(Dims D, Metrics M, const double* __restrict__ v, const double* __restrict__ hin,
               const double* __restrict__ hS, const double* __restrict__ hN,
               const double* __restrict__ vhbt2d, ContOut O, double* vh_ovl, double dt,
               const double* __restrict__ visc_rem = nullptr)
{
    const int nz = D.nk;
    const int tx = (int)threadIdx.x, ty = (int)threadIdx.y;
    const int i = D.is + (int)blockIdx.x * kYTX + tx;
    const int J = D.js - 1 + (int)blockIdx.y * (kYTY - 1) + ty;
    const bool owner = ty >= 1 || blockIdx.y == 0;
    double* ovl = vh_ovl + (((size_t)blockIdx.y * gridDim.x + blockIdx.x) * kYTX + tx) * (size_t)nz;
    if (i <= D.ie && J <= D.je) {
        const size_t f0 = (size_t)(J - 1) * D.n1 + (i - 1);
        FaceCol<size_t> F;
        F.u = v + f0; F.hc = hin + f0; F.hWc = hS + f0; F.hEc = hN + f0;
        F.plane = (size_t)D.plane;
        F.estride = (size_t)D.plane;
        F.nbh = (size_t)D.n1;
        F.nbe = (size_t)D.n1;
        F.dy = MOM6B_A2(M.dxCv, i, J, D);          // width of the v face
        F.IdxT_i = MOM6B_A2(M.IdyT, i, J, D);
        F.IdxT_ip1 = MOM6B_A2(M.IdyT, i, J + 1, D);
        if constexpr (VREM) F.vr = visc_rem + f0;
        double* vh = owner ? O.uh + f0 : ovl;
        const size_t vst = owner ? F.plane : 1;
        face_work<CH, size_t, false, true, VREM>(D, M, F, i, J, f0, vh, vst, owner, vhbt2d, O,
                                                 dt);
    }
    __syncthreads();  // the CTA's transport columns are complete and visible
    // continuity_merid_convergence of cell (i, j = J): faces J-1 (row ty-1) and J
    if (ty >= 1 && i <= D.ie && J >= D.js && J <= D.je) {
        const size_t c0 = (size_t)(J - 1) * D.n1 + (i - 1);
        const double fac = dt * MOM6B_A2(M.IareaT, i, J, D);
        const bool from_ovl = ty == 1 && blockIdx.y > 0;
        for (int k = 1; k <= nz; ++k) {
            const size_t o = (size_t)(k - 1) * D.plane + c0;
            const double vh_s = from_ovl ? ovl[k - 1] : O.uh[o - D.n1];
            const double hn = dmax(hin[o] - fac * (O.uh[o] - vh_s), 0.0);
            if (kContHints) __stcs(O.h + o, hn);
            else O.h[o] = hn;
        }
    }
}

cudaError_t launch_continuity_y(const Dims& D, const Metrics& M, const double* v,
                                const double* hin, double* hS, double* hN,
                                const double* vhbt, const ContOut& O, double* vh_ovl,
                                double dt, double h_min, cudaStream_t s,
                                const double* visc_rem)
{
    {
        dim3 grid((D.ie - D.is + 1 + 127) / 128, D.je - D.js + 3, D.nk);
        k_ppm_edges_y<<<grid, 128, 0, s>>>(D, M, hin, hS, hN, h_min);
    }
    const int nfaces = D.je - (D.js - 1) + 1;
    dim3 grid((D.ie - D.is + 1 + kYTX - 1) / kYTX, (nfaces - 1 + kYTY - 2) / (kYTY - 1), 1);
    if (visc_rem)
        k_cont_faces_y<4, 2, true><<<grid, dim3(kYTX, kYTY, 1), 0, s>>>(
            D, M, v, hin, hS, hN, vhbt, O, vh_ovl, dt, visc_rem);
    else
        k_cont_faces_y<4, 2><<<grid, dim3(kYTX, kYTY, 1), 0, s>>>(D, M, v, hin, hS, hN, vhbt, O,
                                                                  vh_ovl, dt);
    return cudaGetLastError();
}

// Fused variant: the PPM edges of the CTA's cells are computed straight into
// shared memory (no h_W/h_E scratch in HBM) and the Newton passes read them
// there; u and h come from L1/L2.  Warp w of the CTA owns faces
// F0 + 32w .. F0 + 32w + 31 and the 33 cells F0 + 32w .. F0 + 32w + 32.
constexpr int kFusedWarps = 4;
constexpr int kFusedCells = 33;   // cells per warp

template <int CH>
__global__ void __launch_bounds__(32 * kFusedWarps)
k_cont_fused(Dims D, Metrics M, const double* __restrict__ u,
             const double* __restrict__ hin, const double* __restrict__ uhbt2d,
             ContOut O, double* uh_ovl, double dt, double h_min)
{
    extern __shared__ double s_edges[];                   // [warps][2][nz][CW]
    const int nz = D.nk;
    const int CW = kFusedCells;
    const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5;
    const int wbase = warp * 2 * nz * CW;                 // this warp's h_W block
    const int ebase = wbase + nz * CW;                    // this warp's h_E block
    const int step = (int)blockDim.x - 1;
    const int F0 = D.is - 1 + (int)blockIdx.x * step;
    const int I = F0 + (int)threadIdx.x;
    const int j = D.js + (int)blockIdx.y;
    const int c0 = F0 + 32 * warp;                        // first cell of the warp
    const double* mrow = M.mask2dT + (size_t)(j - 1) * D.n1;

    // PPM edges of cells c0 .. c0+32 (within [is-1, ie+1]) for every layer
    for (int k = 1; k <= nz; ++k) {
        const double* hrow = hin + (size_t)(k - 1) * D.plane + (size_t)(j - 1) * D.n1;
        for (int c = lane; c < CW; c += 32) {
            int i = c0 + c;
            double hL = 0.0, hR = 0.0;
            if (i >= D.is - 1 && i <= D.ie + 1) ppm_cell(hrow, mrow, i, h_min, hL, hR);
            s_edges[wbase + (k - 1) * CW + c] = hL;
            s_edges[ebase + (k - 1) * CW + c] = hR;
        }
    }
    __syncwarp();

    const bool face_ok = I <= D.ie;
    const bool owner = threadIdx.x >= 1 || blockIdx.x == 0;
    double* ovl = overlap_column(uh_ovl, nz);
    if (face_ok) {
        const size_t f0 = (size_t)(j - 1) * D.n1 + (I - 1);
        FaceCol<int> F;
        F.u = u + f0; F.hc = hin + f0;
        F.hWc = s_edges + wbase + lane; F.hEc = s_edges + ebase + lane;
        F.plane = (size_t)D.plane;
        F.estride = CW;
        F.dy = MOM6B_A2(M.dy_Cu, I, j, D);
        F.IdxT_i = MOM6B_A2(M.IdxT, I, j, D);
        F.IdxT_ip1 = MOM6B_A2(M.IdxT, I + 1, j, D);
        const bool to_ovl = !owner;
        double* uh = to_ovl ? ovl : O.uh + f0;
        const size_t ust = to_ovl ? 1 : F.plane;
        face_work<CH>(D, M, F, I, j, f0, uh, ust, owner, uhbt2d, O, dt);
    }
    __syncthreads();  // the CTA's transport columns are complete and visible
    cell_convergence(D, M, I, j, hin, ovl, O, dt);
}

// ---------------------------------------------------------------------------
// Tile kernel (selected with MOM6B_CONT_TILE=1): one CTA owns 32 consecutive u faces of one row
// (lane = face) and kTileWarps warps, warp g owning a contiguous chunk of
// layers.  The h of cells F0-2 .. F0+34 and the PPM edges of cells
// F0 .. F0+32 are computed once into shared memory; each thread keeps u and
// the latest transport of its layers in registers.  Every pass over a face
// column (initial fluxes, each Newton iterate, the BT_cont test velocities)
// evaluates the layers of all warps in parallel and then hands the running
// column sums from warp to warp through named barriers, so each sum is formed
// in layer order 1..nz exactly as the serial loop forms it.  The Newton and
// BT_cont scalar logic of a face runs in the last warp.  Consecutive CTAs
// overlap by one face; lane 0 of every CTA but the first recomputes the last
// face of its left neighbour and keeps it private.
// ---------------------------------------------------------------------------
constexpr int kTileWarps = 8;
constexpr int kTileFaces = 32;
constexpr int kTileCells = kTileFaces + 1;          // cells with edges
constexpr int kTileHalo = kTileFaces + 5;           // cells with h (PPM stencil)

__device__ __forceinline__ void named_bar_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_bar_arrive(int id, int count)
{
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

template <int LMAX>
__global__ void __launch_bounds__(32 * kTileWarps, 2)
k_cont_tile(Dims D, Metrics M, const double* __restrict__ u, const double* __restrict__ hin,
            const double* __restrict__ uhbt2d, ContOut O, double dt, double h_min)
{
    extern __shared__ double sm[];
    const int nz = D.nk;
    const int HW = kTileHalo, CW = kTileCells;
    // shared layout (double offsets)
    const int oH = 0;                        // h      [nz][HW]
    const int oW = oH + nz * HW;             // h_W    [nz][CW]
    const int oE = oW + nz * CW;             // h_E    [nz][CW]
    const int oDf = oE + nz * CW;            // h_W - h_E            [nz][CW]
    const int oCv = oDf + nz * CW;           // (h_W + h_E) - 2 h    [nz][CW]
    const int oMask = oCv + nz * CW;         // mask2dT of the HW cells
    const int oCh = oMask + HW;              // chain  [4][32]
    const int oDu = oCh + 4 * 32;            // broadcast du per face
    const int oAct = oDu + 32;               // broadcast flags per face (as double)
    const int tid = (int)threadIdx.x, f = tid & 31, g = tid >> 5;
    const int F0 = D.is - 1 + (int)blockIdx.x * (kTileFaces - 1);
    const int I = F0 + f;
    const int j = D.js + (int)blockIdx.y;
    const size_t plane = (size_t)D.plane;
    const size_t row = (size_t)(j - 1) * D.n1;
    const bool face_ok = I <= D.ie;
    const bool owner = face_ok && (f >= 1 || blockIdx.x == 0);
    const int Ic = face_ok ? I : D.ie;       // clamped face for metric reads

    // ---- load h and masks, then the PPM edges of the tile's cells ----------
    for (int t = tid; t < nz * HW; t += blockDim.x) {
        const int k = t / HW, c = t - k * HW, i = F0 - 2 + c;
        sm[oH + t] = (i >= 1 && i <= D.n1) ? hin[(size_t)k * plane + row + (i - 1)] : 0.0;
    }
    for (int c = tid; c < HW; c += blockDim.x) {
        const int i = F0 - 2 + c;
        sm[oMask + c] = (i >= 1 && i <= D.n1) ? M.mask2dT[row + (i - 1)] : 0.0;
    }
    __syncthreads();
    for (int t = tid; t < nz * CW; t += blockDim.x) {
        const int k = t / CW, c = t - k * CW, i = F0 + c;
        double hL = 0.0, hR = 0.0;
        if (i >= D.is - 1 && i <= D.ie + 1)
            ppm_stencil(&sm[oH + k * HW + c], &sm[oMask + c], h_min, hL, hR);
        sm[oW + t] = hL;
        sm[oE + t] = hR;
        // (other - base) of either upwind case is +-(h_W - h_E) exactly, and
        // curv_3 = (h_W + h_E) - 2 h in both (addition commutes)
        sm[oDf + t] = hL - hR;
        sm[oCv + t] = (hL + hR) - 2.0 * sm[oH + k * HW + c + 2];
    }

    // ---- per-thread layer chunk and face constants --------------------------
    const int L = (nz + kTileWarps - 1) / kTileWarps;
    const int k0 = g * L + 1;
    const int nmine = max(0, min(L, nz - k0 + 1));
    const double dy = MOM6B_A2(M.dy_Cu, Ic, j, D);
    const double Idx_i = MOM6B_A2(M.IdxT, Ic, j, D), Idx_p = MOM6B_A2(M.IdxT, Ic + 1, j, D);
    double uk[LMAX], uhk[LMAX], tA[LMAX], tB[LMAX];
#pragma unroll
    for (int c = 0; c < LMAX; ++c) {
        uk[c] = (c < nmine) ? u[(size_t)(k0 + c - 1) * plane + row + (Ic - 1)] : 0.0;
        uhk[c] = 0.0; tA[c] = 0.0; tB[c] = 0.0;
    }
    __syncthreads();

    // zonal_flux_layer at face velocity uI for layer k (flux_eval on the tile)
    auto eval = [&](int k, double uI, double& hm) -> double {
        const bool pos = uI > 0.0;
        const int cc = pos ? f : f + 1;
        const int e = (k - 1) * CW + cc;
        const double base = sm[(pos ? oE : oW) + e];
        const double dfc = sm[oDf + e];
        const double d = pos ? dfc : -dfc;               // other - base
        const double curv_3 = sm[oCv + e];
        const double Idx = pos ? Idx_i : Idx_p;
        const double CFL = fabs(uI) * dt * Idx;
        const double uh = dy * uI * (base + CFL * (0.5 * d + curv_3 * (CFL - 1.5)));
        const double hmm = base + CFL * (d + 3.0 * curv_3 * (CFL - 1.0));
        if (!(uI > 0.0) && !(uI < 0.0)) {
            hm = 0.5 * (sm[oW + (k - 1) * CW + f + 1] + sm[oE + (k - 1) * CW + f]);
            return 0.0;
        }
        hm = hmm;
        return uh;
    };
    // hand the running values v[0..nv) from warp g-1 to warp g, add this
    // warp's layers with add(c, v), pass them on; the last warp keeps them
    auto chain = [&](int nv, double* v, auto&& add) {
        if (g > 0) {
            named_bar_sync(g, 64);
            for (int q = 0; q < nv; ++q) v[q] = sm[oCh + q * 32 + f];
        }
#pragma unroll
        for (int c = 0; c < LMAX; ++c)
            if (c < nmine) add(c, v);
        if (g < kTileWarps - 1) {
            for (int q = 0; q < nv; ++q) sm[oCh + q * 32 + f] = v[q];
            named_bar_arrive(g + 1, 64);
        }
    };
    const bool last = g == kTileWarps - 1;

    // ---- initial fluxes and CFL limits (:305-433) ----------------------------
    const double CFL_dt = 0.5 / dt;
    const double dx_W = MOM6B_A2(M.dxT, Ic, j, D), dx_E = MOM6B_A2(M.dxT, Ic + 1, j, D);
    const double mCu = MOM6B_A2(M.mask2dCu, Ic, j, D);
#pragma unroll
    for (int c = 0; c < LMAX; ++c)
        if (c < nmine) {
            double hm;
            uhk[c] = eval(k0 + c, uk[c], hm);
            tA[c] = dy * hm;
        }
    double v4[4] = {0.0, 0.0, 2.0 * (CFL_dt * dx_W), -(2.0 * (CFL_dt * dx_E))};
    chain(4, v4, [&](int c, double* v) {
        v[0] = v[0] + uhk[c];
        v[1] = v[1] + tA[c];
        if (v[2] > dx_W * CFL_dt - uk[c] * mCu) v[2] = dx_W * CFL_dt - uk[c];
        if (v[3] < -(dx_E * CFL_dt) - uk[c] * mCu) v[3] = -(dx_E * CFL_dt + uk[c]);
    });
    // Newton state of the face (last warp only)
    const double uhbt = MOM6B_A2(uhbt2d, Ic, j, D);
    const double fac = dt * dmin(MOM6B_A2(M.IareaT, Ic, j, D), MOM6B_A2(M.IareaT, Ic + 1, j, D));
    const double tol_eta_cs = 1.0e-12, tol_vel = 3.0e8;
    const int max_itts = 20;
    const double uh_tot_0 = v4[0], duhdu_tot_0 = v4[1];
    const double du_max_CFL = dmax(v4[2], 0.0), du_min_CFL = dmin(v4[3], 0.0);
    double du = 0.0, du_max = du_max_CFL, du_min = du_min_CFL;
    double uh_err = uh_tot_0 - uhbt, duhdu_tot = duhdu_tot_0, uh_err_best = fabs(uh_err);
    int itt = 1;
    bool do_I = face_ok;
    // one decision of zonal_flux_adjust's loop (:813-890) for iteration itt
    auto decide = [&]() {
        if (!do_I) return;
        double tol_eta;
        if (itt <= 1) tol_eta = F32(1e-6) * tol_eta_cs;
        else if (itt == 2) tol_eta = F32(1e-4) * tol_eta_cs;
        else if (itt == 3) tol_eta = F32(1e-2) * tol_eta_cs;
        else tol_eta = tol_eta_cs;
        if (uh_err > 0.0) du_max = du;
        else if (uh_err < 0.0) du_min = du;
        else do_I = false;
        if (!do_I) return;
        const double ae = fabs(uh_err);
        if ((fac * ae > tol_eta) || ((ae > tol_vel * duhdu_tot) || (ae > uh_err_best))) {
            const double ddu = -(uh_err / duhdu_tot);
            const double du_prev = du;
            du = du + ddu;
            if (fabs(ddu) < F32(1.0e-15) * fabs(du)) {
                do_I = false;
            } else if (ddu > 0.0) {
                if (du >= du_max) {
                    du = 0.5 * (du_prev + du_max);
                    if (du_max - du_prev < F32(1.0e-15) * fabs(du)) do_I = false;
                }
            } else if (du <= du_min) {
                du = 0.5 * (du_prev + du_min);
                if (du_prev - du_min < F32(1.0e-15) * fabs(du)) do_I = false;
            }
        } else {
            do_I = false;
        }
    };
    // Newton passes: keep_uh selects zonal_flux_adjust (transports kept) or
    // the zero-transport solve of set_zonal_BT_cont (nothing kept)
    auto newton = [&](double target, bool keep_uh) {
        for (;;) {
            if (last) {
                decide();
                sm[oDu + f] = du;
                sm[oAct + f] = do_I ? 1.0 : 0.0;
            }
            if (!__syncthreads_or(last && do_I)) break;
            const double du_b = sm[oDu + f];
            const bool act = sm[oAct + f] != 0.0;
#pragma unroll
            for (int c = 0; c < LMAX; ++c)
                if (c < nmine && act) {
                    double hm;
                    const double uh = eval(k0 + c, uk[c] + du_b, hm);
                    if (keep_uh) uhk[c] = uh;
                    tB[c] = uh;
                    tA[c] = dy * hm;
                }
            double v2[2] = {target, 0.0};
            chain(2, v2, [&](int c, double* v) {
                v[0] = v[0] + tB[c];
                v[1] = v[1] + tA[c];
            });
            if (last && do_I) {
                if (itt < max_itts) {
                    uh_err = v2[0];
                    duhdu_tot = v2[1];
                    uh_err_best = dmin(uh_err_best, fabs(uh_err));
                }
                ++itt;
                if (itt > max_itts) do_I = false;
            }
            __syncthreads();
        }
    };
    newton(-uhbt, true);
    const double du_cor = du;

    // ---- set_zonal_BT_cont (:991-1121) ---------------------------------------
    if (last) {   // zero-transport solve only where uhbt != 0
        du = 0.0; du_max = du_max_CFL; du_min = du_min_CFL;
        uh_err = uh_tot_0; duhdu_tot = duhdu_tot_0; uh_err_best = fabs(uh_err);
        itt = 1;
        do_I = owner && uhbt != 0.0;
    }
    __syncthreads();
    newton(-0.0, false);   // e = -uhbt with uhbt = 0
    if (last) {
        const double du0 = (owner && uhbt != 0.0) ? du : du_cor;
        sm[oDu + f] = du0;
        sm[oAct + f] = du_cor;   // reused: du_cor of the face
    }
    __syncthreads();
    const double du0 = sm[oDu + f];
    const double du_c = sm[oAct + f];
    const double Idt = 1.0 / dt;
    const double du_CFL = (F32(1e-6) * Idt) * MOM6B_A2(M.dxCu, Ic, j, D);
    double vLR[2] = {dmin(0.0, du0 - du_CFL), dmax(0.0, du0 + du_CFL)};   // duR, duL
    chain(2, vLR, [&](int c, double* v) {
        if (uk[c] + v[0] > -du_CFL) v[0] = -(uk[c] + du_CFL);
        if (uk[c] + v[1] < du_CFL) v[1] = -(uk[c] - du_CFL);
    });
    if (last) {
        sm[oCh + 0 * 32 + f] = vLR[0];
        sm[oCh + 1 * 32 + f] = vLR[1];
    }
    __syncthreads();
    const double duR = sm[oCh + f], duL = sm[oCh + 32 + f];
    __syncthreads();
    const bool same = du0 == du_c;
    // test velocities u + du0 (FAmt_0, and h_u at u_cor = u + du for the
    // marginal faces) and u + duL (FAmt_L, uhtot_L) in one pass
    double tC[LMAX];
#pragma unroll
    for (int c = 0; c < LMAX; ++c)
        if (c < nmine) {
            double hm0;
            eval(k0 + c, uk[c] + du0, hm0);
            tA[c] = dy * hm0;
            double hmc = hm0;
            if (!same) eval(k0 + c, uk[c] + du_c, hmc);
            if (owner) O.h_u[(size_t)(k0 + c - 1) * plane + row + (I - 1)] = hmc;
            double hmL;
            tC[c] = eval(k0 + c, uk[c] + duL, hmL);
            tB[c] = dy * hmL;
        }
    double v0[1], vL[2];
    {
        double v3[3] = {0.0, 0.0, 0.0};
        chain(3, v3, [&](int c, double* v) {
            v[0] = v[0] + tA[c];
            v[1] = v[1] + tB[c];
            v[2] = v[2] + tC[c];
        });
        v0[0] = v3[0]; vL[0] = v3[1]; vL[1] = v3[2];
    }
    __syncthreads();
    // test velocity u + duR: FAmt_R, uhtot_R
#pragma unroll
    for (int c = 0; c < LMAX; ++c)
        if (c < nmine) {
            double hm;
            tB[c] = eval(k0 + c, uk[c] + duR, hm);
            tA[c] = dy * hm;
        }
    double vR[2] = {0.0, 0.0};
    chain(2, vR, [&](int c, double* v) {
        v[0] = v[0] + tA[c];
        v[1] = v[1] + tB[c];
    });
    if (last && owner) {
        const size_t f0 = row + (I - 1);
        O.du_cor[f0] = du_c;
        const double FAmt_0 = v0[0], FAmt_L = vL[0], uhtot_L = vL[1];
        const double FAmt_R = vR[0], uhtot_R = vR[1];
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

    // ---- transports and continuity_zonal_convergence (:148-176) --------------
    const int i = I;   // cell i = I uses faces I-1 (lane f-1) and I (lane f)
    const bool cell_ok = f >= 1 && i >= D.is && i <= D.ie;
    const double facc = cell_ok ? dt * MOM6B_A2(M.IareaT, i, j, D) : 0.0;
#pragma unroll
    for (int c = 0; c < LMAX; ++c) {
        const double uh_left = __shfl_up_sync(0xffffffffu, uhk[c], 1);
        if (c < nmine) {
            const size_t o = (size_t)(k0 + c - 1) * plane + row;
            if (owner) O.uh[o + (I - 1)] = uhk[c];
            if (cell_ok) {
                const double hc = sm[oH + (k0 + c - 1) * HW + f + 2];
                O.h[o + (i - 1)] = dmax(hc - facc * (uhk[c] - uh_left), 0.0);
            }
        }
    }
}

// CTAs per SM for k_cont_faces; 0 lets the hardware fill the SM.
constexpr int kContCtasPerSM = 0;
// CTAs per SM the face kernel's registers are held to: 4 (128 registers) is
// the fastest on B200 (the unconstrained build takes 204 registers, 2 CTAs).
constexpr int kContMinBlocks = 4;

size_t continuity_overlap_doubles(const Dims& D)
{
    // at most one CTA per 127 faces along each row (both kernels use 128 threads)
    int nfaces = D.ie - (D.is - 1) + 1;
    size_t nbx = (size_t)(nfaces - 1 + 126) / 127;
    return nbx * (size_t)(D.je - D.js + 1) * (size_t)D.nk;
}

cudaError_t launch_continuity(const Dims& D, const Metrics& M, const double* u,
                              const double* hin, double* hW, double* hE,
                              const double* uhbt, const ContOut& O, double* uh_ovl,
                              double dt, double h_min, cudaStream_t s,
                              const double* visc_rem)
{
    // The tile kernel keeps every column on chip (a quarter of the face
    // kernel's DRAM traffic) but is bounded by its serial column sums; the
    // face kernel below is faster on B200 and stays the default.
    if (!visc_rem && D.nk <= 16 * kTileWarps && getenv("MOM6B_CONT_TILE")) {
        const size_t smem = ((size_t)D.nk * (kTileHalo + 4 * kTileCells) + kTileHalo + 6 * 32) *
                            sizeof(double);
        const int nfaces = D.ie - (D.is - 1) + 1;
        dim3 grid((nfaces - 1 + kTileFaces - 2) / (kTileFaces - 1), D.je - D.js + 1, 1);
        if (D.nk <= 10 * kTileWarps) {
            cudaError_t e = cudaFuncSetAttribute(k_cont_tile<10>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
            k_cont_tile<10><<<grid, 32 * kTileWarps, smem, s>>>(D, M, u, hin, uhbt, O, dt, h_min);
        } else {
            cudaError_t e = cudaFuncSetAttribute(k_cont_tile<16>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
            k_cont_tile<16><<<grid, 32 * kTileWarps, smem, s>>>(D, M, u, hin, uhbt, O, dt, h_min);
        }
        return cudaGetLastError();
    }
    {
        const int nb = 32 * kFusedWarps, step = nb - 1;
        size_t smem = (size_t)kFusedWarps * 2 * D.nk * kFusedCells * sizeof(double);
        if (!visc_rem && smem <= 227 * 1024 && getenv("MOM6B_CONT_FUSED")) {
            cudaError_t e = cudaFuncSetAttribute(
                k_cont_fused<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            int nfaces = D.ie - (D.is - 1) + 1;
            dim3 grid((nfaces - 1 + step - 1) / step, D.je - D.js + 1, 1);
            k_cont_fused<1><<<grid, nb, smem, s>>>(D, M, u, hin, uhbt, O, uh_ovl, dt, h_min);
            return cudaGetLastError();
        }
    }
    {
        static int edges_warp = -1;
        if (edges_warp < 0) {
            const char* e = getenv("MOM6B_PPM_WARP");
            edges_warp = e ? atoi(e) : 1;
        }
        int n = (D.ie + 1) - (D.is - 1) + 1;
        if (edges_warp) {
            const int warps = (n + kEdgeCellsPerWarp - 1) / kEdgeCellsPerWarp;
            dim3 grid((warps + 3) / 4, D.je - D.js + 1, (D.nk + kEdgeLayers - 1) / kEdgeLayers);
            k_ppm_edges_warp<<<grid, 128, 0, s>>>(D, M, hin, hW, hE, h_min);
        } else {
            dim3 grid((n + 127) / 128, D.je - D.js + 1, D.nk);
            k_ppm_edges<<<grid, 128, 0, s>>>(D, M, hin, hW, hE, h_min);
        }
    }
    {
        // Residency: each face re-reads its column on every Newton pass, so
        // the resident CTAs' columns should stay in L2.  The dynamic shared
        // memory request is padded to cap the CTAs per SM (kContCtasPerSM).
        const int nb = 128, step = nb - 1;
        int nfaces = D.ie - (D.is - 1) + 1;
        dim3 grid((nfaces - 1 + step - 1) / step, D.je - D.js + 1, 1);
        size_t smem = 0;
        static int ctas = -1;
        if (ctas < 0) {
            const char* e = getenv("MOM6B_CONT_CTAS_PER_SM");
            ctas = e ? atoi(e) : kContCtasPerSM;
        }
        if (ctas > 0) smem = (size_t)(227 * 1024) / (size_t)ctas - 1024;
        static int chunk = -1;
        if (chunk < 0) {
            const char* e = getenv("MOM6B_CONT_CHUNK");
            chunk = e ? atoi(e) : kContChunk;
        }
        static int minb = -1;
        if (minb < 0) {
            const char* e = getenv("MOM6B_CONT_MINB");
            minb = e ? atoi(e) : kContMinBlocks;
        }
        static int lock = -1;
        if (lock < 0) {
            const char* e = getenv("MOM6B_CONT_LOCK");
            lock = e ? atoi(e) : 0;   // one solve after the other: 3.87 ms per step (lockstep 3.92)
        }
        auto kern = chunk == 1   ? k_cont_faces<1>
                    : chunk == 4 ? (lock ? (minb == 4 ? k_cont_faces<4, 4>
                                            : minb == 5 ? k_cont_faces<4, 5>
                                                        : k_cont_faces<4>)
                                         : (minb == 4 ? k_cont_faces<4, 4, false>
                                            : minb == 5 ? k_cont_faces<4, 5, false>
                                                        : k_cont_faces<4, 3, false>))
                                 : (minb == 4 ? k_cont_faces<2, 4> : k_cont_faces<2>);
        // the remnant form runs the default shape only
        if (visc_rem) kern = k_cont_faces<4, 4, false, true>;
        // staged sweeps (chunks of 3 layers copied with cp.async while the
        // previous 3 are evaluated): 3.50 ms per step against 3.60 loading
        // chunks of 4 into registers (2: 3.68, 4 at 3 CTAs/SM: 3.62)
        static int cas = -1;
        if (cas < 0) {
            const char* e = getenv("MOM6B_CONT_ASYNC");
            cas = e ? atoi(e) : 3;
        }
        if (!visc_rem && cas == 2) {
            kern = k_cont_faces<2, 4, false, false, true>;
            smem = (size_t)2 * 2 * 7 * nb * sizeof(double);
        } else if (!visc_rem && cas == 3) {
            kern = k_cont_faces<3, 4, false, false, true>;
            smem = (size_t)2 * 3 * 7 * nb * sizeof(double);
        } else if (!visc_rem && cas == 4) {
            kern = k_cont_faces<4, 3, false, false, true>;
            smem = (size_t)2 * 4 * 7 * nb * sizeof(double);
        }
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, nb, smem, s>>>(D, M, u, hin, hW, hE, uhbt, O, uh_ovl, dt, visc_rem);
    }
    return cudaGetLastError();
}

} // namespace mom6b
