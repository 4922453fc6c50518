// k_continuity.cu -- zonal PPM continuity (FP64), the exact form.
//
// Restates continuity_PPM of mom6_continuity_serial.F90:100-1294 as
// rk2_serial_driver calls it (:293, :380), operation for operation (built
// without FMA contraction, column sums in layer order), so the step is
// bit-identical to the serial driver; k_cont_fast.cu is the fast form.
//   k_ppm_edges_warp  PPM_reconstruction_x + PPM_limit_pos (:1124-1294), lane
//                 per cell, h_W/h_E to a scratch pair;
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
#include "cont_impl.cuh"

namespace mom6b {

// ---------------------------------------------------------------------------
// PPM edge values
// ---------------------------------------------------------------------------
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
constexpr bool kContHints = true;

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

size_t continuity_overlap_doubles(const Dims& D)
{
    // at most one CTA per 127 faces along each row (both kernels use 128 threads)
    int nfaces = D.ie - (D.is - 1) + 1;
    size_t nbx = (size_t)(nfaces - 1 + 126) / 127;
    return nbx * (size_t)(D.je - D.js + 1) * (size_t)D.nk;
}

// The exact form: the PPM edges of every cell (lane per cell, slopes shared by
// shuffle) into the hW/hE scratch pair, then one thread per face.  Shapes
// measured fastest on B200 at 720x720x75: registers held to 4 CTAs per SM
// (the unconstrained build takes 204 registers, 2 CTAs), the two Newton
// solves one after the other (lockstep: 3.92 against 3.87 ms per step), and
// the column sweeps staging chunks of 3 layers in shared memory with cp.async
// while the previous 3 are evaluated (3.50 ms per step against 3.60 loading
// chunks of 4 into registers).  The remnant form loads chunks of 4 into
// registers.
cudaError_t launch_continuity(const Dims& D, const Metrics& M, const double* u,
                              const double* hin, double* hW, double* hE,
                              const double* uhbt, const ContOut& O, double* uh_ovl,
                              double dt, double h_min, cudaStream_t s,
                              const double* visc_rem)
{
    {
        const int n = (D.ie + 1) - (D.is - 1) + 1;
        const int warps = (n + kEdgeCellsPerWarp - 1) / kEdgeCellsPerWarp;
        dim3 grid((warps + 3) / 4, D.je - D.js + 1, (D.nk + kEdgeLayers - 1) / kEdgeLayers);
        k_ppm_edges_warp<<<grid, 128, 0, s>>>(D, M, hin, hW, hE, h_min);
    }
    const int nb = 128, step = nb - 1;
    const int nfaces = D.ie - (D.is - 1) + 1;
    dim3 grid((nfaces - 1 + step - 1) / step, D.je - D.js + 1, 1);
    if (visc_rem) {
        k_cont_faces<4, 4, false, true><<<grid, nb, 0, s>>>(D, M, u, hin, hW, hE, uhbt, O,
                                                            uh_ovl, dt, visc_rem);
        return cudaGetLastError();
    }
    constexpr int CH = 3;
    const size_t smem = (size_t)2 * CH * 7 * nb * sizeof(double);
    auto kern = k_cont_faces<CH, 4, false, false, true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, nb, smem, s>>>(D, M, u, hin, hW, hE, uhbt, O, uh_ovl, dt, nullptr);
    return cudaGetLastError();
}

} // namespace mom6b
