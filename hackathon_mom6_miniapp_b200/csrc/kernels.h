// kernels.h -- parameter blocks and host launchers of the FP64 step kernels.
#pragma once

#include "common.cuh"

namespace mom6b {

// Products of the uniform metrics that the fast FP64 tendency multiplies
// by (formed on the host when the metrics are uniform; the serial
// expressions with the metrics factored out): rel = kRv dv - kRu du,
// q = absv kQn / (S + kQe) with S the four-cell thickness sum of hArea_q,
// str_xy = (kSv dv + kSu du) (h00 + h10 + h01 + h11), KE = kKu (uc^2 + um^2)
// + kKv (vc^2 + vm^2), str_xx = h (kXv dv - kXu du), uh = kTu u (h + h+),
// vh = kTv v (h + h+), CAu = kCu (q0 s0 + q1 s1) - IdxCu dKE, CAv = -kCv
// (...) - IdyCv dKE, h_u = kHm (h + h+), diffu = (kDq dstr_xy + kDh
// dstr_xx) / (h_u + h_neglect), diffv = (kEq dstr_xy - kEh dstr_xx) / (h_v
// + h_neglect).
struct TendFold {
    double kRv, kRu, kQn, kQe, kSv, kSu, kKu, kKv, kXu, kXv, kTu, kTv, kCu, kCv, kHm, kDq,
        kDh, kEq, kEh;
};

// Spatially uniform metrics as scalars.  init_ocean_grid builds every metric
// array uniform (mom6_types.F90:193-228) except CoriolisBu, which varies with
// j only; when the model detects this it passes the values here and the
// kernels read them from the parameter bank instead of 2-D arrays.  The
// exact kernels' arithmetic is unchanged: the same values enter the same
// operations (the fast tendency also multiplies by the products in tf).
struct UniMetrics {
    double IareaT, areaT, dxT, IdxT, dxCu, dyCu, dy_Cu, IdxCu, IdyCu, dxCv, dyCv,
        IdxCv, IdyCv, IareaBu, IareaCu, IareaCv, mask2dT, mask2dBu, mask2dCu,
        mask2dCv, Area_q, DX_dyT, DY_dxT, DX_dyBu, DY_dxBu, dx2h, dy2h, dx2q, dy2q,
        red_xx, red_xy, Kh_xx, Kh_xy;
    const double* cor_row;  // CoriolisBu(:, J) for J = 1..n2 (constant in i)
    int valid;              // 1 when the grid qualifies
    TendFold tf;            // the fast tendency's products (when valid)
    // barotropic metrics (barotropic_init): scalars, and f_4_u/f_4_v per row
    double Datu, Datv, gtot_E, gtot_W, gtot_N, gtot_S, bt_rem_u, bt_rem_v;
    const double* f4u_row;  // f_4_u(c, :, J) at [(J-1)*4 + c-1]
    const double* f4v_row;
    int valid_bt;
};

// vertical viscosity constants (vert_visc_init, mom6_vert_visc_serial.F90:60-112)
struct VVParams {
    double Kv, Kv_ml, Kv_extra_bbl, Hmix, h_neglect, I_Hbbl;
};

// outputs of continuity_PPM: thickness, transports and BT_cont
struct ContOut {
    double* h;
    double* uh;
    double* h_u;
    double *FA_u_W0, *FA_u_WW, *FA_u_E0, *FA_u_EE, *uBT_WW, *uBT_EE, *du_cor;
};

// barotropic work arrays (barotropic_CS, mom6_barotropic_serial.F90:20-58)
struct BTWork {
    double *eta, *eta_pred, *ubt, *vbt, *ubt_prev, *vbt_prev, *uhbt, *vhbt,
        *PFu, *PFv, *ubt_av, *vbt_av;
    unsigned int* bar_count;   // grid barrier state (zeroed at allocation)
    unsigned int* bar_gen;
    int* status;               // kDevOk / kDevTimeout
    unsigned int* tile_flag;   // per-tile substep counters (kBtMaxTiles entries)
};

// Upper bound on the tiles of the tiled barotropic kernel (one or two per SM).
constexpr int kBtMaxTiles = 512;

struct BTParams {
    double dtbt, dgeo_de, trans_wt1, trans_wt2, inv_nstep;
    int nstep, first_direction, extended;
    long long spin_budget;     // clock64 cycles a block may wait at one barrier
    // Testing aid for the timeout path: 1 makes the loop's first grid barrier
    // wait for one more block than the launch holds, an arrival that never
    // comes, so every block's wait runs into spin_budget, records kDevTimeout
    // and returns.  0 in normal use.
    int stall_test = 0;
    // 1: the point-parallel persistent kernel even where the tiled one fits
    int untiled = 0;
    // Part of the loop one launch runs (the point-parallel kernel, privates in
    // the global work arrays): 0 all of it; kBtInit the state copies and the
    // zeroed averages only; n >= 1 substep n only; kBtFinish the output copy
    // only.  A decomposed run exchanges halos between the launches.
    int substep = 0;
};
constexpr int kBtInit = -1, kBtFinish = -2;

// The default wait limit of the barotropic barriers: 2^31 clock64 cycles,
// about 1.1 s at the B200's 1965 MHz.
constexpr long long kBtDefaultWait = 2147483648LL;

// diffu, diffv (both or neither): also store the horizontal-viscosity
// accelerations of the updated points (diagnostics); with ext_visc they are
// inputs instead (launch_hor_visc_gen's) and the kernel does not evaluate
// the Laplacian.  scheme: the Coriolis scheme (1 SADOURNY75_ENERGY,
// 2 ARAKAWA_HSU90, 3 ARAKAWA_LAMB81).
cudaError_t launch_tendency(const Dims& D, const Metrics& M, const UniMetrics& U,
                            const double* uin, const double* vin, const double* h,
                            const double* ubase, const double* vbase, double* uout,
                            double* vout, double coef, double h_neglect, cudaStream_t s,
                            double* diffu = nullptr, double* diffv = nullptr, int scheme = 1,
                            bool ext_visc = false, int* status = nullptr);
// The fast FP64 form (k_tendency_fast.cu): Sadourny scheme, no diagnostics.
// status (optional): with it, the uniform-metric Sadourny tendency stages its
// tiles with TMA and records kDevTimeout there if a tile never lands.
cudaError_t launch_tendency_fast(const Dims& D, const Metrics& M, const UniMetrics& U,
                                 const double* uin, const double* vin, const double* h,
                                 const double* ubase, const double* vbase, double* uout,
                                 double* vout, double coef, double h_neglect, cudaStream_t s,
                                 int* status = nullptr);
// rem_u, rem_v (both or neither): also the vertical-viscosity remnant of
// every u / v column (vert_visc_remnant).
cudaError_t launch_vertvisc(const Dims& D, const Metrics& M, double* u, double* v,
                            const double* h, double dt, const VVParams& P,
                            double* taux_bot, double* tauy_bot, cudaStream_t s,
                            double* rem_u = nullptr, double* rem_v = nullptr);
// uh_ovl: scratch of continuity_overlap_doubles(D) doubles holding the
// recomputed overlap face column of every CTA.
size_t continuity_overlap_doubles(const Dims& D);
// Meridional continuity (v faces; O.uh receives vh, O.h_u h_v and the BT_cont
// fields their meridional counterparts); vh_ovl holds
// continuity_overlap_doubles_y(D) doubles; hS, hN are scratch like hW, hE.
size_t continuity_overlap_doubles_y(const Dims& D);
cudaError_t launch_continuity_y(const Dims& D, const Metrics& M, const double* v,
                                const double* hin, double* hS, double* hN,
                                const double* vhbt, const ContOut& O, double* vh_ovl,
                                double dt, double h_min, cudaStream_t s,
                                const double* visc_rem = nullptr);
// visc_rem (optional, (n1, n2, nk)): the vertical-viscosity remnant of the
// faces; the fluxes then follow zonal_mass_flux's use_visc_rem form.
cudaError_t launch_continuity(const Dims& D, const Metrics& M, const double* u,
                              const double* hin, double* hW, double* hE,
                              const double* uhbt, const ContOut& O, double* uh_ovl,
                              double dt, double h_min, cudaStream_t s,
                              const double* visc_rem = nullptr);
// The fast forms of the vertical viscosity (k_vv_fast.cu): FP64 and the
// mixed form's FP32 storage with the elimination in double.
bool vertvisc_fast_fits(const Dims& D);
cudaError_t launch_vertvisc_fast(const Dims& D, const Metrics& M, double* u, double* v,
                                 const double* h, double dt, const VVParams& P,
                                 double* taux_bot, double* tauy_bot, cudaStream_t s);
cudaError_t launch_vertvisc_fast_f(const Dims& D, const Metrics& M, float* u, float* v,
                                   const float* h, double dt, const VVParams& P,
                                   double* taux_bot, double* tauy_bot, cudaStream_t s);
// The fast FP64 form of the zonal continuity (k_cont_fast.cu): no scratch
// arrays; status receives kDevTimeout if a tile load never lands.  Only for
// grids with continuity_fast_fits(D) (nk <= 128).
bool continuity_fast_fits(const Dims& D);
cudaError_t launch_continuity_fast(const Dims& D, const Metrics& M, const double* u,
                                   const double* hin, const double* uhbt, const ContOut& O,
                                   double dt, double h_min, int* status, cudaStream_t s);
cudaError_t launch_btstep(const Dims& D, const Metrics& M, const UniMetrics& U,
                          const BTWork& W,
                          const BTParams& P, const double* eta_in,
                          const double* ubt_in, const double* vbt_in, double* u_av,
                          double* v_av, double* eta_av, cudaStream_t s);
// The same loop, also leaving the substep-averaged transports in W.uhbt /
// W.vhbt (tiled grids only; cudaErrorNotSupported otherwise).
cudaError_t launch_btstep_tavg(const Dims& D, const Metrics& M, const UniMetrics& U,
                               const BTWork& W, const BTParams& P, const double* eta_in,
                               const double* ubt_in, const double* vbt_in, double* u_av,
                               double* v_av, double* eta_av, cudaStream_t s);
cudaError_t launch_halo_fill(const Dims& D, double* f, int nz, int kind, cudaStream_t s);
// The barotropic loop on the library's static scratch (no allocation), with
// the caller's metric arrays in M and parameters in P; MOM6B_NOALLOC_* codes.
int btstep_static(const double* eta_in, const double* ubt_in, const double* vbt_in,
                  double* u_av, double* v_av, double* eta_av, const Metrics& M, const Dims& D,
                  BTParams P, cudaStream_t s);

// Mixed-precision form (k_mixed.cu): FP32 state and stencils, FP64 column
// sums, Newton scalars, thickness update and tridiagonal elimination.
cudaError_t launch_halo_fill_f(const Dims& D, float* f, int nz, int kind, cudaStream_t s);
// The fills of an h-, a u- and a v-point field (kinds 0, 1, 2) in one launch.
cudaError_t launch_halo_fill3(const Dims& D, double* fh, double* fu, double* fv, int nz,
                              cudaStream_t s);
cudaError_t launch_halo_fill3_f(const Dims& D, float* fh, float* fu, float* fv, int nz,
                                cudaStream_t s);
cudaError_t launch_tendency_f(const Dims& D, const Metrics& M, const UniMetrics& U,
                              const float* uin, const float* vin, const float* h,
                              const float* ubase, const float* vbase, float* uout,
                              float* vout, float coef, float h_neglect, cudaStream_t s);
// f32_elim: the tridiagonal elimination in FP32 too (opt-in; the mixed form
// eliminates in FP64)
cudaError_t launch_vertvisc_f(const Dims& D, const Metrics& M, float* u, float* v,
                              const float* h, double dt, const VVParams& P, double* taux_bot,
                              double* tauy_bot, cudaStream_t s, bool f32_elim = false);
// O2 supplies the FP64 2-D outputs (BT_cont face areas, du_cor); h, uh, h_u
// are the FP32 3-D outputs.
cudaError_t launch_continuity_f(const Dims& D, const Metrics& M, const float* u,
                                const float* hin, float* hW, float* hE, const double* uhbt,
                                float* h, float* uh, float* h_u, const ContOut& O2,
                                double* uh_ovl, double dt, double h_min, cudaStream_t s);

// ---------------------------------------------------------------------------
// Ensemble: many independent domains advanced in the mixed form with one
// launch per phase for all of them (k_ensemble.cu, and k_btstep.cu for the
// FP64 barotropic loop).
// ---------------------------------------------------------------------------
// One domain: dimensions, metrics, parameters and device arrays (3-D state in
// FP32).  An array of these lives in device memory; each CTA of a batched
// kernel copies its domain's entry to shared memory first.
struct EnsDomain {
    Dims D;
    Metrics M;
    UniMetrics U;
    float *u, *v, *hA, *hB, *h0, *up, *vp, *uh, *hW, *hE, *h_u, *ovl;
    double *uhbt0, *taux_bot, *tauy_bot;
    ContOut O2;                 // FP64 2-D outputs of continuity (h, uh, h_u unused)
    double *eta, *ubt, *vbt, *ubt_av, *vbt_av, *eta_av;
    BTWork W;                   // barotropic work arrays (control words unused)
    VVParams VV;
    BTParams P;
    double dt, h_min;
    float hv_neglect;
    int bc_fill;
};

// Launch shapes of the batched kernels, chosen by the ensemble's autotuner.
struct EnsTuning {
    int tend;      // tendency tile: index into kEnsTendTiles
    int tend_kc;   // layers per tendency CTA
    int vv_nb;     // vertvisc threads per CTA (64, 128, 256)
    int vv_ch;     // vertvisc layers per prefetch (2, 4)
    int ppm_nb;    // PPM edge threads per CTA (128, 256)
    int faces_nb;  // continuity faces per CTA + 1 (64, 128, 256)
    int bt_tile;   // largest barotropic tile edge (32, 48, 64)
};

constexpr int kEnsTendTiles[4][2] = {{32, 8}, {32, 4}, {64, 4}, {32, 16}};

// Barotropic tiles of one domain: nbx x nby tiles of tw x th points covering
// [is-1, ie] x [js-1, je]; t0 is the domain's first tile in the global list.
struct EnsBtGeo {
    int nbx, nby, tw, th, t0;
};

// Blocks each batched kernel gives one domain under a tuning (host side).
long long ens_blocks_tendency(const Dims& D, const EnsTuning& T);
long long ens_blocks_vertvisc(const Dims& D, const EnsTuning& T);
long long ens_blocks_ppm(const Dims& D, const EnsTuning& T);
long long ens_blocks_faces(const Dims& D, const EnsTuning& T);
long long ens_blocks_halo(const Dims& D, int which);
// FP32 overlap slots continuity needs for one domain at the smallest face block.
size_t ens_ovl_floats(const Dims& D);
EnsBtGeo ens_bt_geometry(const Dims& D, int max_edge);

// half: 0 = predictor, 1 = corrector.  start[d] is domain d's first block
// (start[n] = total).  uni: every domain has uniform metrics.
cudaError_t launch_ens_tendency(const EnsDomain* doms, const int* start, int n, int total,
                                int half, const EnsTuning& T, bool uni, cudaStream_t s);
cudaError_t launch_ens_vertvisc(const EnsDomain* doms, const int* start, int n, int total,
                                int half, int kmax, const EnsTuning& T, cudaStream_t s);
cudaError_t launch_ens_ppm(const EnsDomain* doms, const int* start, int n, int total, int half,
                           const EnsTuning& T, cudaStream_t s);
cudaError_t launch_ens_faces(const EnsDomain* doms, const int* start, int n, int total,
                             int half, const EnsTuning& T, cudaStream_t s);
// which: 0 = after the predictor (hB, up, vp), 1 = after the corrector (hA, u,
// v), 2 = between the barotropic calls (eta_av, ubt_av, vbt_av), 3 = after
// them (eta).  Jobs are (domain, field) pairs, start over n * fields(which).
cudaError_t launch_ens_halo(const EnsDomain* doms, const int* start, int njobs, int total,
                            int which, cudaStream_t s);
// The barotropic loop of every domain in one cooperative persistent launch.
// call 0: eta, ubt, vbt -> ubt_av, vbt_av, eta_av; call 1: eta_av, ubt_av,
// vbt_av -> ubt_av, vbt_av, eta.  ctl supplies the barrier words, status and
// one flag per tile.
cudaError_t launch_ens_btstep(const EnsDomain* doms, const EnsBtGeo* geo, const int* tstart,
                              int n, int ntiles, int max_tw, int max_th, int call,
                              int max_nstep, const BTWork& ctl, bool uni, cudaStream_t s);

}  // namespace mom6b
