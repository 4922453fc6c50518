/*
 * mom6_oracle.h -- CPU restatement of the MOM6 mini-app's split RK2 step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle for the B200 library:
 * it restates, in plain C, the serial Fortran path of the reference
 * (app/rk2_serial_driver.F90, the Fortran files of src/serial and
 * src/common/mom6_types.F90).
 * Only tests/, the smoke check and the cpu_baseline leg of bench.py may link
 * or call it; the product library never does.
 *
 * Pinning: the reference has no golden vectors and its Fortran does not
 * compile here, but its CUDA C kernels (the .cu files of src/cuda_c) build from their
 * sources into oracle/_ref.  Where the serial semantics and those kernels
 * coincide -- horizontal viscosity, the Sadourny Coriolis term, vertical
 * viscosity without Rayleigh drag, and btstep with extended ranges -- the
 * GPU tests (tests/test_gpu_oracle_pin.py) run this oracle's phase functions
 * and the reference kernels on the same inputs and compare them.
 *
 * Array convention: every field is stored exactly as the reference stores it,
 * Fortran column-major with 1-based indices, dimensions (n1, n2[, nk]) with
 * n1 = ni + 2, n2 = nj + 2 (mom6_types.F90:145-148).
 *
 * Floating point: built with -ffp-contract=off, so every a*b+c is two
 * roundings, as the reference's x86-64 -O3 gfortran build computes it.  The
 * single-precision quirks of the serial Fortran (default-real literals such as
 * 1e-6, 1e-15, 1e-12, 0.1 and the real(4) locals of PPM_limit_pos) are kept.
 */
#ifndef MOM6_ORACLE_H
#define MOM6_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Initial-state constructions. */
enum {
    OR_INIT_REF = 0, /* analytic fields of rk2_serial_driver.F90:466-542 */
    OR_INIT_CFG = 1  /* seeded beta-plane construction (Philox4x32-10) */
};

/* Field identifiers shared with the product's mom6b.h (same numbering). */
enum {
    OR_F_U = 0, OR_F_V, OR_F_H, OR_F_H0, OR_F_UH, OR_F_VH, OR_F_UP, OR_F_VP,
    OR_F_ETA, OR_F_UBT, OR_F_VBT, OR_F_UBT_AV, OR_F_VBT_AV, OR_F_ETA_AV,
    OR_F_HU_BT, OR_F_FA_U_W0, OR_F_FA_U_WW, OR_F_FA_U_E0, OR_F_FA_U_EE,
    OR_F_UBT_WW, OR_F_UBT_EE, OR_F_DU_COR, OR_F_TAUX_BOT, OR_F_TAUY_BOT,
    OR_F_TAUX, OR_F_TAUY, OR_F_RAY_U, OR_F_RAY_V, OR_F_CAU, OR_F_CAV,
    OR_F_DIFFU, OR_F_DIFFV,
    /* meridional continuity (oracle_set_merid): h_v and BT_cont's v fields */
    OR_F_HV_BT, OR_F_FA_V_S0, OR_F_FA_V_SS, OR_F_FA_V_N0, OR_F_FA_V_NN,
    OR_F_VBT_SS, OR_F_VBT_NN, OR_F_DV_COR,
    /* the vertical-viscosity remnant (oracle_set_remnant) */
    OR_F_VISC_REM_U, OR_F_VISC_REM_V, OR_F_COUNT
};

typedef struct oracle_model oracle_model;

typedef struct {
    int ni, nj, nk;
    int bt_nsteps;
    int init_mode;      /* OR_INIT_REF / OR_INIT_CFG */
    uint64_t seed;      /* CFG mode only */
    double dt;          /* baroclinic step [s] */
    double dx_km;       /* grid spacing [km] */
    double lat_deg;     /* REF-mode central latitude for the beta plane */
    double Kh;          /* Laplacian viscosity [m2 s-1] */
    double Kv, Kv_ml, Kv_extra_bbl, Hmix, Hbbl;
    int bc_fill;        /* 1: apply the periodic-x / wall-y halo fill */
    /* one subdomain of a decomposed run (mpi_domain_init, mom6_mpi_domain.F90:
     * 57-137): the global ni, nj (0: this model is the whole domain) and the
     * offsets of this model's compute domain in the global one; the initial
     * state and the grid are those of the global points.  cuts: OR_CUT_* bits,
     * the sides where a neighbouring subdomain lies (no wall). */
    int ni_global, nj_global, i_offset, j_offset;
    int cuts;
} oracle_config;

enum { OR_CUT_W = 1, OR_CUT_E = 2, OR_CUT_S = 4, OR_CUT_N = 8 };

/* The halo exchange of a decomposed run: called on a field (n1 x n2 x nz,
 * Fortran order) whose halo must be refreshed from the neighbours before the
 * next phase reads it.  kind: 0 h points, 1 u faces, 2 v faces. */
typedef void (*oracle_exchange_fn)(void *ctx, double *field, int nz, int kind);

void oracle_config_default(oracle_config *c, int init_mode);

oracle_model *oracle_create(const oracle_config *c);
void oracle_destroy(oracle_model *m);

/* One split RK2 iteration of rk2_serial_driver.F90:218-399 per call. */
void oracle_step(oracle_model *m, int nsteps);

/* Driver diagnostics (rk2_serial_driver.F90 with diag_mode = 1): when on,
 * every step records the fields its diffu_sum and diffv_sum posts carry
 * (mom6_diag's persistent work_2d after each product sum) and each
 * oracle_step call ends with KE and mass of the final state.  which: 0
 * diffu_sum, 1 diffv_sum, 2 KE (n1*n2*nk), 3 mass (n1*n2). */
void oracle_diag_enable(oracle_model *m, int on);
int oracle_diag_get(const oracle_model *m, int which, double *out);

/* Meridional continuity.  on = 1: every continuity of the step runs the
 * zonal pass into an intermediate thickness (the full input array, whose
 * computational domain the pass updates; with bc_fill its halo filled), then
 * the meridional pass from it into h, with vh and the v fields of BT_cont.
 * The meridional pass is the zonal restatement applied to the transposed
 * problem ((i, j) -> (j, i); dyT, IdyT, dxCv, mask2dCv, dyCv in the places of
 * dxT, IdxT, dy_Cu, mask2dCu, dxCu) and transposed back. */
void oracle_set_merid(oracle_model *m, int on);

/* The vertical-viscosity remnant fed to continuity.  on = 1: every vertical
 * viscosity of the step is followed by vert_visc_remnant
 * (mom6_vert_visc_serial.F90:295-387) with the same dt, and the next
 * continuity uses visc_rem_u (and the meridional pass visc_rem_v) in place of
 * the driver's 1. */
void oracle_set_remnant(oracle_model *m, int on);
void oracle_vert_visc_remnant(oracle_model *m, double dt);

/* Coriolis scheme of CorAdCalc (mom6_coriolis_serial.F90:19-21, :171-193,
 * :211-248): 1 SADOURNY75_ENERGY (default, the driver's), 2 ARAKAWA_HSU90,
 * 3 ARAKAWA_LAMB81.  0 on success. */
int oracle_set_coriolis_scheme(oracle_model *m, int scheme);

/* hor_visc_init's scheme options (mom6_hor_visc_serial.F90:160-193): the
 * model is created with Laplacian only (the driver's).  modified_leith sets
 * CS%modified_Leith, which hor_visc_init has no argument for.  Resets the
 * module's work arrays as hor_visc_init does.  0 on success. */
typedef struct {
    int laplacian, biharmonic, smagorinsky, leith, no_slip, better_bound, modified_leith;
    double Ah;   /* background biharmonic viscosity [m4 s-1] (default 1e10) */
} oracle_hor_visc_opts;
int oracle_set_hor_visc(oracle_model *m, const oracle_hor_visc_opts *o);
void oracle_continuity_merid(oracle_model *m, const double *v, const double *hin,
                             double *h, double *vh, double dt);

/* Field access: element count = n1*n2 (2-D) or n1*n2*nk (3-D). */
size_t oracle_field_size(const oracle_model *m, int field);
int oracle_get(const oracle_model *m, int field, double *out);
int oracle_set(oracle_model *m, int field, const double *in);
void oracle_dims(const oracle_model *m, int *out8);
/* btstep transport ranges: 0 serial (default), 1 extended (CUDA C kernels). */
void oracle_set_bt_extended(oracle_model *m, int on);
void oracle_set_bt_first_direction(oracle_model *m, int d);
/* Install the halo exchange of a decomposed run (NULL: none).  The step then
 * exchanges up, vp before the predictor continuity, h after it, u, v before
 * the corrector continuity, and the barotropic eta, ubt, vbt before every
 * substep; the ranges that stop short of a wall reach the cut instead. */
void oracle_set_exchange(oracle_model *m, oracle_exchange_fn fn, void *ctx);
/* Copy a named grid / control-structure array (see mom6_oracle.c). */
int oracle_array(const oracle_model *m, const char *name, double *out, size_t count); /* n1 n2 nk is ie js je ... */

/* verify_state of rk2_serial_driver.F90:563-623: out = {mass_init,
 * mass_final, rel_error, max_u, max_v, max_eta, ke_total}. */
void oracle_verify(const oracle_model *m, double *out7);

/* Single physics phases on the model's grid, for per-kernel tests.  Each
 * operates on caller arrays laid out (n1, n2[, nk]) and on the model's
 * persistent work arrays exactly as the serial module does. */
void oracle_compute_transports(oracle_model *m, const double *u, const double *v,
                               const double *h, double *uh, double *vh);
void oracle_hor_visc(oracle_model *m, const double *u, const double *v,
                     const double *h, double *diffu, double *diffv);
void oracle_coriolis(oracle_model *m, const double *u, const double *v,
                     const double *h, const double *uh, const double *vh,
                     double *CAu, double *CAv);
void oracle_vert_visc(oracle_model *m, double *u, double *v, const double *h,
                      double dt);
void oracle_btstep(oracle_model *m, const double *eta_in, const double *ubt_in,
                   const double *vbt_in, double *u_av, double *v_av,
                   double *eta_av);
void oracle_continuity(oracle_model *m, const double *u, const double *hin,
                       double *h, double *uh, double dt);
void oracle_halo_fill(const oracle_model *m, double *f, int nz, int kind);

/* Philox4x32-10 normal deviate used by the CFG initial state. */
/* Threads of the row-parallel loops in the OpenMP build (liboracle_omp.so);
 * n <= 0 keeps the runtime's choice.  Returns the threads in use (1 in the
 * single-threaded build). */
int oracle_set_threads(int n);
double oracle_normal(uint64_t seed, uint32_t stream, uint64_t index);

#ifdef __cplusplus
}
#endif
#endif
