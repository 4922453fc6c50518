/*
 * mom6b.h -- high-level C ABI of the B200 split RK2 library (libmom6b.so).
 *
 * A model owns the ocean grid of init_ocean_grid (mom6_types.F90:130-258),
 * the state of rk2_serial_driver (u, v, h, h0, eta, ubt, vbt, ...) resident in
 * HBM, and the fused sm_100a kernels that advance it by whole split RK2
 * iterations with the semantics of rk2_serial_driver.F90:218-399.  Every
 * function returns a MOM6B_* status; mom6b_last_error() gives a message.
 *
 * Arrays crossing this boundary use the reference layout: Fortran
 * column-major, 1-based, dimensions (n1, n2[, nk]) with n1 = ni + 2 and
 * n2 = nj + 2, double precision.  No torch types appear in this header.
 *
 * The reference-compatible per-kernel entry points (launch_* and cuda_*_c of
 * the reference's src/cuda_c backend) are declared in mom6_cuda_c.h.
 */
#ifndef MOM6B_H
#define MOM6B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum {
    MOM6B_OK = 0,
    MOM6B_ERR_ARG = 1,      /* invalid argument (sizes, null pointers, ids) */
    MOM6B_ERR_CUDA = 2,     /* a CUDA runtime call failed */
    MOM6B_ERR_NOMEM = 3,    /* device or host allocation failed */
    MOM6B_ERR_TIMEOUT = 4,  /* a grid-wide barrier gave up waiting */
    MOM6B_ERR_STATE = 5     /* call not valid in the current state */
};

/* initial-state constructions */
enum {
    MOM6B_INIT_REF = 0, /* analytic fields of rk2_serial_driver.F90:466-542 */
    MOM6B_INIT_CFG = 1  /* seeded beta plane: h = H/nk (1 + 0.01 N), u,v ~ N(0,0.05),
                           Gaussian eta bump, f = 1e-4 + 2e-11 (y - Ly/2) */
};

/* arithmetic forms */
enum {
    MOM6B_FP64 = 0,  /* every field and every operation in double precision */
    MOM6B_MIXED = 1  /* fields, stencils and the vertical-viscosity
                        coefficients in single precision; the continuity column
                        sums, the thickness update, the vertical tridiagonal
                        elimination and the barotropic loop in double */
};

/* field ids (get/set) */
enum {
    MOM6B_F_U = 0, MOM6B_F_V, MOM6B_F_H, MOM6B_F_H0, MOM6B_F_UH, MOM6B_F_VH,
    MOM6B_F_UP, MOM6B_F_VP, MOM6B_F_ETA, MOM6B_F_UBT, MOM6B_F_VBT,
    MOM6B_F_UBT_AV, MOM6B_F_VBT_AV, MOM6B_F_ETA_AV, MOM6B_F_HU_BT,
    MOM6B_F_FA_U_W0, MOM6B_F_FA_U_WW, MOM6B_F_FA_U_E0, MOM6B_F_FA_U_EE,
    MOM6B_F_UBT_WW, MOM6B_F_UBT_EE, MOM6B_F_DU_COR, MOM6B_F_TAUX_BOT,
    MOM6B_F_TAUY_BOT, MOM6B_F_TAUX, MOM6B_F_TAUY, MOM6B_F_RAY_U, MOM6B_F_RAY_V,
    MOM6B_F_COUNT,
    /* the meridional continuity's outputs (mom6b_set_continuity_merid); ids
       28..31 are the oracle's Coriolis and viscosity fields */
    MOM6B_F_HV_BT = 32, MOM6B_F_FA_V_S0, MOM6B_F_FA_V_SS, MOM6B_F_FA_V_N0,
    MOM6B_F_FA_V_NN, MOM6B_F_VBT_SS, MOM6B_F_VBT_NN, MOM6B_F_DV_COR,
    /* the vertical-viscosity remnant at u and v points
       (mom6b_set_visc_remnant) */
    MOM6B_F_VISC_REM_U = 40, MOM6B_F_VISC_REM_V
};

typedef struct mom6b_config {
    int ni, nj, nk;        /* computational sizes as passed to init_ocean_grid */
    int bt_nsteps;         /* barotropic substeps per btstep call */
    int init_mode;         /* MOM6B_INIT_REF / MOM6B_INIT_CFG */
    uint64_t seed;         /* CFG initial state seed */
    double dt;             /* baroclinic step [s] */
    double dx_km;          /* grid spacing [km] */
    double lat_deg;        /* REF beta-plane latitude [deg] */
    double Kh;             /* Laplacian viscosity [m2 s-1] */
    double Kv, Kv_ml, Kv_extra_bbl, Hmix, Hbbl; /* vertical viscosity */
    int bc_fill;           /* 1: periodic-x / solid-wall-y halo fill per step */
    int precision;         /* MOM6B_FP64 / MOM6B_MIXED */
    int device;            /* CUDA device ordinal */
    int use_graph;         /* 1: replay each step from a captured CUDA graph */
    int exact;             /* 1: every FP64 kernel keeps the serial driver's
                              roundings (no FMA contraction, column sums in
                              layer order): the step is bit-identical to
                              rk2_serial_driver.  0 (default): the FP64
                              kernels may contract multiply-adds and sum
                              columns in another order; every prognostic
                              field stays within a relative L2 of 1e-12 of
                              the exact form after 10 steps */
    int bt_untiled;        /* 1: the point-parallel barotropic kernel even where
                              the tiled one fits (both give the same answers) */
    int general_metrics;   /* 1: read every metric from its 2-D array even when
                              the grid is uniform (same answers) */
    long long wait_cycles; /* limit of each barotropic barrier wait in clock64
                              cycles; 0: the default (2^31, about 1.1 s) */
    int mixed_f32_vertvisc;/* MOM6B_MIXED only, opt-in: the vertical tridiagonal
                              elimination in FP32 as well (outside the mixed
                              form's definition, which eliminates in FP64) */
    /* One subdomain of a 2-D decomposition (mpi_domain_init,
     * mom6_mpi_domain.F90:57-137, non-periodic).  ni_global, nj_global: the
     * whole domain's ni, nj (0: this model is the whole domain); ni, nj
     * above are then this subdomain's (its compute width + 4), and i_offset,
     * j_offset the 0-based offsets of its compute domain in the global one.
     * The grid and the initial state are those of the global points
     * (init_ocean_grid_mpi, :144-258).  cuts: MOM6B_CUT_* bits, the sides
     * with a neighbouring subdomain; a step with cuts needs a halo exchange
     * (mom6b_set_exchange). */
    int ni_global, nj_global, i_offset, j_offset;
    int cuts;
} mom6b_config;

enum { MOM6B_CUT_W = 1, MOM6B_CUT_E = 2, MOM6B_CUT_S = 4, MOM6B_CUT_N = 8 };

typedef struct mom6b_model mom6b_model;

/* Fill *cfg with the defaults of the given initial-state mode:
 * REF: 180x180x75, dt 300 s, Kh 100, no halo fill (rk2_serial_driver.F90:91-143);
 * CFG: 180x180x75, dt 600 s, Kh 1000, halo fill on. */
int mom6b_config_default(mom6b_config *cfg, int init_mode);

/* Allocate the model on cfg->device, build grid metrics and the initial state
 * on the host and upload them.  Sizes must satisfy ni, nj >= 8, nk >= 2. */
int mom6b_create(const mom6b_config *cfg, mom6b_model **out);
int mom6b_destroy(mom6b_model *m);

/* Enqueue nsteps split RK2 iterations on the model's stream (asynchronous). */
int mom6b_step(mom6b_model *m, int nsteps);
/* Block until all enqueued work has finished; reports barrier timeouts. */
int mom6b_synchronize(mom6b_model *m);

/* Number of doubles in a field (n1*n2 or n1*n2*nk); 0 for an unknown id. */
size_t mom6b_field_size(const mom6b_model *m, int field);
/* Copy a field to / from host memory (synchronous). */
int mom6b_get_field(mom6b_model *m, int field, double *host, size_t count);
int mom6b_set_field(mom6b_model *m, int field, const double *host, size_t count);
/* Device address of a field (reference layout), for zero-copy callers. */
int mom6b_field_device_ptr(mom6b_model *m, int field, void **dptr);
/* out = {n1, n2, nk, is, ie, js, je, bt_nsteps} (1-based compute bounds). */
int mom6b_dims(const mom6b_model *m, int *out8);
/* The model's CUDA stream, as a cudaStream_t cast to void*. */
int mom6b_stream(mom6b_model *m, void **stream);

/* End-to-end step through host buffers: upload u, v, h, eta (pinned host
 * pointers may be passed), run nsteps, download u, v, h, eta.  Any pointer may
 * be NULL to skip that field. */
int mom6b_step_host(mom6b_model *m, int nsteps, double *u, double *v, double *h,
                    double *eta);
/* The same with the step's inputs and outputs apart: upload u_in, v_in,
 * eta_in (the state a step reads; h restarts from h0 at every step,
 * rk2_serial_driver.F90:225-232, so an uploaded h would be overwritten
 * unread), run nsteps, download u_out, v_out, h_out, eta_out.  Any pointer
 * may be NULL; an input and an output may be the same buffer.  With
 * nsteps = 1 (FP64, a whole domain) the barotropic chain, which reads only
 * eta, ubt and vbt, runs beside the upload of u and v. */
int mom6b_step_host_io(mom6b_model *m, int nsteps, const double *u_in, const double *v_in,
                       const double *eta_in, double *u_out, double *v_out, double *h_out,
                       double *eta_out);

/* verify_state of rk2_serial_driver.F90:563-623 computed on the device:
 * out = {mass_init, mass_final, rel_error, max_u, max_v, max_eta, ke_total}. */
int mom6b_verify(mom6b_model *m, double *out7);

/* Bound of every barotropic barrier wait of later steps (clock64 cycles; 0:
 * the default) and, with stall_test = 1, a testing aid that makes the first
 * barrier of each barotropic loop wait for an arrival that never comes: its
 * wait runs into the limit, every block returns, and mom6b_synchronize
 * reports MOM6B_ERR_TIMEOUT (the step's barotropic outputs are then
 * incomplete).  The model stays usable: set stall_test = 0 and step again. */
int mom6b_set_wait_limit(mom6b_model *m, long long cycles, int stall_test);

/* ---- domain decomposition (no reference counterpart in src/cuda_c: the
 * reference decomposes in its MPI drivers, rk2_mpi_cuda_c_driver.F90:248-577,
 * with halo_exchange_3d / _2d of mom6_mpi_halo_omp.F90:106-427) ----
 *
 * A halo exchange refreshes the halo of one of the model's device fields
 * (n1 x n2 x nz, Fortran order; kind 0 h points, 1 u faces, 2 v faces) from
 * the neighbouring subdomains.  The step calls it from the host thread that
 * called mom6b_step, with the model's stream, at these points: up, vp before
 * the predictor continuity, the predictor's h after it, u, v before the
 * corrector continuity, and the barotropic eta, ubt, vbt before every
 * substep.  The fields of one point come in consecutive calls, all but the
 * last with more = 1: an exchange may hold them and move them together when
 * the call with more = 0 comes, and every field of the point must be
 * exchanged when that call returns.  It returns 0, or nonzero to abandon the
 * step (mom6b_step then returns MOM6B_ERR_STATE).  Work it enqueues on the
 * stream is ordered with the step's kernels.  With cuts, the ranges that stop short of a wall
 * (velocity update, CorAdCalc's u and v points) reach the cut, CorAdCalc's
 * and hor_visc's intermediates on the cut exist, and the barotropic loop
 * runs one launch per substep on ranges two points into the halo, so that
 * the decomposed step equals the single-domain one bit for bit (exact
 * form).  Supported: MOM6B_FP64 without halo fill, the default Sadourny
 * Coriolis and Laplacian hor_visc, zonal continuity, no remnant, no
 * diagnostics, no surrogate; the step is not captured in a CUDA graph. */
typedef int (*mom6b_exchange_fn)(void *ctx, double *field, int nz, int kind, int more,
                                 void *stream);
int mom6b_set_exchange(mom6b_model *m, mom6b_exchange_fn fn, void *ctx);

/* An in-process exchange among npes_x * npes_y subdomain models (one host
 * thread per model, on one or several devices; rank = pos_x * npes_y +
 * pos_y as MPI_Cart_create orders a 2-D grid).  Each exchange point posts
 * its fields, waits for every member, copies each neighbour's edge strips
 * into this model's halos (peer copies between devices), and waits again
 * before the owners may change them.  East/west strips span the compute rows plus
 * the halo rows on a side without a north/south neighbour, north/south
 * strips the compute columns plus the halo columns on a side without an
 * east/west neighbour, the corner blocks come from the diagonal neighbours,
 * so every halo point is written once.  A member that does not arrive
 * within timeout_s seconds fails the exchange of the others. */
typedef struct mom6b_halo_group mom6b_halo_group;
int mom6b_halo_group_create(int npes_x, int npes_y, double timeout_s, mom6b_halo_group **out);
/* Install the group's exchange on m as member `rank` (m's cuts must be its
 * position's). */
int mom6b_halo_group_join(mom6b_halo_group *g, mom6b_model *m, int rank);
void mom6b_halo_group_destroy(mom6b_halo_group *g);

/* Per-kernel launch accounting: number of kernels of this library launched
 * on the model's stream since the last reset. */
int64_t mom6b_launch_count(const mom6b_model *m);
void mom6b_reset_launch_count(mom6b_model *m);

/* Set a timing hook: the step records CUDA events around the dominant kernel
 * so callers can read its average duration (milliseconds per launch). */
int mom6b_kernel_timing(mom6b_model *m, int enable);
int mom6b_kernel_time_ms(mom6b_model *m, const char *kernel, double *avg_ms,
                         int64_t *launches);

/* ---- diagnostics (mom6_diag.F90) ----------------------------------------
 * The mini-app's diagnostic module for fields resident on the device, one
 * per model.  mom6b_diag_init replaces diag_init (:77-112; output_freq >= 1);
 * mom6b_diag_register replaces register_diag_field (:130-166) and gives the
 * id (-1 for MOM6B_DIAG_NONE or when 100 fields are registered).  A post
 * (post_data_2d / post_data_3d, :169-272; the product sums of
 * post_product_sum_u / _v, :274-334, on the GPU) counts a call, prints
 * "  Diag: <name> min/max/mean/rms: " and the four values of the
 * computational domain in Fortran ES14.6 when the mode has STATS, and when
 * it has FILE writes every output_freq-th call to
 * <output_dir>/<name><6-digit call count>.bin: ni, nj[, nk] as int32, then
 * the computational domain as float64, column-major (:362-431).  Posts are
 * synchronous; fields are device arrays of the model's shape.  The product
 * sums share one work array, which keeps the points a sum does not cover. */
enum { MOM6B_DIAG_NONE = 0, MOM6B_DIAG_STATS = 1, MOM6B_DIAG_FILE = 2, MOM6B_DIAG_BOTH = 3 };
int mom6b_diag_init(mom6b_model *m, const char *output_dir, int output_freq);
int mom6b_diag_end(mom6b_model *m);
int mom6b_diag_register(mom6b_model *m, const char *name, const char *long_name,
                        const char *units, int ndims, const char *position,
                        int output_mode, int *id);
int mom6b_diag_post_2d(mom6b_model *m, int id, const double *field);
int mom6b_diag_post_3d(mom6b_model *m, int id, const double *field);
int mom6b_diag_post_product_sum_u(mom6b_model *m, int id, const double *u_a,
                                  const double *u_b);
int mom6b_diag_post_product_sum_v(mom6b_model *m, int id, const double *v_a,
                                  const double *v_b);
/* out4 = {min, max, mean, rms} of the last post of id. */
int mom6b_diag_stats(const mom6b_model *m, int id, double *out4);
/* out3 = {registered fields, post calls, call count}; prints the summary of
 * diag_report_timing (:336-346). */
int mom6b_diag_report(mom6b_model *m, int *out3);
/* The diagnostics of rk2_serial_driver with diag_mode = 1 (:152-170):
 * registers KE, diffu_sum, diffv_sum and mass with output_mode; from then on
 * every mom6b_step iteration posts diffu_sum and diffv_sum (the predictor's
 * horizontal viscosity summed with the predicted thickness, :299-304) and
 * every mom6b_step call ends with KE and mass of the final state (:385-391).
 * FP64 form only; steps then run without the CUDA graph. */
int mom6b_diag_driver(mom6b_model *m, int output_mode);

/* Coriolis scheme of CorAdCalc in the step (coriolis_init's scheme argument,
 * mom6_coriolis_serial.F90:19-21): 1 SADOURNY75_ENERGY (the default, the
 * driver's), 2 ARAKAWA_HSU90, 3 ARAKAWA_LAMB81 (:171-193, :228-248).  The
 * Arakawa schemes are built for the FP64 form. */
enum { MOM6B_SADOURNY75_ENERGY = 1, MOM6B_ARAKAWA_HSU90 = 2, MOM6B_ARAKAWA_LAMB81 = 3 };
int mom6b_set_coriolis_scheme(mom6b_model *m, int scheme);

/* Meridional continuity (MOM6's continuity_PPM follows the zonal pass with
 * it; the reference mini-app is zonal only, mom6_continuity_serial.F90:143).
 * on = 1: every continuity of the step runs the zonal pass into an
 * intermediate thickness (a copy of the input whose computational domain the
 * pass updates; its halo filled when bc_fill), then the meridional pass --
 * the zonal algorithm on the v faces with the y metrics -- into h, writing vh
 * (MOM6B_F_VH), h_v and the v fields of BT_cont (MOM6B_F_HV_BT ..
 * MOM6B_F_DV_COR).  FP64 form only. */
int mom6b_set_continuity_merid(mom6b_model *m, int on);
/* One continuity pass of one direction on the model's fields, as one call of
 * continuity_PPM: dir 0 zonal, from u and h0 into h, uh, h_u and BT_cont's u
 * fields; dir 1 meridional, from v and h0 into h, vh, h_v and the v fields
 * (after mom6b_set_continuity_merid(m, 1)).  Only the computational domain
 * of h is written.  With mom6b_set_visc_remnant(m, 1) the pass reads the
 * model's visc_rem_u / visc_rem_v.  FP64 form; synchronous. */
int mom6b_continuity_pass(mom6b_model *m, int dir, double dt);

/* on = 1: the barotropic chain of each step (both btstep calls and their
 * halo fills) runs on a second stream concurrently with the 3-D chain; its
 * inputs (eta, ubt, vbt) and outputs are disjoint from the 3-D chain's, so
 * the results are unchanged.  The btstep is a cooperative launch whose
 * blocks wait at grid barriers; blocks that become resident while the 3-D
 * kernels hold SMs wait (bounded) for the rest. */
int mom6b_set_bt_overlap(mom6b_model *m, int on);

/* hor_visc_init's scheme options (mom6_hor_visc_serial.F90:160-193); the
 * model starts with the driver's: Laplacian only, free slip, no bounds.
 * Smagorinsky applies to whichever of the Laplacian and biharmonic
 * viscosities is on, Leith to the Laplacian and (with biharmonic) the
 * biharmonic one; better_bound sets the thickness-aware bounds of both;
 * modified_leith (CS%modified_Leith, no hor_visc_init argument) adds the
 * divergence gradient to Leith's.  Kh is the config's; Ah the background
 * biharmonic viscosity (hor_visc_init's default 1e10 m4 s-1).  Any option
 * other than the driver's runs a separate hor_visc kernel before each
 * tendency (FP64 form). */
typedef struct mom6b_hor_visc {
    int laplacian, biharmonic, smagorinsky, leith, no_slip, better_bound, modified_leith;
    double Ah;
} mom6b_hor_visc;
int mom6b_set_hor_visc(mom6b_model *m, const mom6b_hor_visc *opts);

/* The vertical-viscosity remnant (vert_visc_remnant,
 * mom6_vert_visc_serial.F90:295-387; the reference's step does not call it,
 * MOM6's continuity_PPM takes it as visc_rem_u / visc_rem_v).  on = 1: every
 * vertvisc of the step also writes visc_rem_u / visc_rem_v (MOM6B_F_VISC_REM_U
 * / _V; 1 in masked columns and outside the vertvisc ranges), the fraction of
 * a barotropic acceleration each layer keeps after the implicit viscosity,
 * and the continuity after it runs with use_visc_rem: the CFL limits, the
 * Newton velocities, the marginal areas, BT_cont's bounding velocities and
 * the face thicknesses carry visc_rem (mom6_continuity_serial.F90:335-433,
 * :581, :880, :1001-1018, :730).  FP64 form only. */
int mom6b_set_visc_remnant(mom6b_model *m, int on);

/* Dump one field's computational domain in the diagnostics' binary format
 * (a checkpoint; mixed-form fields are written as their values in double), or
 * restore it from such a file (the halo is left as is).  Synchronous. */
int mom6b_write_field_bin(mom6b_model *m, int field, const char *path);
int mom6b_read_field_bin(mom6b_model *m, int field, const char *path);

/* ---- allocation-free barotropic loop ------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory where they run the barotropic solver -- a Fortran host whose device
 * arrays belong to an OpenMP-target or OpenACC runtime, which owns the device
 * pool and which a separate cudaMalloc would bypass -- this entry point runs all
 * nstep substeps of btstep (mom6_barotropic_serial.F90:178-304; extended
 * uhbt/vhbt ranges when extended_ranges != 0, as btstep_do_step and the CUDA C
 * kernels use) and allocates nothing.  The caller passes every input, metric
 * and output as device arrays in the reference layout (n1, n2; f_4_u and
 * f_4_v are (4, n1, n2)); the outputs may alias the inputs.  The loop's work
 * arrays live in one static device array of the library sized for
 * n1 * n2 <= 589,824 points (768 x 768, about 28.3 MB per GPU, held until the
 * process exits); larger grids return MOM6B_NOALLOC_ERR_TOO_LARGE.  The loop
 * also splits its updated box of bw x bh = (ie - is + 2) x (je - js + 2)
 * points into tiles of at most 64 x 64, at most one per SM, so it needs
 * ceil(bw / 64) * ceil(bh / 64) <= the SM count (148 on a B200: every square
 * box of the capacity, 1024 x 576 and the like qualify; a 4096 x 144 box does
 * not); a box that does not qualify also returns MOM6B_NOALLOC_ERR_TOO_LARGE.
 * All calls share that array, so calls that overlap on the GPU race.  The
 * first call on each device looks up the array's device address: make it
 * before any stream capture.  The work is enqueued on `stream` (a
 * cudaStream_t); the call does not synchronize.
 *
 * The loop's grid barriers wait a bounded time (about 1.1 s by default); a
 * barrier that gives up makes every block return and leaves a timeout status
 * in the static array.  mom6b_btstep_noalloc_status synchronizes `stream`,
 * reads that status for the current device and clears it: it returns
 * MOM6B_NOALLOC_ERR_TIMEOUT when the last call's loop gave up (its outputs
 * are then incomplete), MOM6B_NOALLOC_OK otherwise.  Query it before the next
 * call on that device, which resets the status.
 * mom6b_btstep_noalloc_set_wait sets the wait limit of later calls in clock64
 * cycles (0: the default); stall_test = 1 is a testing aid that makes the
 * loop's first barrier wait for an arrival that never comes, so that the
 * timeout path can be exercised without a fault. */
enum {
    MOM6B_NOALLOC_OK = 0,
    MOM6B_NOALLOC_ERR_ARG = 1,       /* null pointer or inconsistent bounds */
    MOM6B_NOALLOC_ERR_TOO_LARGE = 2, /* grid above the static capacity */
    MOM6B_NOALLOC_ERR_CUDA = 3,      /* a CUDA runtime call failed */
    MOM6B_NOALLOC_ERR_TIMEOUT = 4    /* a barrier of the last call gave up */
};
int mom6b_btstep_noalloc(const double *eta_in, const double *ubt_in,
                         const double *vbt_in, double *u_av, double *v_av,
                         double *eta_av, const double *Datu, const double *Datv,
                         const double *gtot_E, const double *gtot_W,
                         const double *gtot_N, const double *gtot_S,
                         const double *f_4_u, const double *f_4_v,
                         const double *bt_rem_u, const double *bt_rem_v,
                         const double *IareaT, const double *IdxCu,
                         const double *IdyCv, int n1, int n2, int is, int ie,
                         int js, int je, int nstep, double dtbt, double bebt,
                         double dgeo_de, int first_direction,
                         int extended_ranges, void *stream);
int mom6b_btstep_noalloc_status(void *stream);
int mom6b_btstep_noalloc_set_wait(long long cycles, int stall_test);

/* ---- barotropic deferral of the reference ABI -----------------------------
 * No counterpart in the reference.  The launch_bt_* entry points of
 * mom6_cuda_c.h defer the substep kernels of one btstep_cuda_c call
 * (launch_bt_init_kernel runs and opens a record; the substep calls that
 * continue the wrapper's fixed sequence are recorded; launch_bt_copy_output_kernel
 * runs the whole loop as one persistent launch on the library's static
 * scratch, bit-identical to the substep kernels).  Any call that breaks the
 * sequence, any other launch_* entry point and any cuda_*_c helper first
 * replay the record call by call.  The substep kernels' own arrays of the
 * control structure are not written by a deferred loop (the wrapper reads
 * only the copy's outputs).  on = 0 runs every launch_bt_* call as it comes
 * (on by default).  The setting is process-wide; a record belongs to the
 * host thread that opened it. */
int mom6b_abi_set_deferral(int on);

/* Device address of one of the model's 2-D metric arrays by name ("IareaT",
 * "IdxCu", "IdyCv", "Datu", "Datv", "gtot_E", "gtot_W", "gtot_N", "gtot_S",
 * "f_4_u", "f_4_v", "bt_rem_u", "bt_rem_v"). */
int mom6b_metric_device_ptr(mom6b_model *m, const char *name, void **dptr);

/* ---- the reference's CUDA C host side, mirrored ---------------------------
 * No counterpart as a C function in the reference: rk2_cuda_c_driver.F90 and
 * the Fortran wrappers of src/cuda_c (*_cuda_c.F90) are restated in C++ so
 * that a whole split RK2 iteration can be driven through the launch_* ABI of
 * mom6_cuda_c.h.  The state is the driver's analytic initial state
 * (rk2_cuda_c_driver.F90:663-700) on init_ocean_grid's grid; each call of
 * mom6b_cudac_step runs rk2_cuda_c_driver.F90:263-481 once per step, with the
 * wrappers' launch order, arguments and per-phase device synchronisation.
 * kernel_lib NULL drives this library's own launch_* entry points (the
 * drop-in path); otherwise the path of a shared object exporting the same
 * symbols is opened and its entry points are driven instead.  Fields are read
 * with the MOM6B_F_* ids (u, v, h, h0, uh, vh, up, vp, eta, ubt, vbt, ubt_av,
 * vbt_av, eta_av, the BT_cont arrays, taux_bot = the last bottom stress,
 * taux, tauy). */
typedef struct mom6b_cudac mom6b_cudac;
int mom6b_cudac_create(int ni, int nj, int nk, int bt_nsteps, double dt,
                       const char *kernel_lib, mom6b_cudac **out);
/* The same mirror on the grid, forcing and initial state a model of *cfg
 * would build (cfg->init_mode REF or CFG, seed, dt, Kh, vertical viscosity);
 * the reference's host side has no halo fill, so cfg->bc_fill, precision and
 * the model-only options are ignored. */
int mom6b_cudac_create_cfg(const mom6b_config *cfg, const char *kernel_lib,
                           mom6b_cudac **out);
int mom6b_cudac_step(mom6b_cudac *m, int nsteps);
size_t mom6b_cudac_field_size(const mom6b_cudac *m, int field);
int mom6b_cudac_get_field(mom6b_cudac *m, int field, double *host, size_t count);
int mom6b_cudac_destroy(mom6b_cudac *m);

/* ---- ensemble: many domains in one launch per phase -----------------------
 * No counterpart in the reference (its drivers advance one domain).  n
 * independent domains of any sizes (cfgs[d], each with precision
 * MOM6B_MIXED, all on one device, nk <= 256) are built exactly as
 * mom6b_create builds them and advanced together: one RK2 step is fourteen
 * launches whatever n is (ten without halo fills), each covering all domains
 * (the barotropic loops of all domains share one cooperative persistent
 * launch per call).  Each domain gets the same arithmetic as a mixed-form
 * model of its own.  The launch shapes come from mom6b_ensemble_autotune,
 * which times the candidate shapes of every phase on the ensemble's domains
 * (their state is saved before and restored after) and keeps the fastest;
 * out_ms (5 doubles, optional) receives the best tendency, vertvisc, PPM,
 * faces and barotropic launch times.  Tuning as 7 ints: tendency tile (0: 32x8,
 * 1: 32x4, 2: 64x4, 3: 32x16), tendency layers per CTA (1..16), vertvisc
 * threads per CTA (64, 128, 256), vertvisc prefetch depth (2, 4), PPM threads
 * per CTA (128, 256), threads per continuity face CTA (64, 128, 256),
 * barotropic tile edge (32, 48, 64).  mom6b_ensemble_member returns domain d
 * as a model (owned by the ensemble; read it after
 * mom6b_ensemble_synchronize, or with mom6b_ensemble_get_field). */
typedef struct mom6b_ensemble mom6b_ensemble;
int mom6b_ensemble_create(int n, const mom6b_config *cfgs, mom6b_ensemble **out);
int mom6b_ensemble_destroy(mom6b_ensemble *e);
int mom6b_ensemble_size(const mom6b_ensemble *e);
int mom6b_ensemble_step(mom6b_ensemble *e, int nsteps);
int mom6b_ensemble_synchronize(mom6b_ensemble *e);
int mom6b_ensemble_stream(mom6b_ensemble *e, void **stream);
int64_t mom6b_ensemble_launch_count(const mom6b_ensemble *e);
mom6b_model *mom6b_ensemble_member(mom6b_ensemble *e, int d);
int mom6b_ensemble_get_field(mom6b_ensemble *e, int d, int field, double *host,
                             size_t count);
int mom6b_ensemble_autotune(mom6b_ensemble *e, int reps, double *out_ms);
int mom6b_ensemble_get_tuning(const mom6b_ensemble *e, int *out7);
int mom6b_ensemble_set_tuning(mom6b_ensemble *e, const int *in7);

/* ---- learned barotropic surrogate -----------------------------------------
 * No counterpart in the reference.  A 175-256-256-2 MLP (GELU, bf16 weights and
 * activations on the tensor cores, fp32 accumulation) maps the 5 x 5 stencil
 * of 7 channels (eta, ubt, vbt, barotropic forcing u and v (zero: btstep has
 * no forcing), depth, f) of a cell, each divided by its channel std, to the
 * substep-averaged transports of its east and north faces; eta is then
 * advanced in FP64 from their divergence (volume conserved to rounding), and
 * the averaged velocities are transport / Datu, / Datv.
 *
 * mom6b_surrogate_train trains the model's network on the GPU: nstates
 * seeded barotropic initial states (Gaussian eta bumps of seeded amplitude,
 * centre and radius, ubt = vbt = 0), nsteps RK2 steps of the plain btstep
 * each; every barotropic call gives one batch of `batch` sampled columns and
 * one Adam step (lr).  The channel and target stds come from the first 10
 * steps of the first state.  stats4 (optional): mean loss of the first 10 and
 * of the last 100 batches, batches, seconds.
 *
 * mom6b_surrogate_enable(on = 1) makes mom6b_step use the network instead of
 * btstep; every shadow_every steps (0: never) the plain btstep runs from the
 * same state as the check: when the relative L2 difference of the two etas over
 * the compute domain exceeds threshold, the plain results are kept and the
 * model uses the plain btstep from then on (mom6b_surrogate_enable again
 * re-arms it).  status10: enabled, fallen back, steps, shadow checks,
 * fallbacks, last and largest shadow error, first and last training loss,
 * training batches.  The parameters (mom6b_surrogate_param_count floats: the
 * network's, then the 7 feature stds and the 2 target stds) move a trained
 * network between models. */
int mom6b_surrogate_train(mom6b_model *m, int nstates, int nsteps, int batch,
                          double lr, uint64_t seed, double *stats4);
/* Transport error on state k of the seeded family (pick a k the training did
 * not use): out3 = relative L2 error of the network's averaged transports
 * against the plain btstep's over nsteps RK2 barotropic chains, the same for
 * the zero-transport prediction, calls. */
int mom6b_surrogate_eval(mom6b_model *m, uint64_t seed, int k, int nsteps, double *out3);
int mom6b_surrogate_enable(mom6b_model *m, int on, int shadow_every, double threshold);
int mom6b_surrogate_status(const mom6b_model *m, double *status10);
size_t mom6b_surrogate_param_count(void);
int mom6b_surrogate_get_params(const mom6b_model *m, float *host, size_t n);
int mom6b_surrogate_set_params(mom6b_model *m, const float *host, size_t n);

/* The network alone, for checks against a CPU restatement: batches of B rows
 * (128 <= B <= the batch it was created with, B a multiple of 8) of 175 fp32
 * features (rounded to bf16 on upload) and 2 fp32 targets.
 * mom6b_mlp_gradients: forward, loss = sum (out - y)^2 / (2 B), backward; the
 * gradient of every parameter (mom6b_mlp_param_count floats, layout W1
 * [256][176] (column 175 is padding), b1, W2 [256][256], b2, W3 [2][256], b3).
 * mom6b_mlp_train: nsteps Adam steps (0.9, 0.999, 1e-8) on one batch.
 * mom6b_mlp_predict: outputs of n rows. */
typedef struct mom6b_mlp mom6b_mlp;
int mom6b_mlp_param_count(void);
int mom6b_mlp_create(int batch, uint64_t seed, mom6b_mlp **out);
int mom6b_mlp_destroy(mom6b_mlp *p);
int mom6b_mlp_get_params(mom6b_mlp *p, float *host, size_t n);
int mom6b_mlp_set_params(mom6b_mlp *p, const float *host, size_t n);
int mom6b_mlp_gradients(mom6b_mlp *p, const float *X, const float *Y, int B,
                        float *grads, float *loss, float *out);
int mom6b_mlp_train(mom6b_mlp *p, const float *X, const float *Y, int B, float lr,
                    int nsteps, float *losses);
int mom6b_mlp_predict(mom6b_mlp *p, const float *X, int n, float *out);

const char *mom6b_last_error(void);
const char *mom6b_version(void);

#ifdef __cplusplus
}
#endif
#endif
