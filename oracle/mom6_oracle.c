/*
 * mom6_oracle.c -- CPU restatement of the MOM6 mini-app split RK2 step.
 *
 * TEST INFRASTRUCTURE ONLY (see mom6_oracle.h).  Each routine names the
 * reference routine it restates, file:line, paths relative to the reference
 * project root.  Loop ranges, evaluation order and the default-real (FP32)
 * literals and locals of the serial Fortran are kept exactly, because the
 * B200 kernels are checked against this file bit for bit.
 *
 * Conventions: 1-based Fortran indices everywhere; A2/A3 map (i,j[,k]) into
 * the column-major arrays.  "F32(x)" marks a Fortran default-real literal
 * (real(4)) that is promoted to double in a mixed expression.
 */
#include "mom6_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define F32(x) ((double)(x##f))

/* Row-parallel loops.  Built with -fopenmp (liboracle_omp.so) the marked
 * loops, whose iterations write disjoint rows (or layers) and read only
 * arrays no iteration writes, run on all host threads; the results equal the
 * single-threaded build's bit for bit.  Without OpenMP the marks vanish. */
#ifdef _OPENMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#define OMP_COLS _Pragma("omp for schedule(static)")
#else
#define OMP_FOR
#define OMP_COLS
#endif

/* Physical constants, mom6_types.F90:80-85. */
static const double G_EARTH = 9.80;
static const double RHO_0 = 1035.0;
static const double OMEGA = 7.2921e-5;
static const double PI_REF = 3.14159265358979323846;
static const double EARTH_RADIUS = 6.371e6;

struct oracle_model {
    oracle_config cfg;
    int ni, nj, nk, n1, n2;
    int isd, ied, jsd, jed, is, ie, js, je;
    double dt, dx;
    int nstep;

    /* grid metrics, mom6_types.F90:19-58 */
    double *IareaT, *areaT, *dxT, *dyT, *IdxT, *IdyT, *dxCu, *dyCu, *dy_Cu,
        *IdxCu, *IdyCu, *dxCv, *dyCv, *IdxCv, *IdyCv, *IareaBu, *areaBu,
        *CoriolisBu, *IareaCu, *IareaCv, *dxBu, *dyBu, *IdxBu, *IdyBu, *bathyT,
        *mask2dT, *mask2dBu, *mask2dCu, *mask2dCv;

    /* Coriolis scheme (coriolis_init's scheme argument, mom6_coriolis_serial.F90:47-56):
     * 1 SADOURNY75_ENERGY (the driver's), 2 ARAKAWA_HSU90, 3 ARAKAWA_LAMB81, and the
     * scheme's coefficient arrays a, b, c, d (:29-39) */
    int cor_scheme;
    double *co_a, *co_b, *co_c, *co_d;

    /* the vertical-viscosity remnant fed to continuity (oracle_set_remnant):
     * visc_rem_v beside the driver's visc_rem_u */
    int remnant;
    double *visc_rem_v;

    /* meridional continuity (oracle_set_merid): its outputs, the
     * intermediate thickness and the transposed problem's arrays */
    int merid;
    double *hz, *BT_h_v, *FA_v_S0, *FA_v_SS, *FA_v_N0, *FA_v_NN, *vBT_SS, *vBT_NN, *dv_cor;
    double *mt[22];

    /* driver diagnostics (diag_mode = 1, rk2_serial_driver.F90:149-170):
     * diag_work is mom6_diag's persistent work_2d (mom6_diag.F90:61, zero at
     * diag_init); the posted fields are kept for the tests */
    int diag_on;
    double *diag_work, *diag_usum, *diag_vsum, *diag_KE, *diag_mass;

    /* driver state, rk2_serial_driver.F90:59-76 (zero-initialised) */
    double *u, *v, *h, *h0, *htmp, *uh, *vh, *CAu, *CAv, *up, *vp, *diffu,
        *diffv;
    double *eta, *ubt, *vbt, *ubt_av, *vbt_av, *eta_av;
    double *taux, *tauy, *Ray_u, *Ray_v;

    /* continuity, mom6_continuity_serial.F90:53-78 and BT_cont */
    double *c_uhbt, *u_cor, *du_cor, *por_face_areaU, *visc_rem_u;
    double *hW, *hE; /* h_W, h_E locals of continuity_PPM */
    double *FA_u_W0, *FA_u_WW, *FA_u_E0, *FA_u_EE, *uBT_WW, *uBT_EE, *BT_h_u;

    /* Coriolis CS work arrays, mom6_coriolis_serial.F90:28-39 */
    double *co_dvdx, *co_dudy, *co_rel_vort, *co_abs_vort, *co_q, *co_Ih_q,
        *co_hArea_u, *co_hArea_v, *co_Area_q, *co_KE;

    /* hor_visc CS, mom6_hor_visc_serial.F90:32-152 (active subset) */
    double *hv_Kh_bg_xx, *hv_Kh_bg_xy, *hv_dx2h, *hv_dy2h, *hv_dx2q, *hv_dy2q,
        *hv_DX_dyT, *hv_DY_dxT, *hv_DX_dyBu, *hv_DY_dxBu, *hv_red_xx,
        *hv_red_xy, *hv_dudx, *hv_dvdy, *hv_dvdx, *hv_dudy, *hv_sh_xx,
        *hv_sh_xy, *hv_str_xx, *hv_str_xy, *hv_h_u, *hv_h_v, *hv_hq, *hv_Kh;
    double hv_Kh_bg_min, hv_h_neglect;
    /* the scheme branches (:37-57, :71-152): flags, background / maximum
     * viscosities and the Smagorinsky / Leith constants (xx at h-points, xy
     * at q-points), biharmonic metrics and the persistent work arrays */
    int hv_lap, hv_bih, hv_smag_kh, hv_smag_ah, hv_leith_kh, hv_leith_ah, hv_no_slip,
        hv_bound_kh, hv_bound_ah, hv_bb_kh, hv_bb_ah, hv_mod_leith;
    double *hv_Ah_bg_xx, *hv_Ah_bg_xy, *hv_Kh_Max_xx, *hv_Kh_Max_xy, *hv_Ah_Max_xx,
        *hv_Ah_Max_xy, *hv_L2c_xx, *hv_L2c_xy, *hv_Bc_xx, *hv_Bc_xy, *hv_L3c_xx,
        *hv_L3c_xy, *hv_B6c_xx, *hv_B6c_xy, *hv_Idx2dyCu, *hv_Idxdy2u, *hv_Idx2dyCv,
        *hv_Idxdy2v, *hv_Ah, *hv_Shear_mag, *hv_Del2u, *hv_Del2v, *hv_hrat_min,
        *hv_vbr, *hv_vort, *hv_vort_dx, *hv_vort_dy, *hv_gvm_h, *hv_gvm_q, *hv_vvm,
        *hv_Del2vort_q, *hv_div, *hv_div_dx, *hv_div_dy, *hv_gdm_h, *hv_bhstr_xx,
        *hv_bhstr_xy;

    /* vert_visc CS, mom6_vert_visc_serial.F90:27-55 */
    double *vv_a_u, *vv_a_v, *vv_h_u, *vv_h_v, *vv_taux_bot, *vv_tauy_bot;
    double Angstrom_H;

    /* barotropic CS, mom6_barotropic_serial.F90:20-58 */
    double bt_dtbt, bt_bebt, bt_dgeo_de;
    double *bt_eta, *bt_eta_pred, *bt_ubt, *bt_vbt, *bt_ubt_prev, *bt_vbt_prev,
        *bt_uhbt, *bt_vhbt, *bt_PFu, *bt_PFv, *bt_Cor_u, *bt_Cor_v, *bt_Datu,
        *bt_Datv, *bt_gtot_E, *bt_gtot_W, *bt_gtot_N, *bt_gtot_S, *bt_f_4_u,
        *bt_f_4_v, *bt_rem_u, *bt_rem_v, *bt_ubt_av, *bt_vbt_av;
    int first_direction;
    int bt_extended; /* 1: uhbt/vhbt and averages on the extended ranges */
    /* decomposed runs: global sizes, offsets, the cut sides (0 / 1) and the
     * halo exchange */
    int gni, gnj, ioff, joff, cw, ce, cs, cn;
    oracle_exchange_fn xfn;
    void *xctx;
};

/* ------------------------------------------------------------------------ */
/* indexing                                                                 */
/* ------------------------------------------------------------------------ */
#define N1 (m->n1)
#define N2 (m->n2)
#define A2(a, i, j) (a)[((size_t)(j)-1) * (size_t)N1 + ((size_t)(i)-1)]
#define A3(a, i, j, k)                                                         \
    (a)[(((size_t)(k)-1) * (size_t)N2 + ((size_t)(j)-1)) * (size_t)N1 +         \
        ((size_t)(i)-1)]
/* f_4_u(c,i,j): leading dimension 4 (mom6_barotropic_serial.F90:97-98) */
#define F4(a, c, i, j)                                                         \
    (a)[((((size_t)(j)-1) * (size_t)N1 + ((size_t)(i)-1)) * 4) + ((size_t)(c)-1)]

static double fmax_(double a, double b) { return a > b ? a : b; }
static double fmin_(double a, double b) { return a < b ? a : b; }
/* Fortran MAX/MIN of non-NaN values; the order of comparison does not
 * change the result. */
#define MAX(a, b) fmax_((a), (b))
#define MIN(a, b) fmin_((a), (b))

static double *zalloc(size_t n) {
    double *p = (double *)calloc(n ? n : 1, sizeof(double));
    return p;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) and a Box-Muller normal */
/* ------------------------------------------------------------------------ */
static void philox4x32_10(uint32_t ctr[4], uint32_t key[2]) {
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        uint32_t n3 = lo0;
        ctr[0] = n0; ctr[1] = n1; ctr[2] = n2; ctr[3] = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

int oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

double oracle_normal(uint64_t seed, uint32_t stream, uint64_t index) {
    uint32_t ctr[4] = {(uint32_t)index, (uint32_t)(index >> 32), stream, 0u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    philox4x32_10(ctr, key);
    uint64_t a = (((uint64_t)ctr[0] << 32) | ctr[1]) >> 11;
    uint64_t b = (((uint64_t)ctr[2] << 32) | ctr[3]) >> 11;
    double u1 = (double)a * 0x1.0p-53 + 0x1.0p-54; /* (0,1) */
    double u2 = (double)b * 0x1.0p-53;
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

/* ------------------------------------------------------------------------ */
/* configuration and grid                                                   */
/* ------------------------------------------------------------------------ */
void oracle_config_default(oracle_config *c, int init_mode) {
    memset(c, 0, sizeof(*c));
    c->ni = 180; c->nj = 180; c->nk = 75;
    c->bt_nsteps = 30;
    c->init_mode = init_mode;
    c->seed = 0;
    c->dx_km = 10.0;
    c->lat_deg = 45.0;
    c->Kv = 1.0e-4; c->Kv_ml = 1.0e-2; c->Kv_extra_bbl = 1.0e-2;
    c->Hmix = 50.0; c->Hbbl = 10.0;
    if (init_mode == OR_INIT_REF) {
        /* rk2_serial_driver.F90:91-93,141-143 */
        c->dt = 300.0; c->Kh = 100.0; c->bc_fill = 0;
    } else {
        /* seeded beta-plane configuration */
        c->dt = 600.0; c->Kh = 1.0e3; c->bc_fill = 1;
    }
}

/* init_ocean_grid, mom6_types.F90:130-258 (REF); the CFG mode only changes
 * the Coriolis profile to f = 1e-4 + 2e-11 (y - Ly/2). */
static void init_grid(oracle_model *m) {
    const oracle_config *c = &m->cfg;
    size_t n = (size_t)N1 * N2;
    double **arrs[] = {&m->IareaT, &m->areaT, &m->dxT, &m->dyT, &m->IdxT,
                       &m->IdyT, &m->dxCu, &m->dyCu, &m->dy_Cu, &m->IdxCu,
                       &m->IdyCu, &m->dxCv, &m->dyCv, &m->IdxCv, &m->IdyCv,
                       &m->IareaBu, &m->areaBu, &m->CoriolisBu, &m->IareaCu,
                       &m->IareaCv, &m->dxBu, &m->dyBu, &m->IdxBu, &m->IdyBu,
                       &m->bathyT, &m->mask2dT, &m->mask2dBu, &m->mask2dCu,
                       &m->mask2dCv};
    for (size_t a = 0; a < sizeof(arrs) / sizeof(arrs[0]); ++a)
        *arrs[a] = zalloc(n);

    double dx_m = c->dx_km * 1000.0;
    m->dx = dx_m;
    double f0 = 2.0 * OMEGA * sin(c->lat_deg * PI_REF / 180.0);
    double beta = 2.0 * OMEGA * cos(c->lat_deg * PI_REF / 180.0) / EARTH_RADIUS;
    const int gie = m->gni - 1, gje = m->gnj - 1;   /* the global ie, je */
    double Ly = (double)(gje - m->js + 1) * dx_m;
    (void)gie;
    for (int j = m->jsd; j <= m->jed; ++j)
        for (int i = m->isd; i <= m->ied; ++i) {
            A2(m->areaT, i, j) = dx_m * dx_m;
            A2(m->IareaT, i, j) = 1.0 / (dx_m * dx_m);
            A2(m->dxT, i, j) = dx_m;
            A2(m->dyT, i, j) = dx_m;
            A2(m->IdxT, i, j) = 1.0 / dx_m;
            A2(m->IdyT, i, j) = 1.0 / dx_m;
            A2(m->dxCu, i, j) = dx_m;
            A2(m->dyCu, i, j) = dx_m;
            A2(m->dy_Cu, i, j) = dx_m;
            A2(m->IdxCu, i, j) = 1.0 / dx_m;
            A2(m->IdyCu, i, j) = 1.0 / dx_m;
            A2(m->dxCv, i, j) = dx_m;
            A2(m->dyCv, i, j) = dx_m;
            A2(m->IdxCv, i, j) = 1.0 / dx_m;
            A2(m->IdyCv, i, j) = 1.0 / dx_m;
            A2(m->areaBu, i, j) = dx_m * dx_m;
            A2(m->IareaBu, i, j) = 1.0 / (dx_m * dx_m);
            A2(m->IareaCu, i, j) = 1.0 / (dx_m * dx_m);
            A2(m->IareaCv, i, j) = 1.0 / (dx_m * dx_m);
            A2(m->dxBu, i, j) = dx_m;
            A2(m->dyBu, i, j) = dx_m;
            A2(m->IdxBu, i, j) = 1.0 / dx_m;
            A2(m->IdyBu, i, j) = 1.0 / dx_m;
            A2(m->mask2dT, i, j) = 1.0;
            A2(m->mask2dBu, i, j) = 1.0;
            A2(m->mask2dCu, i, j) = 1.0;
            A2(m->mask2dCv, i, j) = 1.0;
            A2(m->bathyT, i, j) = 4000.0;
            if (c->init_mode == OR_INIT_REF) {
                A2(m->CoriolisBu, i, j) =
                    f0 + beta * ((double)(j + m->joff - 1 - m->gnj / 2) - 0.5) * dx_m;
            } else {
                double yq = (double)(j + m->joff - m->js + 1) * dx_m;
                A2(m->CoriolisBu, i, j) = 1.0e-4 + 2.0e-11 * (yq - 0.5 * Ly);
            }
        }
    m->first_direction = 0;
}

/* ------------------------------------------------------------------------ */
/* module init routines                                                     */
/* ------------------------------------------------------------------------ */
static void alloc_all(oracle_model *m) {
    size_t n2d = (size_t)N1 * N2, n3d = n2d * (size_t)m->nk;
    size_t n3p = n2d * (size_t)(m->nk + 1);
    m->u = zalloc(n3d); m->v = zalloc(n3d); m->h = zalloc(n3d);
    m->h0 = zalloc(n3d); m->htmp = zalloc(n3d); m->uh = zalloc(n3d);
    m->vh = zalloc(n3d); m->CAu = zalloc(n3d); m->CAv = zalloc(n3d);
    m->up = zalloc(n3d); m->vp = zalloc(n3d); m->diffu = zalloc(n3d);
    m->diffv = zalloc(n3d);
    m->eta = zalloc(n2d); m->ubt = zalloc(n2d); m->vbt = zalloc(n2d);
    m->ubt_av = zalloc(n2d); m->vbt_av = zalloc(n2d); m->eta_av = zalloc(n2d);
    m->taux = zalloc(n2d); m->tauy = zalloc(n2d);
    m->Ray_u = zalloc(n3d); m->Ray_v = zalloc(n3d);

    /* continuity_init, mom6_continuity_serial.F90:53-78 */
    m->c_uhbt = zalloc(n2d); m->u_cor = zalloc(n3d); m->du_cor = zalloc(n2d);
    m->por_face_areaU = zalloc(n3d); m->visc_rem_u = zalloc(n3d);
    for (size_t q = 0; q < n3d; ++q) {
        m->por_face_areaU[q] = 1.0;
        m->visc_rem_u[q] = 1.0;
    }
    m->hW = zalloc(n3d); m->hE = zalloc(n3d);
    /* alloc_BT_cont_type, mom6_types.F90:334-367 */
    m->FA_u_W0 = zalloc(n2d); m->FA_u_WW = zalloc(n2d);
    m->FA_u_E0 = zalloc(n2d); m->FA_u_EE = zalloc(n2d);
    m->uBT_WW = zalloc(n2d); m->uBT_EE = zalloc(n2d); m->BT_h_u = zalloc(n3d);

    /* coriolis_init, mom6_coriolis_serial.F90:48-84 */
    m->co_dvdx = zalloc(n2d); m->co_dudy = zalloc(n2d);
    m->co_rel_vort = zalloc(n2d); m->co_abs_vort = zalloc(n2d);
    m->co_q = zalloc(n2d); m->co_Ih_q = zalloc(n2d);
    m->co_hArea_u = zalloc(n2d); m->co_hArea_v = zalloc(n2d);
    m->co_Area_q = zalloc(n2d); m->co_KE = zalloc(n2d);
    m->co_a = zalloc(n2d); m->co_b = zalloc(n2d); m->co_c = zalloc(n2d); m->co_d = zalloc(n2d);
    m->cor_scheme = 1;
    for (int j = m->jsd; j <= m->jed - 1; ++j)
        for (int i = m->isd; i <= m->ied - 1; ++i)
            A2(m->co_Area_q, i, j) = (A2(m->areaT, i, j) + A2(m->areaT, i + 1, j + 1)) +
                                     (A2(m->areaT, i + 1, j) + A2(m->areaT, i, j + 1));

    /* hor_visc_init, mom6_hor_visc_serial.F90:160-286 (Laplacian subset) */
    double **hv[] = {&m->hv_Kh_bg_xx, &m->hv_Kh_bg_xy, &m->hv_dx2h, &m->hv_dy2h,
                     &m->hv_dx2q, &m->hv_dy2q, &m->hv_DX_dyT, &m->hv_DY_dxT,
                     &m->hv_DX_dyBu, &m->hv_DY_dxBu, &m->hv_red_xx,
                     &m->hv_red_xy, &m->hv_dudx, &m->hv_dvdy, &m->hv_dvdx,
                     &m->hv_dudy, &m->hv_sh_xx, &m->hv_sh_xy, &m->hv_str_xx,
                     &m->hv_str_xy, &m->hv_h_u, &m->hv_h_v, &m->hv_hq, &m->hv_Kh,
                     &m->hv_Ah_bg_xx, &m->hv_Ah_bg_xy, &m->hv_Kh_Max_xx, &m->hv_Kh_Max_xy,
                     &m->hv_Ah_Max_xx, &m->hv_Ah_Max_xy, &m->hv_L2c_xx, &m->hv_L2c_xy,
                     &m->hv_Bc_xx, &m->hv_Bc_xy, &m->hv_L3c_xx, &m->hv_L3c_xy,
                     &m->hv_B6c_xx, &m->hv_B6c_xy, &m->hv_Idx2dyCu, &m->hv_Idxdy2u,
                     &m->hv_Idx2dyCv, &m->hv_Idxdy2v, &m->hv_Ah, &m->hv_Shear_mag,
                     &m->hv_Del2u, &m->hv_Del2v, &m->hv_hrat_min, &m->hv_vbr, &m->hv_vort,
                     &m->hv_vort_dx, &m->hv_vort_dy, &m->hv_gvm_h, &m->hv_gvm_q, &m->hv_vvm,
                     &m->hv_Del2vort_q, &m->hv_div, &m->hv_div_dx, &m->hv_div_dy,
                     &m->hv_gdm_h, &m->hv_bhstr_xx, &m->hv_bhstr_xy};
    for (size_t a = 0; a < sizeof(hv) / sizeof(hv[0]); ++a) *hv[a] = zalloc(n2d);
    m->hv_Kh_bg_min = 0.0;
    m->Angstrom_H = 1.0e-10; /* init_verticalGrid, mom6_types.F90:318-331 */
    m->hv_h_neglect = MAX(m->Angstrom_H, 1.0e-3);
    for (int j = m->jsd; j <= m->jed; ++j)
        for (int i = m->isd; i <= m->ied; ++i) {
            A2(m->hv_dx2h, i, j) = A2(m->dxT, i, j) * A2(m->dxT, i, j);
            A2(m->hv_dy2h, i, j) = A2(m->dyT, i, j) * A2(m->dyT, i, j);
            A2(m->hv_dx2q, i, j) = A2(m->dxBu, i, j) * A2(m->dxBu, i, j);
            A2(m->hv_dy2q, i, j) = A2(m->dyBu, i, j) * A2(m->dyBu, i, j);
            A2(m->hv_DX_dyT, i, j) = A2(m->dxT, i, j) * A2(m->IdyT, i, j);
            A2(m->hv_DY_dxT, i, j) = A2(m->dyT, i, j) * A2(m->IdxT, i, j);
            A2(m->hv_DX_dyBu, i, j) = A2(m->dxBu, i, j) * A2(m->IdyBu, i, j);
            A2(m->hv_DY_dxBu, i, j) = A2(m->dyBu, i, j) * A2(m->IdxBu, i, j);
            A2(m->hv_red_xx, i, j) = 1.0;
            A2(m->hv_red_xy, i, j) = 1.0;
            A2(m->hv_Kh_bg_xx, i, j) = m->cfg.Kh;
            A2(m->hv_Kh_bg_xy, i, j) = m->cfg.Kh;
        }
    {
        oracle_hor_visc_opts o = {1, 0, 0, 0, 0, 0, 0, 1.0e10};
        oracle_set_hor_visc(m, &o);
    }

    /* vert_visc_init, mom6_vert_visc_serial.F90:60-112 */
    m->vv_a_u = zalloc(n3p); m->vv_a_v = zalloc(n3p);
    m->vv_h_u = zalloc(n3d); m->vv_h_v = zalloc(n3d);
    m->vv_taux_bot = zalloc(n2d); m->vv_tauy_bot = zalloc(n2d);

    /* barotropic_init, mom6_barotropic_serial.F90:63-137 */
    m->bt_dtbt = m->dt / (double)m->nstep;
    m->bt_bebt = 0.2;
    m->bt_dgeo_de = 1.0;
    double depth = 4000.0;
    double **bt[] = {&m->bt_eta, &m->bt_eta_pred, &m->bt_ubt, &m->bt_vbt,
                     &m->bt_ubt_prev, &m->bt_vbt_prev, &m->bt_uhbt, &m->bt_vhbt,
                     &m->bt_PFu, &m->bt_PFv, &m->bt_Cor_u, &m->bt_Cor_v,
                     &m->bt_Datu, &m->bt_Datv, &m->bt_gtot_E, &m->bt_gtot_W,
                     &m->bt_gtot_N, &m->bt_gtot_S, &m->bt_rem_u, &m->bt_rem_v,
                     &m->bt_ubt_av, &m->bt_vbt_av};
    for (size_t a = 0; a < sizeof(bt) / sizeof(bt[0]); ++a) *bt[a] = zalloc(n2d);
    m->bt_f_4_u = zalloc(4 * n2d);
    m->bt_f_4_v = zalloc(4 * n2d);
    for (int j = m->jsd; j <= m->jed; ++j)
        for (int i = m->isd; i <= m->ied; ++i) {
            A2(m->bt_Datu, i, j) = depth * A2(m->dyCu, i, j);
            A2(m->bt_Datv, i, j) = depth * A2(m->dxCv, i, j);
            A2(m->bt_gtot_E, i, j) = G_EARTH;
            A2(m->bt_gtot_W, i, j) = G_EARTH;
            A2(m->bt_gtot_N, i, j) = G_EARTH;
            A2(m->bt_gtot_S, i, j) = G_EARTH;
            A2(m->bt_rem_u, i, j) = 0.999;
            A2(m->bt_rem_v, i, j) = 0.999;
            double f0 = A2(m->CoriolisBu, i, j);
            for (int c = 1; c <= 4; ++c) {
                F4(m->bt_f_4_u, c, i, j) = 0.25 * f0;
                F4(m->bt_f_4_v, c, i, j) = 0.25 * f0;
            }
        }
}

/* initialize_state + initialize_forces_visc, rk2_serial_driver.F90:466-542
 * (REF), or the seeded construction (CFG). */
static void init_state(oracle_model *m) {
    const oracle_config *c = &m->cfg;
    int nk = m->nk;
    /* the global point of each local one (init_ocean_grid_mpi,
     * mom6_mpi_domain.F90:144-258: positions by global index) */
    const int io = m->ioff, jo = m->joff, gni = m->gni, gnj = m->gnj;
    for (int j = m->jsd; j <= m->jed; ++j)
        for (int i = m->isd; i <= m->ied; ++i) {
            A2(m->taux, i, j) = 0.1 * sin((double)(j + jo - 1) / (double)gnj * 3.14159);
            A2(m->tauy, i, j) = 0.0;
        }
    for (int j = m->jsd; j <= m->jed; ++j)
        for (int i = m->isd; i <= m->ied; ++i) {
            A3(m->Ray_u, i, j, nk) = 1.0e-4;
            A3(m->Ray_v, i, j, nk) = 1.0e-4;
        }
    if (c->init_mode == OR_INIT_REF) {
        double total_depth = 4000.0;
        for (int k = 1; k <= nk; ++k)
            for (int j = m->jsd; j <= m->jed; ++j)
                for (int i = m->isd; i <= m->ied; ++i) {
                    A3(m->h0, i, j, k) =
                        total_depth / (double)nk +
                        10.0 * sin((double)(i + io - 1) / (double)gni * 3.14159) *
                            cos((double)(j + jo - 1) / (double)gnj * 3.14159) *
                            exp(-(double)k / 20.0);
                    A3(m->h, i, j, k) = A3(m->h0, i, j, k);
                    A3(m->u, i, j, k) =
                        0.1 * sin((double)(j + jo - 1) / (double)gnj * 3.14159 * 2.0) *
                        exp(-(double)k / 30.0);
                    A3(m->v, i, j, k) =
                        0.1 * cos((double)(i + io - 1) / (double)gni * 3.14159 * 2.0) *
                        exp(-(double)k / 30.0);
                }
        for (int j = m->jsd; j <= m->jed; ++j)
            for (int i = m->isd; i <= m->ied; ++i) {
                A2(m->eta, i, j) =
                    0.5 * sin((double)(i + io - 1) / (double)gni * 3.14159 * 2.0) *
                    cos((double)(j + jo - 1) / (double)gnj * 3.14159 * 2.0);
                A2(m->ubt, i, j) = 0.05 * sin((double)(j + jo - 1) / (double)gnj * 3.14159);
                A2(m->vbt, i, j) = 0.05 * cos((double)(i + io - 1) / (double)gni * 3.14159);
            }
    } else {
        double hbar = 4000.0 / (double)nk;
        for (int k = 1; k <= nk; ++k)
            for (int j = m->jsd; j <= m->jed; ++j)
                for (int i = m->isd; i <= m->ied; ++i) {
                    uint64_t idx = ((uint64_t)(k - 1) * (uint64_t)(gnj + 2) +
                                    (uint64_t)(j + jo - 1)) * (uint64_t)(gni + 2) +
                                   (uint64_t)(i + io - 1);
                    double hv = hbar * (1.0 + 0.01 * oracle_normal(c->seed, 1u, idx));
                    if (hv < 0.01 * hbar) hv = 0.01 * hbar;
                    A3(m->h0, i, j, k) = hv;
                    A3(m->h, i, j, k) = hv;
                    A3(m->u, i, j, k) = 0.05 * oracle_normal(c->seed, 2u, idx);
                    A3(m->v, i, j, k) = 0.05 * oracle_normal(c->seed, 3u, idx);
                }
        double dx = m->dx;
        double Lx = (double)((gni - 1) - m->is + 1) * dx;
        double Ly = (double)((gnj - 1) - m->js + 1) * dx;
        double R = 200.0e3;
        for (int j = m->jsd; j <= m->jed; ++j)
            for (int i = m->isd; i <= m->ied; ++i) {
                double x = ((double)(i + io - m->is) + 0.5) * dx - 0.5 * Lx;
                double y = ((double)(j + jo - m->js) + 0.5) * dx - 0.5 * Ly;
                A2(m->eta, i, j) = 0.1 * exp(-(x * x + y * y) / (R * R));
                A2(m->ubt, i, j) = 0.0;
                A2(m->vbt, i, j) = 0.0;
            }
    }
}

oracle_model *oracle_create(const oracle_config *c) {
    if (c->ni < 8 || c->nj < 8 || c->nk < 2 || c->bt_nsteps < 1) return NULL;
    const int gni = c->ni_global > 0 ? c->ni_global : c->ni;
    const int gnj = c->nj_global > 0 ? c->nj_global : c->nj;
    if (c->i_offset < 0 || c->j_offset < 0 || c->i_offset + (c->ni - 4) > gni - 4 ||
        c->j_offset + (c->nj - 4) > gnj - 4 || (c->cuts & ~15) || (c->cuts && c->bc_fill))
        return NULL;
    oracle_model *m = (oracle_model *)calloc(1, sizeof(oracle_model));
    m->cfg = *c;
    m->ni = c->ni; m->nj = c->nj; m->nk = c->nk;
    m->gni = gni; m->gnj = gnj; m->ioff = c->i_offset; m->joff = c->j_offset;
    m->cw = (c->cuts & OR_CUT_W) != 0; m->ce = (c->cuts & OR_CUT_E) != 0;
    m->cs = (c->cuts & OR_CUT_S) != 0; m->cn = (c->cuts & OR_CUT_N) != 0;
    /* mom6_types.F90:145-148 */
    m->isd = 1; m->ied = c->ni + 2; m->jsd = 1; m->jed = c->nj + 2;
    m->is = m->isd + 3; m->ie = m->ied - 3; m->js = m->jsd + 3; m->je = m->jed - 3;
    m->n1 = m->ied; m->n2 = m->jed;
    m->dt = c->dt;
    m->nstep = c->bt_nsteps;
    init_grid(m);
    alloc_all(m);
    init_state(m);
    if (c->bc_fill) {
        oracle_halo_fill(m, m->h0, m->nk, 0);
        oracle_halo_fill(m, m->h, m->nk, 0);
        oracle_halo_fill(m, m->u, m->nk, 1);
        oracle_halo_fill(m, m->v, m->nk, 2);
        oracle_halo_fill(m, m->eta, 1, 0);
        oracle_halo_fill(m, m->ubt, 1, 1);
        oracle_halo_fill(m, m->vbt, 1, 2);
    }
    return m;
}

void oracle_destroy(oracle_model *m) {
    if (!m) return;
    /* free every pointer member: they are laid out contiguously after cfg */
    double **p[] = {
        &m->IareaT, &m->areaT, &m->dxT, &m->dyT, &m->IdxT, &m->IdyT, &m->dxCu,
        &m->dyCu, &m->dy_Cu, &m->IdxCu, &m->IdyCu, &m->dxCv, &m->dyCv,
        &m->IdxCv, &m->IdyCv, &m->IareaBu, &m->areaBu, &m->CoriolisBu,
        &m->IareaCu, &m->IareaCv, &m->dxBu, &m->dyBu, &m->IdxBu, &m->IdyBu,
        &m->bathyT, &m->mask2dT, &m->mask2dBu, &m->mask2dCu, &m->mask2dCv,
        &m->u, &m->v, &m->h, &m->h0, &m->htmp, &m->uh, &m->vh, &m->CAu, &m->CAv,
        &m->up, &m->vp, &m->diffu, &m->diffv, &m->eta, &m->ubt, &m->vbt,
        &m->ubt_av, &m->vbt_av, &m->eta_av, &m->taux, &m->tauy, &m->Ray_u,
        &m->Ray_v, &m->c_uhbt, &m->u_cor, &m->du_cor, &m->por_face_areaU,
        &m->visc_rem_u, &m->hW, &m->hE, &m->FA_u_W0, &m->FA_u_WW, &m->FA_u_E0,
        &m->FA_u_EE, &m->uBT_WW, &m->uBT_EE, &m->BT_h_u, &m->co_dvdx,
        &m->co_dudy, &m->co_rel_vort, &m->co_abs_vort, &m->co_q, &m->co_Ih_q,
        &m->co_hArea_u, &m->co_hArea_v, &m->co_Area_q, &m->co_KE,
        &m->hv_Kh_bg_xx, &m->hv_Kh_bg_xy, &m->hv_dx2h, &m->hv_dy2h, &m->hv_dx2q,
        &m->hv_dy2q, &m->hv_DX_dyT, &m->hv_DY_dxT, &m->hv_DX_dyBu,
        &m->hv_DY_dxBu, &m->hv_red_xx, &m->hv_red_xy, &m->hv_dudx, &m->hv_dvdy,
        &m->hv_dvdx, &m->hv_dudy, &m->hv_sh_xx, &m->hv_sh_xy, &m->hv_str_xx,
        &m->hv_str_xy, &m->hv_h_u, &m->hv_h_v, &m->hv_hq, &m->hv_Kh, &m->vv_a_u,
        &m->vv_a_v, &m->vv_h_u, &m->vv_h_v, &m->vv_taux_bot, &m->vv_tauy_bot,
        &m->bt_eta, &m->bt_eta_pred, &m->bt_ubt, &m->bt_vbt, &m->bt_ubt_prev,
        &m->bt_vbt_prev, &m->bt_uhbt, &m->bt_vhbt, &m->bt_PFu, &m->bt_PFv,
        &m->bt_Cor_u, &m->bt_Cor_v, &m->bt_Datu, &m->bt_Datv, &m->bt_gtot_E,
        &m->bt_gtot_W, &m->bt_gtot_N, &m->bt_gtot_S, &m->bt_f_4_u, &m->bt_f_4_v,
        &m->bt_rem_u, &m->bt_rem_v, &m->bt_ubt_av, &m->bt_vbt_av,
        &m->hv_Ah_bg_xx, &m->hv_Ah_bg_xy, &m->hv_Kh_Max_xx, &m->hv_Kh_Max_xy,
        &m->hv_Ah_Max_xx, &m->hv_Ah_Max_xy, &m->hv_L2c_xx, &m->hv_L2c_xy, &m->hv_Bc_xx,
        &m->hv_Bc_xy, &m->hv_L3c_xx, &m->hv_L3c_xy, &m->hv_B6c_xx, &m->hv_B6c_xy,
        &m->hv_Idx2dyCu, &m->hv_Idxdy2u, &m->hv_Idx2dyCv, &m->hv_Idxdy2v, &m->hv_Ah,
        &m->hv_Shear_mag, &m->hv_Del2u, &m->hv_Del2v, &m->hv_hrat_min, &m->hv_vbr,
        &m->hv_vort, &m->hv_vort_dx, &m->hv_vort_dy, &m->hv_gvm_h, &m->hv_gvm_q,
        &m->hv_vvm, &m->hv_Del2vort_q, &m->hv_div, &m->hv_div_dx, &m->hv_div_dy,
        &m->hv_gdm_h, &m->hv_bhstr_xx, &m->hv_bhstr_xy};
    for (size_t a = 0; a < sizeof(p) / sizeof(p[0]); ++a) free(*p[a]);
    free(m->diag_work); free(m->diag_usum); free(m->diag_vsum);
    free(m->diag_KE); free(m->diag_mass);
    free(m->co_a); free(m->co_b); free(m->co_c); free(m->co_d); free(m->visc_rem_v);
    free(m->hz); free(m->BT_h_v); free(m->FA_v_S0); free(m->FA_v_SS); free(m->FA_v_N0);
    free(m->FA_v_NN); free(m->vBT_SS); free(m->vBT_NN); free(m->dv_cor);
    for (int q = 0; q < 22; ++q) free(m->mt[q]);
    free(m);
}

/* ------------------------------------------------------------------------ */
/* halo / boundary fill (periodic in i, solid walls in j)                   */
/* kind 0: h-point, 1: u-point, 2: v-point.                                 */
/* ------------------------------------------------------------------------ */
void oracle_halo_fill(const oracle_model *m, double *f, int nz, int kind) {
    int is = m->is, ie = m->ie, js = m->js, je = m->je;
    int P = ie - is + 1;
    for (int k = 1; k <= nz; ++k) {
        /* walls in j: mirror h/u rows, antisymmetric v rows about the wall
         * faces js-1 and je (which stay as the dynamics left them) */
        for (int i = 1; i <= N1; ++i) {
            if (kind == 2) {
                for (int J = 1; J <= js - 2; ++J)
                    A3(f, i, J, k) = -A3(f, i, 2 * (js - 1) - J, k);
                for (int J = je + 1; J <= N2; ++J)
                    A3(f, i, J, k) = -A3(f, i, 2 * je - J, k);
            } else {
                for (int j = 1; j <= js - 1; ++j)
                    A3(f, i, j, k) = A3(f, i, 2 * js - 1 - j, k);
                for (int j = je + 1; j <= N2; ++j)
                    A3(f, i, j, k) = A3(f, i, 2 * je + 1 - j, k);
            }
        }
        /* periodic in i (corners take the j-filled values) */
        int lo_end = (kind == 1) ? is - 2 : is - 1; /* u faces is-1 and ie */
        for (int j = 1; j <= N2; ++j) {
            for (int i = 1; i <= lo_end; ++i) A3(f, i, j, k) = A3(f, i + P, j, k);
            for (int i = ie + 1; i <= N1; ++i) A3(f, i, j, k) = A3(f, i - P, j, k);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* compute_transports, rk2_serial_driver.F90:544-561                        */
/* ------------------------------------------------------------------------ */
void oracle_compute_transports(oracle_model *m, const double *u, const double *v,
                               const double *h, double *uh, double *vh) {
    OMP_FOR
    for (int k = 1; k <= m->nk; ++k)
        for (int j = m->jsd; j <= m->jed; ++j)
            for (int i = m->isd; i <= m->ied; ++i) {
                int ip = MIN(i + 1, m->ied), jp = j + 1 < m->jed ? j + 1 : m->jed;
                A3(uh, i, j, k) = A3(u, i, j, k) * 0.5 *
                                  (A3(h, i, j, k) + A3(h, ip, j, k)) * A2(m->dyCu, i, j);
                A3(vh, i, j, k) = A3(v, i, j, k) * 0.5 *
                                  (A3(h, i, j, k) + A3(h, i, jp, k)) * A2(m->dxCv, i, j);
            }
}

/* ------------------------------------------------------------------------ */
/* hor_visc_init's scheme options, mom6_hor_visc_serial.F90:160-286: the     */
/* flags as the optional arguments set them (:177-193), the background and   */
/* maximum viscosities, the Smagorinsky / Leith constants and biharmonic     */
/* metrics (:207-268), and the work arrays reset to their initial values     */
/* (:271-282).  modified_Leith (:49) has no hor_visc_init argument; it is    */
/* the extra flag here.                                                      */
/* ------------------------------------------------------------------------ */
int oracle_set_hor_visc(oracle_model *m, const oracle_hor_visc_opts *o) {
    m->hv_lap = o->laplacian != 0;
    m->hv_bih = o->biharmonic != 0;
    m->hv_smag_kh = o->smagorinsky && m->hv_lap;
    m->hv_smag_ah = o->smagorinsky && m->hv_bih;
    m->hv_leith_kh = o->leith != 0;
    m->hv_leith_ah = o->leith && m->hv_bih;
    m->hv_no_slip = o->no_slip != 0;
    m->hv_bb_kh = m->hv_bb_ah = m->hv_bound_kh = m->hv_bound_ah = o->better_bound != 0;
    m->hv_mod_leith = o->modified_leith != 0;
    const double Smag_Lap_const = 0.15, Smag_bi_const = 0.06, Leith_const = 1.0;
    for (int j = m->jsd; j <= m->jed; ++j)
        for (int i = m->isd; i <= m->ied; ++i) {
            A2(m->hv_Idx2dyCu, i, j) = A2(m->IdxCu, i, j) * A2(m->IdxCu, i, j) * A2(m->IdyCu, i, j);
            A2(m->hv_Idxdy2u, i, j) = A2(m->IdxCu, i, j) * A2(m->IdyCu, i, j) * A2(m->IdyCu, i, j);
            A2(m->hv_Idx2dyCv, i, j) = A2(m->IdxCv, i, j) * A2(m->IdxCv, i, j) * A2(m->IdyCv, i, j);
            A2(m->hv_Idxdy2v, i, j) = A2(m->IdxCv, i, j) * A2(m->IdyCv, i, j) * A2(m->IdyCv, i, j);
            double h2 = A2(m->areaT, i, j);
            double h3 = sqrt(h2) * h2;
            double h4 = h2 * h2;
            A2(m->hv_Ah_bg_xx, i, j) = o->Ah;
            A2(m->hv_Ah_bg_xy, i, j) = o->Ah;
            A2(m->hv_Kh_Max_xx, i, j) = 0.25 * h2 / 1.0;
            A2(m->hv_Kh_Max_xy, i, j) = 0.25 * h2 / 1.0;
            A2(m->hv_Ah_Max_xx, i, j) = 0.0625 * h4 / 1.0;
            A2(m->hv_Ah_Max_xy, i, j) = 0.0625 * h4 / 1.0;
            A2(m->hv_L2c_xx, i, j) = Smag_Lap_const * Smag_Lap_const * h2;
            A2(m->hv_L2c_xy, i, j) = Smag_Lap_const * Smag_Lap_const * h2;
            A2(m->hv_Bc_xx, i, j) = Smag_bi_const * Smag_bi_const * h4;
            A2(m->hv_Bc_xy, i, j) = Smag_bi_const * Smag_bi_const * h4;
            A2(m->hv_L3c_xx, i, j) = Leith_const * h3;
            A2(m->hv_L3c_xy, i, j) = Leith_const * h3;
            A2(m->hv_B6c_xx, i, j) = Leith_const * h3 * h3;
            A2(m->hv_B6c_xy, i, j) = Leith_const * h3 * h3;
        }
    size_t n2d = (size_t)N1 * N2;
    double *zero[] = {m->hv_dudx, m->hv_dvdy, m->hv_dvdx, m->hv_dudy, m->hv_sh_xx,
                      m->hv_sh_xy, m->hv_str_xx, m->hv_str_xy, m->hv_h_u, m->hv_h_v,
                      m->hv_hq, m->hv_Kh, m->hv_Ah, m->hv_Shear_mag, m->hv_Del2u,
                      m->hv_Del2v, m->hv_vort, m->hv_vort_dx, m->hv_vort_dy, m->hv_gvm_h,
                      m->hv_gvm_q, m->hv_vvm, m->hv_div, m->hv_div_dx, m->hv_div_dy,
                      m->hv_gdm_h, m->hv_bhstr_xx, m->hv_bhstr_xy, m->hv_Del2vort_q};
    for (size_t a = 0; a < sizeof(zero) / sizeof(zero[0]); ++a)
        memset(zero[a], 0, n2d * sizeof(double));
    for (size_t q = 0; q < n2d; ++q) {
        m->hv_hrat_min[q] = 1.0;
        m->hv_vbr[q] = 1.0;
    }
    return 0;
}

/* inv_PI3 = 1/3.14159265358979**3 and inv_PI6 = 1/3.14159265358979**6
 * (mom6_hor_visc_serial.F90:154-155): the powers and quotients correctly
 * rounded (a compile-time constant folded exactly; the run-time products
 * x*x*x and (x*x*x)*(x*x*x) round to the same doubles). */
static const double kInvPI3 = 0x1.08345eb45d78dp-5;
static const double kInvPI6 = 0x1.10ac0e0a9d181p-10;
#define SQ(x) ((x) * (x))

/* ------------------------------------------------------------------------ */
/* hor_visc, mom6_hor_visc_serial.F90:464-1109, every branch but FrictWork   */
/* (compute_FrictWork has no setter).  CS%Kh and CS%Ah are persistent arrays */
/* shared by h- and q-points, as in the reference; the other work arrays     */
/* keep their values outside the ranges each step writes.                    */
/* ------------------------------------------------------------------------ */
static void hor_visc_rows(oracle_model *m, const double *u, const double *v,
                          const double *h, double *diffu, double *diffv, int k) {
    int is = m->is, ie = m->ie, js = m->js, je = m->je;
    int Isq = is - 1, Ieq = ie, Jsq = js - 1, Jeq = je;
    double h_neglect = m->hv_h_neglect;
    double *dudx = m->hv_dudx, *dvdy = m->hv_dvdy, *dvdx = m->hv_dvdx,
           *dudy = m->hv_dudy, *sh_xx = m->hv_sh_xx, *sh_xy = m->hv_sh_xy,
           *str_xx = m->hv_str_xx, *str_xy = m->hv_str_xy, *h_u = m->hv_h_u,
           *h_v = m->hv_h_v, *hq = m->hv_hq, *Kh = m->hv_Kh, *Ah = m->hv_Ah,
           *Del2u = m->hv_Del2u, *Del2v = m->hv_Del2v, *vort = m->hv_vort,
           *vdx = m->hv_vort_dx, *vdy = m->hv_vort_dy, *D2vq = m->hv_Del2vort_q,
           *div = m->hv_div, *ddx = m->hv_div_dx, *ddy = m->hv_div_dy,
           *hrat = m->hv_hrat_min, *vbr = m->hv_vbr;
    /* STEP 1 */
    OMP_FOR
    for (int j = Jsq; j <= Jeq + 1; ++j)
        for (int i = Isq; i <= Ieq + 1; ++i) {
            A2(dudx, i, j) = A2(m->hv_DY_dxT, i, j) *
                             ((A2(m->IdyCu, i, j) * A3(u, i, j, k)) -
                              (A2(m->IdyCu, i - 1, j) * A3(u, i - 1, j, k)));
            A2(dvdy, i, j) = A2(m->hv_DX_dyT, i, j) *
                             ((A2(m->IdxCv, i, j) * A3(v, i, j, k)) -
                              (A2(m->IdxCv, i, j - 1) * A3(v, i, j - 1, k)));
        }
    OMP_FOR
    for (int J = Jsq; J <= Jeq; ++J)
        for (int I = Isq; I <= Ieq; ++I) {
            A2(dvdx, I, J) = A2(m->hv_DY_dxBu, I, J) *
                             ((A3(v, I + 1, J, k) * A2(m->IdyCv, I + 1, J)) -
                              (A3(v, I, J, k) * A2(m->IdyCv, I, J)));
            A2(dudy, I, J) = A2(m->hv_DX_dyBu, I, J) *
                             ((A3(u, I, J + 1, k) * A2(m->IdxCu, I, J + 1)) -
                              (A3(u, I, J, k) * A2(m->IdxCu, I, J)));
        }
    /* STEP 2 */
    OMP_FOR
    for (int j = Jsq; j <= Jeq + 1; ++j)
        for (int i = Isq; i <= Ieq + 1; ++i)
            A2(sh_xx, i, j) = A2(dudx, i, j) - A2(dvdy, i, j);
    OMP_FOR
    for (int J = Jsq; J <= Jeq; ++J)
        for (int I = Isq; I <= Ieq; ++I)
            A2(sh_xy, I, J) = (m->hv_no_slip ? (2.0 - A2(m->mask2dBu, I, J))
                                             : A2(m->mask2dBu, I, J)) *
                              (A2(dvdx, I, J) + A2(dudy, I, J));
    /* STEP 3 (use_land_mask) */
    OMP_FOR
    for (int j = js - 1; j <= je + 1; ++j)
        for (int I = Isq; I <= Ieq; ++I)
            A2(h_u, I, j) = 0.5 * (A2(m->mask2dT, I, j) * A3(h, I, j, k) +
                                   A2(m->mask2dT, I + 1, j) * A3(h, I + 1, j, k));
    OMP_FOR
    for (int J = Jsq; J <= Jeq; ++J)
        for (int i = is - 1; i <= ie + 1; ++i)
            A2(h_v, i, J) = 0.5 * (A2(m->mask2dT, i, J) * A3(h, i, J, k) +
                                   A2(m->mask2dT, i, J + 1) * A3(h, i, J + 1, k));
    OMP_FOR
    for (int J = Jsq; J <= Jeq; ++J)
        for (int I = Isq; I <= Ieq; ++I)
            A2(hq, I, J) = 0.25 * ((A3(h, I, J, k) + A3(h, I + 1, J + 1, k)) +
                                   (A3(h, I + 1, J, k) + A3(h, I, J + 1, k)));
    /* STEP 4: Del2u, Del2v (:587-608) */
    if (m->hv_bih) {
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int I = Isq; I <= Ieq; ++I)
                A2(Del2u, I, j) =
                    A2(m->hv_Idx2dyCu, I, j) * ((A2(m->hv_dx2q, I, j) * A2(sh_xy, I, j)) -
                                                (A2(m->hv_dx2q, I, j - 1) * A2(sh_xy, I, j - 1))) +
                    A2(m->hv_Idxdy2u, I, j) * ((A2(m->hv_dy2h, I + 1, j) * A2(sh_xx, I + 1, j)) -
                                               (A2(m->hv_dy2h, I, j) * A2(sh_xx, I, j)));
        OMP_FOR
        for (int J = Jsq; J <= Jeq; ++J)
            for (int i = is; i <= ie; ++i)
                A2(Del2v, i, J) =
                    A2(m->hv_Idxdy2v, i, J) * ((A2(m->hv_dy2q, i, J) * A2(sh_xy, i, J)) -
                                               (A2(m->hv_dy2q, i - 1, J) * A2(sh_xy, i - 1, J))) -
                    A2(m->hv_Idx2dyCv, i, J) * ((A2(m->hv_dx2h, i, J + 1) * A2(sh_xx, i, J + 1)) -
                                                (A2(m->hv_dx2h, i, J) * A2(sh_xx, i, J)));
    }
    /* STEP 5: Leith vorticity (:612-714) */
    if (m->hv_leith_kh) {
        OMP_FOR
        for (int J = Jsq; J <= Jeq; ++J)
            for (int I = Isq; I <= Ieq; ++I)
                A2(vort, I, J) = (m->hv_no_slip ? (2.0 - A2(m->mask2dBu, I, J))
                                                : A2(m->mask2dBu, I, J)) *
                                 (A2(dvdx, I, J) - A2(dudy, I, J));
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int i = is; i <= ie; ++i) {
                double DY_dxBu_loc = A2(m->dyBu, i, j) * A2(m->IdxBu, i, j);
                A2(vdx, i, j) = DY_dxBu_loc * ((A2(vort, i, j) * A2(m->IdyCu, i, j)) -
                                               (A2(vort, i - 1, j) * A2(m->IdyCu, i - 1, j)));
            }
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int I = Isq; I <= Ieq; ++I) {
                double DX_dyBu_loc = A2(m->dxBu, I, j) * A2(m->IdyBu, I, j);
                A2(vdy, I, j) = DX_dyBu_loc * ((A2(vort, I, j) * A2(m->IdxCv, I, j)) -
                                               (A2(vort, I, j - 1) * A2(m->IdxCv, I, j - 1)));
            }
        if (m->hv_leith_ah) {
            OMP_FOR
            for (int J = Jsq; J <= Jeq; ++J)
                for (int I = Isq; I <= Ieq; ++I)
                    A2(D2vq, I, J) =
                        A2(m->hv_DY_dxBu, I, J) * ((A2(vdx, I + 1, J) * A2(m->IdyCv, I + 1, J)) -
                                                   (A2(vdx, I, J) * A2(m->IdyCv, I, J))) +
                        A2(m->hv_DX_dyBu, I, J) * ((A2(vdy, I, J + 1) * A2(m->IdxCu, I, J + 1)) -
                                                   (A2(vdy, I, J) * A2(m->IdxCu, I, J)));
        }
        if (m->hv_mod_leith) {
            OMP_FOR
            for (int j = js; j <= je; ++j)
                for (int i = is; i <= ie; ++i) A2(div, i, j) = A2(dudx, i, j) + A2(dvdy, i, j);
            OMP_FOR
            for (int j = js; j <= je; ++j)
                for (int I = Isq; I <= Ieq; ++I)
                    A2(ddx, I, j) = A2(m->IdxCu, I, j) * (A2(div, I + 1, j) - A2(div, I, j));
            OMP_FOR
            for (int J = Jsq; J <= Jeq; ++J)
                for (int i = is; i <= ie; ++i)
                    A2(ddy, i, J) = A2(m->IdyCv, i, J) * (A2(div, i, J + 1) - A2(div, i, J));
            OMP_FOR
            for (int j = js; j <= je; ++j)
                for (int i = is; i <= ie; ++i)
                    A2(m->hv_gdm_h, i, j) =
                        sqrt(SQ(0.5 * (A2(ddx, i, j) + A2(ddx, i - 1, j))) +
                             SQ(0.5 * (A2(ddy, i, j) + A2(ddy, i, j - 1))));
        } else {
            OMP_FOR
            for (int j = js; j <= je; ++j)
                for (int i = is; i <= ie; ++i) A2(m->hv_gdm_h, i, j) = 0.0;
        }
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int i = is; i <= ie; ++i) {
                A2(m->hv_gvm_h, i, j) = sqrt(SQ(0.5 * (A2(vdx, i, j) + A2(vdx, i, j - 1))) +
                                             SQ(0.5 * (A2(vdy, i, j) + A2(vdy, i - 1, j))));
                A2(m->hv_vvm, i, j) = A2(m->hv_gvm_h, i, j) + A2(m->hv_gdm_h, i, j);
            }
        OMP_FOR
        for (int J = Jsq; J <= Jeq; ++J)
            for (int I = Isq; I <= Ieq; ++I)
                A2(m->hv_gvm_q, I, J) = sqrt(SQ(0.5 * (A2(vdx, I, J) + A2(vdx, I + 1, J))) +
                                             SQ(0.5 * (A2(vdy, I, J) + A2(vdy, I, J + 1))));
    }
    /* STEP 6: Smagorinsky shear magnitude (:718-727) */
    if (m->hv_smag_kh || m->hv_smag_ah) {
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int i = is; i <= ie; ++i) {
                double sh_xx_sq = SQ(A2(sh_xx, i, j));
                double sh_xy_sq = 0.25 * ((SQ(A2(sh_xy, i - 1, j - 1)) + SQ(A2(sh_xy, i, j))) +
                                          (SQ(A2(sh_xy, i - 1, j)) + SQ(A2(sh_xy, i, j - 1))));
                A2(m->hv_Shear_mag, i, j) = sqrt(sh_xx_sq + sh_xy_sq);
            }
    }
    /* STEP 7: thickness ratio (:732-739) */
    if (m->hv_bb_kh || m->hv_bb_ah) {
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int i = is; i <= ie; ++i) {
                double h_min = MIN(MIN(MIN(A2(h_u, i, j), A2(h_u, i - 1, j)), A2(h_v, i, j)),
                                   A2(h_v, i, j - 1));
                A2(hrat, i, j) = MIN(1.0, h_min / (A3(h, i, j, k) + h_neglect));
            }
    }
    /* STEP 8: Kh at h-points, str_xx (:744-816).  str_xx(ie+1, :) and
     * str_xx(:, je+1) read the shared Kh where this step does not write it;
     * at an east / north cut those cells are interior and get their Kh. */
    if (m->hv_lap) {
        OMP_FOR
        for (int j = js; j <= je + m->cn; ++j)
            for (int i = is; i <= ie + m->ce; ++i) {
                double K = A2(m->hv_Kh_bg_xx, i, j);
                if (m->hv_smag_kh) K = MAX(K, A2(m->hv_L2c_xx, i, j) * A2(m->hv_Shear_mag, i, j));
                if (m->hv_leith_kh)
                    K = MAX(K, A2(m->hv_L3c_xx, i, j) * A2(m->hv_vvm, i, j) * kInvPI3);
                K = MAX(K, m->hv_Kh_bg_min);
                if (m->hv_bb_kh && m->hv_bb_ah) {
                    A2(vbr, i, j) = 1.0;
                    double Kh_max_here = A2(hrat, i, j) * A2(m->hv_Kh_Max_xx, i, j);
                    if (K >= Kh_max_here) {
                        A2(vbr, i, j) = 0.0;
                        K = Kh_max_here;
                    } else if (K > 0.0) {
                        A2(vbr, i, j) = 1.0 - K / Kh_max_here;
                    }
                } else if (m->hv_bb_kh) {
                    K = MIN(K, A2(hrat, i, j) * A2(m->hv_Kh_Max_xx, i, j));
                } else if (m->hv_bound_kh) {
                    K = MIN(K, A2(m->hv_Kh_Max_xx, i, j));
                }
                A2(Kh, i, j) = K;
            }
        OMP_FOR
        for (int j = Jsq; j <= Jeq + 1; ++j)
            for (int i = Isq; i <= Ieq + 1; ++i)
                A2(str_xx, i, j) = -(A2(Kh, i, j) * A2(sh_xx, i, j));
    } else {
        OMP_FOR
        for (int j = Jsq; j <= Jeq + 1; ++j)
            for (int i = Isq; i <= Ieq + 1; ++i) A2(str_xx, i, j) = 0.0;
    }
    /* STEP 9: Ah at h-points, biharmonic str_xx (:824-896) */
    if (m->hv_bih) {
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int i = is; i <= ie; ++i) {
                double A = A2(m->hv_Ah_bg_xx, i, j);
                if (m->hv_smag_ah) A = MAX(A, A2(m->hv_Bc_xx, i, j) * A2(m->hv_Shear_mag, i, j));
                if (m->hv_leith_ah) {
                    double Del2vort_h = 0.25 * ((A2(D2vq, i, j) + A2(D2vq, i - 1, j - 1)) +
                                                (A2(D2vq, i - 1, j) + A2(D2vq, i, j - 1)));
                    A = MAX(A, A2(m->hv_B6c_xx, i, j) * fabs(Del2vort_h) * kInvPI6);
                }
                if (m->hv_bb_ah) {
                    if (m->hv_bb_kh)
                        A = MIN(A, A2(vbr, i, j) * A2(hrat, i, j) * A2(m->hv_Ah_Max_xx, i, j));
                    else
                        A = MIN(A, A2(hrat, i, j) * A2(m->hv_Ah_Max_xx, i, j));
                } else if (m->hv_bound_ah) {
                    A = MIN(A, A2(m->hv_Ah_Max_xx, i, j));
                }
                A2(Ah, i, j) = A;
            }
        OMP_FOR
        for (int j = Jsq; j <= Jeq + 1; ++j)
            for (int i = Isq; i <= Ieq + 1; ++i) {
                double d_del2u = (A2(m->IdyCu, i, j) * A2(Del2u, i, j)) -
                                 (A2(m->IdyCu, i - 1, j) * A2(Del2u, i - 1, j));
                double d_del2v = (A2(m->IdxCv, i, j) * A2(Del2v, i, j)) -
                                 (A2(m->IdxCv, i, j - 1) * A2(Del2v, i, j - 1));
                double d_str = A2(Ah, i, j) * ((A2(m->hv_DY_dxT, i, j) * d_del2u) -
                                               (A2(m->hv_DX_dyT, i, j) * d_del2v));
                A2(m->hv_bhstr_xx, i, j) = d_str * (A3(h, i, j, k) * A2(m->hv_red_xx, i, j));
                A2(str_xx, i, j) = A2(str_xx, i, j) + d_str;
            }
    }
    /* STEP 10 */
    OMP_FOR
    for (int j = Jsq; j <= Jeq + 1; ++j)
        for (int i = Isq; i <= Ieq + 1; ++i)
            A2(str_xx, i, j) = A2(str_xx, i, j) * (A3(h, i, j, k) * A2(m->hv_red_xx, i, j));
    /* STEP 11: Kh at q-points (overwrites the shared CS%Kh), str_xy (:900-974) */
    if (m->hv_lap) {
        OMP_FOR
        for (int J = Jsq; J <= Jeq; ++J)
            for (int I = Isq; I <= Ieq; ++I) {
                double K = A2(m->hv_Kh_bg_xy, I, J);
                if (m->hv_smag_kh) {
                    double sh_xx_sq = 0.25 * ((SQ(A2(sh_xx, I, J)) + SQ(A2(sh_xx, I + 1, J + 1))) +
                                              (SQ(A2(sh_xx, I + 1, J)) + SQ(A2(sh_xx, I, J + 1))));
                    double sh_xy_sq = SQ(A2(sh_xy, I, J));
                    K = MAX(K, A2(m->hv_L2c_xy, I, J) * sqrt(sh_xx_sq + sh_xy_sq));
                }
                if (m->hv_leith_kh)
                    K = MAX(K, A2(m->hv_L3c_xy, I, J) * A2(m->hv_gvm_q, I, J) * kInvPI3);
                K = MAX(K, m->hv_Kh_bg_min);
                if (m->hv_bb_kh) {
                    double h_min = 0.25 * ((A2(hrat, I, J) + A2(hrat, I + 1, J + 1)) +
                                           (A2(hrat, I + 1, J) + A2(hrat, I, J + 1)));
                    K = MIN(K, h_min * A2(m->hv_Kh_Max_xy, I, J));
                } else if (m->hv_bound_kh) {
                    K = MIN(K, A2(m->hv_Kh_Max_xy, I, J));
                }
                A2(Kh, I, J) = K;
                A2(str_xy, I, J) = -(K * A2(sh_xy, I, J));
            }
    } else {
        OMP_FOR
        for (int J = Jsq; J <= Jeq; ++J)
            for (int I = Isq; I <= Ieq; ++I) A2(str_xy, I, J) = 0.0;
    }
    /* STEP 12: Ah at q-points, biharmonic str_xy (:979-1035) */
    if (m->hv_bih) {
        OMP_FOR
        for (int J = Jsq; J <= Jeq; ++J)
            for (int I = Isq; I <= Ieq; ++I) {
                double A = A2(m->hv_Ah_bg_xy, I, J);
                if (m->hv_smag_ah) {
                    double sh_xx_sq = 0.25 * ((SQ(A2(sh_xx, I, J)) + SQ(A2(sh_xx, I + 1, J + 1))) +
                                              (SQ(A2(sh_xx, I + 1, J)) + SQ(A2(sh_xx, I, J + 1))));
                    double sh_xy_sq = SQ(A2(sh_xy, I, J));
                    A = MAX(A, A2(m->hv_Bc_xy, I, J) * sqrt(sh_xx_sq + sh_xy_sq));
                }
                if (m->hv_leith_ah)
                    A = MAX(A, A2(m->hv_B6c_xy, I, J) * fabs(A2(D2vq, I, J)) * kInvPI6);
                if (m->hv_bb_ah) {
                    double h_min = 0.25 * ((A2(hrat, I, J) + A2(hrat, I + 1, J + 1)) +
                                           (A2(hrat, I + 1, J) + A2(hrat, I, J + 1)));
                    A = MIN(A, h_min * A2(m->hv_Ah_Max_xy, I, J));
                } else if (m->hv_bound_ah) {
                    A = MIN(A, A2(m->hv_Ah_Max_xy, I, J));
                }
                A2(Ah, I, J) = A;
                double d_str =
                    A * ((A2(m->hv_DY_dxBu, I, J) * ((A2(Del2v, I + 1, J) * A2(m->IdyCv, I + 1, J)) -
                                                     (A2(Del2v, I, J) * A2(m->IdyCv, I, J)))) +
                         (A2(m->hv_DX_dyBu, I, J) * ((A2(Del2u, I, J + 1) * A2(m->IdxCu, I, J + 1)) -
                                                     (A2(Del2u, I, J) * A2(m->IdxCu, I, J)))));
                A2(m->hv_bhstr_xy, I, J) = d_str * (A2(hq, I, J) * A2(m->hv_red_xy, I, J));
                A2(str_xy, I, J) = A2(str_xy, I, J) + d_str;
            }
    }
    /* STEP 13 */
    OMP_FOR
    for (int J = Jsq; J <= Jeq; ++J)
        for (int I = Isq; I <= Ieq; ++I)
            A2(str_xy, I, J) =
                m->hv_no_slip
                    ? A2(str_xy, I, J) * (A2(hq, I, J) * A2(m->hv_red_xy, I, J))
                    : A2(str_xy, I, J) *
                          (A2(hq, I, J) * A2(m->mask2dBu, I, J) * A2(m->hv_red_xy, I, J));
    /* STEP 14 */
    OMP_FOR
    for (int j = js; j <= je; ++j)
        for (int I = Isq; I <= Ieq; ++I)
            A3(diffu, I, j, k) =
                ((A2(m->IdxCu, I, j) * ((A2(m->hv_dx2q, I, j - 1) * A2(str_xy, I, j - 1)) -
                                        (A2(m->hv_dx2q, I, j) * A2(str_xy, I, j))) +
                  A2(m->IdyCu, I, j) * ((A2(m->hv_dy2h, I, j) * A2(str_xx, I, j)) -
                                        (A2(m->hv_dy2h, I + 1, j) * A2(str_xx, I + 1, j)))) *
                 A2(m->IareaCu, I, j)) /
                (A2(h_u, I, j) + h_neglect);
    OMP_FOR
    for (int J = Jsq; J <= Jeq; ++J)
        for (int i = is; i <= ie; ++i)
            A3(diffv, i, J, k) =
                ((A2(m->IdyCv, i, J) * ((A2(m->hv_dy2q, i - 1, J) * A2(str_xy, i - 1, J)) -
                                        (A2(m->hv_dy2q, i, J) * A2(str_xy, i, J))) -
                  A2(m->IdxCv, i, J) * ((A2(m->hv_dx2h, i, J) * A2(str_xx, i, J)) -
                                        (A2(m->hv_dx2h, i, J + 1) * A2(str_xx, i, J + 1)))) *
                 A2(m->IareaCv, i, J)) /
                (A2(h_v, i, J) + h_neglect);
}
#undef SQ

void oracle_hor_visc(oracle_model *m, const double *u, const double *v,
                     const double *h, double *diffu, double *diffv) {
    size_t n3d = (size_t)N1 * N2 * m->nk;
    memset(diffu, 0, n3d * sizeof(double));
    memset(diffv, 0, n3d * sizeof(double));
    for (int k = 1; k <= m->nk; ++k) hor_visc_rows(m, u, v, h, diffu, diffv, k);
}

/* ------------------------------------------------------------------------ */
/* CorAdCalc, mom6_coriolis_serial.F90:112-252 (Sadourny energy scheme).    */
/* hArea_u(:,js-1) and hArea_v(is-1,:) are never written and stay zero.     */
/* ------------------------------------------------------------------------ */
void oracle_coriolis(oracle_model *m, const double *u, const double *v,
                     const double *h, const double *uh, const double *vh,
                     double *CAu, double *CAv) {
    int is = m->is, ie = m->ie, js = m->js, je = m->je;
    const double vol_neglect = 1.0e-20;
    double *dvdx = m->co_dvdx, *dudy = m->co_dudy, *rel = m->co_rel_vort,
           *absv = m->co_abs_vort, *q = m->co_q, *Ihq = m->co_Ih_q,
           *hAu = m->co_hArea_u, *hAv = m->co_hArea_v, *KE = m->co_KE;
    for (int k = 1; k <= m->nk; ++k) {
        OMP_FOR
        for (int j = js - 1; j <= je; ++j)
            for (int i = is - 1; i <= ie; ++i) {
                A2(dvdx, i, j) = (A3(v, i + 1, j, k) * A2(m->dyCv, i + 1, j)) -
                                 (A3(v, i, j, k) * A2(m->dyCv, i, j));
                A2(dudy, i, j) = (A3(u, i, j + 1, k) * A2(m->dxCu, i, j + 1)) -
                                 (A3(u, i, j, k) * A2(m->dxCu, i, j));
            }
        /* at a west / south cut the q-points on the cut are interior: their
         * hArea_v(is-1, :) / hArea_u(:, js-1) exist */
        OMP_FOR
        for (int j = js - 1; j <= je; ++j)
            for (int i = is - m->cw; i <= ie + 1; ++i)
                A2(hAv, i, j) = 0.5 * ((A2(m->areaT, i, j) * A3(h, i, j, k)) +
                                       (A2(m->areaT, i, j + 1) * A3(h, i, j + 1, k)));
        OMP_FOR
        for (int j = js - m->cs; j <= je + 1; ++j)
            for (int i = is - 1; i <= ie; ++i)
                A2(hAu, i, j) = 0.5 * ((A2(m->areaT, i, j) * A3(h, i, j, k)) +
                                       (A2(m->areaT, i + 1, j) * A3(h, i + 1, j, k)));
        OMP_FOR
        for (int j = js - 1; j <= je; ++j)
            for (int i = is - 1; i <= ie; ++i) {
                A2(rel, i, j) = A2(m->mask2dBu, i, j) * (A2(dvdx, i, j) - A2(dudy, i, j)) *
                                A2(m->IareaBu, i, j);
                A2(absv, i, j) = A2(m->CoriolisBu, i, j) + A2(rel, i, j);
            }
        OMP_FOR
        for (int j = js - 1; j <= je; ++j)
            for (int i = is - 1; i <= ie; ++i) {
                double hArea_q = (A2(hAu, i, j) + A2(hAu, i, j + 1)) +
                                 (A2(hAv, i, j) + A2(hAv, i + 1, j));
                A2(Ihq, i, j) = A2(m->co_Area_q, i, j) / (hArea_q + vol_neglect);
                A2(q, i, j) = A2(absv, i, j) * A2(Ihq, i, j);
            }
        /* the Arakawa schemes' coefficients, :171-193 */
        double *ca = m->co_a, *cb = m->co_b, *cc = m->co_c, *cd = m->co_d;
        const double C1_12 = 1.0 / 12.0, C1_24 = 1.0 / 24.0;
        if (m->cor_scheme == 2) {
            for (int j = js; j <= je; ++j)
                for (int i = is - 1; i <= ie; ++i) {
                    A2(ca, i, j) = (A2(q, i, j) + (A2(q, i + 1, j) + A2(q, i, j - 1))) * C1_12;
                    A2(cd, i, j) = ((A2(q, i, j) + A2(q, i + 1, j - 1)) + A2(q, i, j - 1)) * C1_12;
                }
            for (int j = js; j <= je; ++j)
                for (int i = is; i <= ie; ++i) {
                    A2(cb, i, j) = (A2(q, i, j) + (A2(q, i - 1, j) + A2(q, i, j - 1))) * C1_12;
                    A2(cc, i, j) = ((A2(q, i, j) + A2(q, i - 1, j - 1)) + A2(q, i, j - 1)) * C1_12;
                }
        } else if (m->cor_scheme == 3) {
            for (int j = js; j <= je; ++j)
                for (int i = is; i <= ie; ++i) {
                    A2(ca, i - 1, j) = (2.0 * (A2(q, i, j) + A2(q, i - 1, j - 1)) +
                                        (A2(q, i - 1, j) + A2(q, i, j - 1))) * C1_24;
                    A2(cd, i - 1, j) = ((A2(q, i, j) + A2(q, i - 1, j - 1)) +
                                        2.0 * (A2(q, i - 1, j) + A2(q, i, j - 1))) * C1_24;
                    A2(cb, i, j) = ((A2(q, i, j) + A2(q, i - 1, j - 1)) +
                                    2.0 * (A2(q, i - 1, j) + A2(q, i, j - 1))) * C1_24;
                    A2(cc, i, j) = (2.0 * (A2(q, i, j) + A2(q, i - 1, j - 1)) +
                                    (A2(q, i - 1, j) + A2(q, i, j - 1))) * C1_24;
                }
        }
        /* at a cut the face on it is interior: KE one cell further */
        OMP_FOR
        for (int j = js; j <= je + m->cn; ++j)
            for (int i = is; i <= ie + m->ce; ++i) {
                double u0 = A3(u, i, j, k), um = A3(u, i - 1, j, k);
                double v0 = A3(v, i, j, k), vm = A3(v, i, j - 1, k);
                A2(KE, i, j) = 0.25 *
                               ((A2(m->dyCu, i, j) * (u0 * u0) + A2(m->dyCu, i - 1, j) * (um * um)) +
                                (A2(m->dxCv, i, j) * (v0 * v0) + A2(m->dxCv, i, j - 1) * (vm * vm))) /
                               A2(m->areaT, i, j);
            }
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int i = is; i <= ie - 1 + m->ce; ++i) {
                double KEx = (A2(KE, i + 1, j) - A2(KE, i, j)) * A2(m->IdxCu, i, j);
                if (m->cor_scheme <= 1)
                    A3(CAu, i, j, k) =
                        0.25 *
                            ((A2(q, i, j) * (A3(vh, i + 1, j, k) + A3(vh, i, j, k))) +
                             (A2(q, i, j - 1) * (A3(vh, i, j - 1, k) + A3(vh, i + 1, j - 1, k)))) *
                            A2(m->IdxCu, i, j) -
                        KEx;
                else   /* :230-236 */
                    A3(CAu, i, j, k) =
                        (((A2(ca, i, j) * A3(vh, i + 1, j, k)) + (A2(cc, i, j) * A3(vh, i, j - 1, k))) +
                         ((A2(cb, i, j) * A3(vh, i, j, k)) +
                          (A2(cd, i, j) * A3(vh, i + 1, j - 1, k)))) *
                            A2(m->IdxCu, i, j) -
                        KEx;
            }
        OMP_FOR
        for (int j = js; j <= je - 1 + m->cn; ++j)
            for (int i = is; i <= ie; ++i) {
                double KEy = (A2(KE, i, j + 1) - A2(KE, i, j)) * A2(m->IdyCv, i, j);
                if (m->cor_scheme <= 1)
                    A3(CAv, i, j, k) =
                        -0.25 *
                            ((A2(q, i - 1, j) * (A3(uh, i - 1, j, k) + A3(uh, i - 1, j + 1, k))) +
                             (A2(q, i, j) * (A3(uh, i, j, k) + A3(uh, i, j + 1, k)))) *
                            A2(m->IdyCv, i, j) -
                        KEy;
                else   /* :238-245 */
                    A3(CAv, i, j, k) =
                        -(((A2(ca, i - 1, j) * A3(uh, i - 1, j, k)) +
                           (A2(cc, i, j + 1) * A3(uh, i, j + 1, k))) +
                          ((A2(cb, i, j) * A3(uh, i, j, k)) +
                           (A2(cd, i - 1, j + 1) * A3(uh, i - 1, j + 1, k)))) *
                            A2(m->IdyCv, i, j) -
                        KEy;
            }
    }
}

/* ------------------------------------------------------------------------ */
/* vert_visc_coef + vert_visc_apply, mom6_vert_visc_serial.F90:138-287 and  */
/* :394-506, with the driver's forces (taux, tauy) and Rayleigh drag.       */
/* ------------------------------------------------------------------------ */
static double botfn_of(double z2) {
    return 1.0 / (1.0 + 0.09 * z2 * z2 * z2 * z2 * z2 * z2);
}

static void vv_coef_column(oracle_model *m, const double *vel, const double *h,
                           int i, int j, int di, int dj, double *a, double *hv_out,
                           double *hvel, double *z_i) {
    const oracle_config *c = &m->cfg;
    int nz = m->nk;
    double h_neglect = m->Angstrom_H;
    double I_Hbbl = 1.0 / (c->Hbbl + h_neglect);
    z_i[nz + 1] = 0.0;
    for (int k = nz; k >= 1; --k) {
        double h0 = A3(h, i, j, k), h1 = A3(h, i + di, j + dj, k);
        double h_harm = 2.0 * h0 * h1 / (h0 + h1 + h_neglect);
        double h_arith = 0.5 * (h1 + h0);
        double h_delta = h1 - h0;
        hvel[k] = h_harm;
        if (A3(vel, i, j, k) * h_delta < 0.0) {
            double z2 = z_i[k + 1];
            double botfn = botfn_of(z2);
            hvel[k] = (1.0 - botfn) * h_harm + botfn * h_arith;
        }
        z_i[k] = z_i[k + 1] + h_harm * I_Hbbl;
    }
    a[1] = 0.0;
    double z_top = 0.0;
    for (int K2 = 2; K2 <= nz; ++K2) {
        z_top = z_top + hvel[K2 - 1];
        double Kv_tot = c->Kv;
        if (z_top < c->Hmix) {
            double topfn = 1.0 - z_top / c->Hmix;
            Kv_tot = Kv_tot + (c->Kv_ml - c->Kv) * topfn;
        }
        double z2 = z_i[K2];
        double botfn = botfn_of(z2);
        Kv_tot = Kv_tot + c->Kv_extra_bbl * botfn;
        double h_shear = 0.5 * (hvel[K2] + hvel[K2 - 1] + h_neglect);
        a[K2] = Kv_tot / h_shear;
    }
    a[nz + 1] = (c->Kv + c->Kv_extra_bbl) / (0.5 * hvel[nz] + h_neglect);
    for (int k = 1; k <= nz; ++k) hv_out[k] = hvel[k] + h_neglect;
}

static void vv_apply_column(oracle_model *m, double *vel, const double *Ray3,
                            int i, int j, double dt, double tau, double mask,
                            const double *a, const double *hcol, double *c1,
                            double *tau_bot) {
    int nz = m->nk;
    double dt_Rho0 = dt / RHO_0;
    double sfc_stress = dt_Rho0 * tau * mask;
    double Ray = A3(Ray3, i, j, 1);
    double b_denom_1 = hcol[1] + dt * (Ray + a[1]);
    double b1 = 1.0 / (b_denom_1 + dt * a[2]);
    double d1 = b_denom_1 * b1;
    A3(vel, i, j, 1) = b1 * (hcol[1] * A3(vel, i, j, 1) + sfc_stress);
    for (int k = 2; k <= nz; ++k) {
        Ray = A3(Ray3, i, j, k);
        c1[k] = dt * a[k] * b1;
        b_denom_1 = hcol[k] + dt * (Ray + a[k] * d1);
        b1 = 1.0 / (b_denom_1 + dt * a[k + 1]);
        d1 = b_denom_1 * b1;
        A3(vel, i, j, k) = (hcol[k] * A3(vel, i, j, k) + dt * a[k] * A3(vel, i, j, k - 1)) * b1;
    }
    for (int k = nz - 1; k >= 1; --k)
        A3(vel, i, j, k) = A3(vel, i, j, k) + c1[k + 1] * A3(vel, i, j, k + 1);
    *tau_bot = RHO_0 * A3(vel, i, j, nz) * a[nz + 1];
    for (int k = 1; k <= nz; ++k)
        *tau_bot = *tau_bot + RHO_0 * A3(Ray3, i, j, k) * A3(vel, i, j, k);
}

void oracle_vert_visc(oracle_model *m, double *u, double *v, const double *h,
                      double dt) {
    int is = m->is, ie = m->ie, js = m->js, je = m->je, nz = m->nk;
    double h_neglect = m->Angstrom_H;
    /* columns are independent: with OpenMP each thread has its own column
     * scratch and takes whole rows */
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
    double *a = (double *)malloc(sizeof(double) * (nz + 2));
    double *hc = (double *)malloc(sizeof(double) * (nz + 2));
    double *hvel = (double *)malloc(sizeof(double) * (nz + 2));
    double *z_i = (double *)malloc(sizeof(double) * (nz + 2));
    double *c1 = (double *)malloc(sizeof(double) * (nz + 2));
    /* vert_visc_coef, u-points then v-points */
    OMP_COLS
    for (int j = js; j <= je; ++j)
        for (int i = is - 1; i <= ie; ++i) {
            if (A2(m->mask2dCu, i, j) > 0.0) {
                vv_coef_column(m, u, h, i, j, 1, 0, a, hc, hvel, z_i);
                for (int K = 1; K <= nz + 1; ++K) A3(m->vv_a_u, i, j, K) = a[K];
                for (int k = 1; k <= nz; ++k) A3(m->vv_h_u, i, j, k) = hc[k];
            } else {
                for (int k = 1; k <= nz; ++k) A3(m->vv_h_u, i, j, k) = h_neglect;
                for (int K = 1; K <= nz + 1; ++K) A3(m->vv_a_u, i, j, K) = 0.0;
            }
        }
    OMP_COLS
    for (int j = js - 1; j <= je; ++j)
        for (int i = is; i <= ie; ++i) {
            if (A2(m->mask2dCv, i, j) > 0.0) {
                vv_coef_column(m, v, h, i, j, 0, 1, a, hc, hvel, z_i);
                for (int K = 1; K <= nz + 1; ++K) A3(m->vv_a_v, i, j, K) = a[K];
                for (int k = 1; k <= nz; ++k) A3(m->vv_h_v, i, j, k) = hc[k];
            } else {
                for (int k = 1; k <= nz; ++k) A3(m->vv_h_v, i, j, k) = h_neglect;
                for (int K = 1; K <= nz + 1; ++K) A3(m->vv_a_v, i, j, K) = 0.0;
            }
        }
    /* vert_visc_apply, u-points then v-points */
    OMP_COLS
    for (int j = js; j <= je; ++j)
        for (int i = is - 1; i <= ie; ++i) {
            if (!(A2(m->mask2dCu, i, j) > 0.0)) continue;
            for (int K = 1; K <= nz + 1; ++K) a[K] = A3(m->vv_a_u, i, j, K);
            for (int k = 1; k <= nz; ++k) hc[k] = A3(m->vv_h_u, i, j, k);
            vv_apply_column(m, u, m->Ray_u, i, j, dt, A2(m->taux, i, j),
                            A2(m->mask2dCu, i, j), a, hc, c1, &A2(m->vv_taux_bot, i, j));
        }
    OMP_COLS
    for (int j = js - 1; j <= je; ++j)
        for (int i = is; i <= ie; ++i) {
            if (!(A2(m->mask2dCv, i, j) > 0.0)) continue;
            for (int K = 1; K <= nz + 1; ++K) a[K] = A3(m->vv_a_v, i, j, K);
            for (int k = 1; k <= nz; ++k) hc[k] = A3(m->vv_h_v, i, j, k);
            vv_apply_column(m, v, m->Ray_v, i, j, dt, A2(m->tauy, i, j),
                            A2(m->mask2dCv, i, j), a, hc, c1, &A2(m->vv_tauy_bot, i, j));
        }
    free(a); free(hc); free(hvel); free(z_i); free(c1);
    }
}

/* vert_visc_remnant, mom6_vert_visc_serial.F90:295-387: the fraction of a
 * barotropic acceleration left in each layer after the implicit viscosity of
 * the last oracle_vert_visc call (its a and h_u), with the driver's Rayleigh
 * drag; 1 in masked columns. */
static void alloc_visc_rem_v(oracle_model *m) {
    if (m->visc_rem_v) return;
    size_t n3d = (size_t)N1 * N2 * m->nk;
    m->visc_rem_v = zalloc(n3d);
    for (size_t q = 0; q < n3d; ++q) m->visc_rem_v[q] = 1.0;
}

void oracle_vert_visc_remnant(oracle_model *m, double dt) {
    int is = m->is, ie = m->ie, js = m->js, je = m->je, nz = m->nk;
    alloc_visc_rem_v(m);
    double *c1 = (double *)malloc(sizeof(double) * (nz + 2));
    for (int pass = 0; pass < 2; ++pass) {
        const int u_pts = pass == 0;
        const double *mask = u_pts ? m->mask2dCu : m->mask2dCv;
        const double *a3 = u_pts ? m->vv_a_u : m->vv_a_v, *h3 = u_pts ? m->vv_h_u : m->vv_h_v;
        const double *Ray3 = u_pts ? m->Ray_u : m->Ray_v;
        double *rem = u_pts ? m->visc_rem_u : m->visc_rem_v;
        const int j0 = u_pts ? js : js - 1, i0 = u_pts ? is - 1 : is;
        for (int j = j0; j <= je; ++j)
            for (int i = i0; i <= ie; ++i) {
                if (!(A2(mask, i, j) > 0.0)) {
                    for (int k = 1; k <= nz; ++k) A3(rem, i, j, k) = 1.0;
                    continue;
                }
                double Ray = A3(Ray3, i, j, 1);
                double b_denom_1 = A3(h3, i, j, 1) + dt * (Ray + A3(a3, i, j, 1));
                double b1 = 1.0 / (b_denom_1 + dt * A3(a3, i, j, 2));
                double d1 = b_denom_1 * b1;
                A3(rem, i, j, 1) = b1 * A3(h3, i, j, 1);
                for (int k = 2; k <= nz; ++k) {
                    Ray = A3(Ray3, i, j, k);
                    c1[k] = dt * A3(a3, i, j, k) * b1;
                    b_denom_1 = A3(h3, i, j, k) + dt * (Ray + A3(a3, i, j, k) * d1);
                    b1 = 1.0 / (b_denom_1 + dt * A3(a3, i, j, k + 1));
                    d1 = b_denom_1 * b1;
                    A3(rem, i, j, k) = (A3(h3, i, j, k) + dt * A3(a3, i, j, k) * A3(rem, i, j, k - 1)) * b1;
                }
                for (int k = nz - 1; k >= 1; --k)
                    A3(rem, i, j, k) = A3(rem, i, j, k) + c1[k + 1] * A3(rem, i, j, k + 1);
            }
    }
    free(c1);
}

void oracle_set_remnant(oracle_model *m, int on) {
    m->remnant = on;
    alloc_visc_rem_v(m);
}

/* ------------------------------------------------------------------------ */
/* btstep + update_u/update_v, mom6_barotropic_serial.F90:178-356.          */
/* uhbt(is-1,:), uhbt(ie,:), vhbt(:,js-1), vhbt(:,je) are never written.   */
/* ------------------------------------------------------------------------ */
static void bt_update_u(oracle_model *m, int is, int ie, int js, int je) {
    OMP_FOR
    for (int j = js; j <= je; ++j)
        for (int i = is; i <= ie; ++i)
            A2(m->bt_Cor_u, i, j) =
                (((F4(m->bt_f_4_u, 4, i, j) * A2(m->bt_vbt, i + 1, j)) +
                  (F4(m->bt_f_4_u, 1, i, j) * A2(m->bt_vbt, i, j - 1))) +
                 ((F4(m->bt_f_4_u, 3, i, j) * A2(m->bt_vbt, i, j)) +
                  (F4(m->bt_f_4_u, 2, i, j) * A2(m->bt_vbt, i + 1, j - 1))));
    OMP_FOR
    for (int j = js; j <= je; ++j)
        for (int i = is; i <= ie; ++i)
            A2(m->bt_ubt, i, j) =
                A2(m->bt_rem_u, i, j) *
                (A2(m->bt_ubt, i, j) + m->bt_dtbt * (A2(m->bt_Cor_u, i, j) + A2(m->bt_PFu, i, j)));
}

static void bt_update_v(oracle_model *m, int is, int ie, int js, int je) {
    OMP_FOR
    for (int j = js; j <= je; ++j)
        for (int i = is; i <= ie; ++i)
            A2(m->bt_Cor_v, i, j) =
                -1.0 * (((F4(m->bt_f_4_v, 1, i, j) * A2(m->bt_ubt, i - 1, j)) +
                         (F4(m->bt_f_4_v, 4, i, j) * A2(m->bt_ubt, i, j + 1))) +
                        ((F4(m->bt_f_4_v, 2, i, j) * A2(m->bt_ubt, i, j)) +
                         (F4(m->bt_f_4_v, 3, i, j) * A2(m->bt_ubt, i - 1, j + 1))));
    OMP_FOR
    for (int j = js; j <= je; ++j)
        for (int i = is; i <= ie; ++i)
            A2(m->bt_vbt, i, j) =
                A2(m->bt_rem_v, i, j) *
                (A2(m->bt_vbt, i, j) + m->bt_dtbt * (A2(m->bt_Cor_v, i, j) + A2(m->bt_PFv, i, j)));
}

void oracle_btstep(oracle_model *m, const double *eta_in, const double *ubt_in,
                   const double *vbt_in, double *u_av, double *v_av,
                   double *eta_av) {
    int is = m->is, ie = m->ie, js = m->js, je = m->je;
    double trans_wt1 = 1.0 + m->bt_bebt;
    double trans_wt2 = -m->bt_bebt;
    double inv_nstep = 1.0 / (double)m->nstep;
    double dtbt = m->bt_dtbt;
    /* A subdomain of a decomposed run reaches two points into the halo at a
     * cut: then the substep's values at the owned points need only the halo
     * exchanged before the substep (a point's new eta reads ubt, vbt and eta
     * of the old substep up to two points away).  Without cuts these are the
     * serial ranges. */
    const int xw = 2 * m->cw, xe = 2 * m->ce, xs = 2 * m->cs, xn = 2 * m->cn;
    const int ci0 = is - xw, ci1 = ie + xe, cj0 = js - xs, cj1 = je + xn;
    const int ui1 = ie - 1 + xe, vj1 = je - 1 + xn;
    OMP_FOR
    for (int j = m->jsd; j <= m->jed; ++j)
        for (int i = m->isd; i <= m->ied; ++i) {
            A2(m->bt_eta, i, j) = A2(eta_in, i, j);
            A2(m->bt_ubt, i, j) = A2(ubt_in, i, j);
            A2(m->bt_vbt, i, j) = A2(vbt_in, i, j);
            A2(m->bt_ubt_av, i, j) = 0.0;
            A2(m->bt_vbt_av, i, j) = 0.0;
        }
    for (int n = 1; n <= m->nstep; ++n) {
        if (m->xfn) {
            m->xfn(m->xctx, m->bt_ubt, 1, 1);
            m->xfn(m->xctx, m->bt_vbt, 1, 2);
            m->xfn(m->xctx, m->bt_eta, 1, 0);
        }
        OMP_FOR
        for (int j = cj0; j <= cj1; ++j)
            for (int i = is - 1 - xw; i <= ie + 1 + xe; ++i)
                A2(m->bt_ubt_prev, i, j) = A2(m->bt_ubt, i, j);
        OMP_FOR
        for (int j = js - 1 - xs; j <= je + 1 + xn; ++j)
            for (int i = ci0; i <= ci1; ++i)
                A2(m->bt_vbt_prev, i, j) = A2(m->bt_vbt, i, j);
        OMP_FOR
        for (int j = cj0; j <= cj1; ++j)
            for (int i = ci0; i <= ci1; ++i)
                A2(m->bt_eta_pred, i, j) =
                    A2(m->bt_eta, i, j) +
                    (dtbt * A2(m->IareaT, i, j)) *
                        (((A2(m->bt_Datu, i - 1, j) * A2(m->bt_ubt, i - 1, j)) -
                          (A2(m->bt_Datu, i, j) * A2(m->bt_ubt, i, j))) +
                         ((A2(m->bt_Datv, i, j - 1) * A2(m->bt_vbt, i, j - 1)) -
                          (A2(m->bt_Datv, i, j) * A2(m->bt_vbt, i, j))));
        OMP_FOR
        for (int j = cj0; j <= cj1; ++j)
            for (int i = ci0; i <= ui1; ++i)
                A2(m->bt_PFu, i, j) =
                    ((A2(m->bt_eta_pred, i, j) * A2(m->bt_gtot_E, i, j)) -
                     (A2(m->bt_eta_pred, i + 1, j) * A2(m->bt_gtot_W, i + 1, j))) *
                    m->bt_dgeo_de * A2(m->IdxCu, i, j);
        OMP_FOR
        for (int j = cj0; j <= vj1; ++j)
            for (int i = ci0; i <= ci1; ++i)
                A2(m->bt_PFv, i, j) =
                    ((A2(m->bt_eta_pred, i, j) * A2(m->bt_gtot_N, i, j)) -
                     (A2(m->bt_eta_pred, i, j + 1) * A2(m->bt_gtot_S, i, j + 1))) *
                    m->bt_dgeo_de * A2(m->IdyCv, i, j);
        int v_first = ((n + m->first_direction) % 2) == 1;
        if (v_first) {
            bt_update_v(m, ci0, ci1, cj0, vj1);
            bt_update_u(m, ci0, ui1, cj0, cj1);
        } else {
            bt_update_u(m, ci0, ui1, cj0, cj1);
            bt_update_v(m, ci0, ci1, cj0, vj1);
        }
        /* transport ranges: serial (:263-291) or, with bt_extended, those
         * of btstep_do_step and the CUDA C kernels (:443-452) */
        const int iu0 = xw ? ci0 : (m->bt_extended ? is - 1 : is);
        const int iu1 = xe ? ui1 : (m->bt_extended ? ie : ie - 1);
        const int jv0 = xs ? cj0 : (m->bt_extended ? js - 1 : js);
        const int jv1 = xn ? vj1 : (m->bt_extended ? je : je - 1);
        OMP_FOR
        for (int j = cj0; j <= cj1; ++j)
            for (int i = iu0; i <= iu1; ++i)
                A2(m->bt_uhbt, i, j) =
                    A2(m->bt_Datu, i, j) *
                    (trans_wt1 * A2(m->bt_ubt, i, j) + trans_wt2 * A2(m->bt_ubt_prev, i, j));
        OMP_FOR
        for (int j = jv0; j <= jv1; ++j)
            for (int i = ci0; i <= ci1; ++i)
                A2(m->bt_vhbt, i, j) =
                    A2(m->bt_Datv, i, j) *
                    (trans_wt1 * A2(m->bt_vbt, i, j) + trans_wt2 * A2(m->bt_vbt_prev, i, j));
        OMP_FOR
        for (int j = cj0; j <= cj1; ++j)
            for (int i = ci0; i <= ci1; ++i)
                A2(m->bt_eta, i, j) =
                    A2(m->bt_eta, i, j) -
                    dtbt * A2(m->IareaT, i, j) *
                        ((A2(m->bt_uhbt, i, j) - A2(m->bt_uhbt, i - 1, j)) +
                         (A2(m->bt_vhbt, i, j) - A2(m->bt_vhbt, i, j - 1)));
        OMP_FOR
        for (int j = js; j <= je; ++j)
            for (int i = iu0; i <= iu1; ++i)
                A2(m->bt_ubt_av, i, j) = A2(m->bt_ubt_av, i, j) + A2(m->bt_ubt, i, j) * inv_nstep;
        OMP_FOR
        for (int j = jv0; j <= jv1; ++j)
            for (int i = is; i <= ie; ++i)
                A2(m->bt_vbt_av, i, j) = A2(m->bt_vbt_av, i, j) + A2(m->bt_vbt, i, j) * inv_nstep;
    }
    OMP_FOR
    for (int j = m->jsd; j <= m->jed; ++j)
        for (int i = m->isd; i <= m->ied; ++i) {
            A2(u_av, i, j) = A2(m->bt_ubt_av, i, j);
            A2(v_av, i, j) = A2(m->bt_vbt_av, i, j);
            A2(eta_av, i, j) = A2(m->bt_eta, i, j);
        }
}

/* ------------------------------------------------------------------------ */
/* continuity_PPM, mom6_continuity_serial.F90:100-1294 (zonal only).        */
/* CS: upwind_1st = simple_2nd = vol_CFL = aggress_adjust = .false.,        */
/* monotonic = .false. (never set; the PPM_limit_pos path), better_iter =   */
/* use_visc_rem_max = marginal_faces = .true., tol_eta = 1e-12,             */
/* tol_vel = 3e8, CFL_limit_adjust = 0.5.                                   */
/* ------------------------------------------------------------------------ */

/* PPM_reconstruction_x + PPM_limit_pos for one layer, :1124-1294 */
static void ppm_layer(oracle_model *m, const double *h_in, double *h_W,
                      double *h_E, int k) {
    const double oneSixth = 1.0 / 6.0;
    double h_min = F32(2.0) * m->Angstrom_H;
    int isl = m->is - 1, iel = m->ie + 1, jsl = m->js, jel = m->je;
    double *slp = (double *)malloc(sizeof(double) * (N1 + 2));
    for (int j = jsl; j <= jel; ++j) {
        for (int i = isl - 1; i <= iel + 1; ++i) {
            double s;
            if ((A2(m->mask2dT, i - 1, j) * A2(m->mask2dT, i, j) * A2(m->mask2dT, i + 1, j)) == 0.0) {
                s = 0.0;
            } else {
                double hp = A3(h_in, i + 1, j, k), hm = A3(h_in, i - 1, j, k),
                       hc = A3(h_in, i, j, k);
                s = 0.5 * (hp - hm);
                double dMx = MAX(MAX(hp, hm), hc) - hc;
                double dMn = hc - MIN(MIN(hp, hm), hc);
                s = copysign(1.0, s) * MIN(fabs(s), 2.0 * MIN(dMx, dMn));
            }
            slp[i] = s;
        }
        for (int i = isl; i <= iel; ++i) {
            double hc = A3(h_in, i, j, k);
            double h_im1 = A2(m->mask2dT, i - 1, j) * A3(h_in, i - 1, j, k) +
                           (1.0 - A2(m->mask2dT, i - 1, j)) * hc;
            double h_ip1 = A2(m->mask2dT, i + 1, j) * A3(h_in, i + 1, j, k) +
                           (1.0 - A2(m->mask2dT, i + 1, j)) * hc;
            A3(h_W, i, j, k) = 0.5 * (h_im1 + hc) + oneSixth * (slp[i - 1] - slp[i]);
            A3(h_E, i, j, k) = 0.5 * (h_ip1 + hc) + oneSixth * (slp[i] - slp[i + 1]);
        }
        /* PPM_limit_pos: curv, dh and scale are default real (FP32) */
        for (int i = isl; i <= iel; ++i) {
            double hc = A3(h_in, i, j, k);
            double hL = A3(h_W, i, j, k), hR = A3(h_E, i, j, k);
            float curv = (float)(3.0 * ((hL + hR) - 2.0 * hc));
            if ((double)curv > 0.0) {
                float dh = (float)(hR - hL);
                if (fabsf(dh) < curv) {
                    if (hc <= h_min) {
                        A3(h_W, i, j, k) = hc;
                        A3(h_E, i, j, k) = hc;
                    } else {
                        float c12 = 12.0f * curv;
                        float den = curv * curv + 3.0f * (dh * dh);
                        if ((double)c12 * (hc - h_min) < (double)den) {
                            float scale = (float)(((double)c12 * (hc - h_min)) / (double)den);
                            A3(h_W, i, j, k) = hc + (double)scale * (hL - hc);
                            A3(h_E, i, j, k) = hc + (double)scale * (hR - hc);
                        }
                    }
                }
            }
        }
    }
    free(slp);
}

/* zonal_flux_layer, :516-598, for one row j and layer k */
static void flux_layer(oracle_model *m, const double *u_row, const double *h,
                       const double *h_W, const double *h_E, double *uh,
                       double *duhdu, const double *visc_rem, double dt, int j,
                       int k, const unsigned char *do_I, const double *por) {
    int ish = m->is, ieh = m->ie;
    for (int I = ish - 1; I <= ieh; ++I) {
        if (!do_I[I]) continue;
        int i = I;
        double uI = u_row[I], h_marg;
        double dyp = A2(m->dy_Cu, I, j) * por[I];
        if (uI > 0.0) {
            double CFL = uI * dt * A2(m->IdxT, i, j);
            double hWi = A3(h_W, i, j, k), hEi = A3(h_E, i, j, k);
            double curv_3 = (hWi + hEi) - 2.0 * A3(h, i, j, k);
            uh[I] = dyp * uI * (hEi + CFL * (0.5 * (hWi - hEi) + curv_3 * (CFL - 1.5)));
            h_marg = hEi + CFL * ((hWi - hEi) + 3.0 * curv_3 * (CFL - 1.0));
        } else if (uI < 0.0) {
            double CFL = -(uI * dt * A2(m->IdxT, i + 1, j));
            double hWp = A3(h_W, i + 1, j, k), hEp = A3(h_E, i + 1, j, k);
            double curv_3 = (hWp + hEp) - 2.0 * A3(h, i + 1, j, k);
            uh[I] = dyp * uI * (hWp + CFL * (0.5 * (hEp - hWp) + curv_3 * (CFL - 1.5)));
            h_marg = hWp + CFL * ((hEp - hWp) + 3.0 * curv_3 * (CFL - 1.0));
        } else {
            uh[I] = 0.0;
            h_marg = 0.5 * (A3(h_W, i + 1, j, k) + A3(h_E, i, j, k));
        }
        duhdu[I] = dyp * h_marg * visc_rem[I];
    }
}

typedef struct {
    double *u_row, *uh_row, *por_row, *vr_row; /* length n1+1, index I */
} row_tmp;

/* zonal_flux_adjust, :739-916.  uh_3d != NULL mirrors the present(uh_3d)
 * call from zonal_mass_flux; visc_rem is (n1+1) x nz. */
static void flux_adjust(oracle_model *m, const double *u, const double *h_in,
                        const double *h_W, const double *h_E, const double *uhbt,
                        const double *uh_tot_0, const double *duhdu_tot_0,
                        double *du, const double *du_max_CFL,
                        const double *du_min_CFL, double dt,
                        const double *visc_rem, int j, const unsigned char *do_I_in,
                        double *uh_3d) {
    const int max_itts = 20;
    int ish = m->is, ieh = m->ie, nz = m->nk;
    size_t L = (size_t)N1 + 2;
    double *uh_aux = zalloc(L * (nz + 1)), *duhdu = zalloc(L * (nz + 1));
    double *uh_err = zalloc(L), *uh_err_best = zalloc(L), *u_new = zalloc(L),
           *duhdu_tot = zalloc(L), *du_min = zalloc(L), *du_max = zalloc(L),
           *vr = zalloc(L), *por = zalloc(L);
    unsigned char *do_I = (unsigned char *)calloc(L, 1);
    const double tol_eta_cs = 1.0e-12, tol_vel_cs = 3.0e8;
#define VR(I, k) visc_rem[(size_t)(k) * L + (size_t)(I)]
#define UA(I, k) uh_aux[(size_t)(k) * L + (size_t)(I)]
#define DH(I, k) duhdu[(size_t)(k) * L + (size_t)(I)]
    if (uh_3d)
        for (int k = 1; k <= nz; ++k)
            for (int I = ish - 1; I <= ieh; ++I) UA(I, k) = A3(uh_3d, I, j, k);
    for (int I = ish - 1; I <= ieh; ++I) {
        du[I] = 0.0;
        do_I[I] = do_I_in[I];
        du_max[I] = du_max_CFL[I];
        du_min[I] = du_min_CFL[I];
        uh_err[I] = uh_tot_0[I] - uhbt[I];
        duhdu_tot[I] = duhdu_tot_0[I];
        uh_err_best[I] = fabs(uh_err[I]);
    }
    for (int itt = 1; itt <= max_itts; ++itt) {
        double tol_eta;
        if (itt <= 1) tol_eta = F32(1e-6) * tol_eta_cs;
        else if (itt == 2) tol_eta = F32(1e-4) * tol_eta_cs;
        else if (itt == 3) tol_eta = F32(1e-2) * tol_eta_cs;
        else tol_eta = tol_eta_cs;
        double tol_vel = tol_vel_cs;
        for (int I = ish - 1; I <= ieh; ++I) {
            if (uh_err[I] > 0.0) du_max[I] = du[I];
            else if (uh_err[I] < 0.0) du_min[I] = du[I];
            else do_I[I] = 0;
        }
        int domore = 0;
        for (int I = ish - 1; I <= ieh; ++I) {
            if (!do_I[I]) continue;
            double ae = fabs(uh_err[I]);
            if ((dt * MIN(A2(m->IareaT, I, j), A2(m->IareaT, I + 1, j)) * ae > tol_eta) ||
                ((ae > tol_vel * duhdu_tot[I]) || (ae > uh_err_best[I]))) {
                double ddu = -(uh_err[I] / duhdu_tot[I]);
                double du_prev = du[I];
                du[I] = du[I] + ddu;
                if (fabs(ddu) < F32(1.0e-15) * fabs(du[I])) {
                    do_I[I] = 0;
                } else if (ddu > 0.0) {
                    if (du[I] >= du_max[I]) {
                        du[I] = 0.5 * (du_prev + du_max[I]);
                        if (du_max[I] - du_prev < F32(1.0e-15) * fabs(du[I])) do_I[I] = 0;
                    }
                } else {
                    if (du[I] <= du_min[I]) {
                        du[I] = 0.5 * (du_prev + du_min[I]);
                        if (du_prev - du_min[I] < F32(1.0e-15) * fabs(du[I])) do_I[I] = 0;
                    }
                }
                if (do_I[I]) domore = 1;
            } else {
                do_I[I] = 0;
            }
        }
        if (!domore) break;
        if ((itt < max_itts) || uh_3d) {
            for (int k = 1; k <= nz; ++k) {
                for (int I = ish - 1; I <= ieh; ++I) {
                    u_new[I] = A3(u, I, j, k) + du[I] * VR(I, k);
                    vr[I] = VR(I, k);
                    por[I] = A3(m->por_face_areaU, I, j, k);
                }
                double *uhk = &UA(0, k), *dhk = &DH(0, k);
                flux_layer(m, u_new, h_in, h_W, h_E, uhk, dhk, vr, dt, j, k, do_I, por);
            }
        }
        if (itt < max_itts) {
            for (int I = ish - 1; I <= ieh; ++I) {
                uh_err[I] = -uhbt[I];
                duhdu_tot[I] = 0.0;
            }
            for (int k = 1; k <= nz; ++k)
                for (int I = ish - 1; I <= ieh; ++I) {
                    uh_err[I] = uh_err[I] + UA(I, k);
                    duhdu_tot[I] = duhdu_tot[I] + DH(I, k);
                }
            for (int I = ish - 1; I <= ieh; ++I)
                uh_err_best[I] = MIN(uh_err_best[I], fabs(uh_err[I]));
        }
    }
    if (uh_3d)
        for (int k = 1; k <= nz; ++k)
            for (int I = ish - 1; I <= ieh; ++I) A3(uh_3d, I, j, k) = UA(I, k);
#undef UA
#undef DH
    free(uh_aux); free(duhdu); free(uh_err); free(uh_err_best); free(u_new);
    free(duhdu_tot); free(du_min); free(du_max); free(vr); free(por); free(do_I);
}

/* set_zonal_BT_cont, :920-1121 */
static void set_bt_cont(oracle_model *m, const double *u, const double *h_in,
                        const double *h_W, const double *h_E,
                        const double *uh_tot_0, const double *duhdu_tot_0,
                        const double *du_max_CFL, const double *du_min_CFL,
                        double dt, const double *visc_rem,
                        const double *visc_rem_max, int j,
                        const unsigned char *do_I) {
    int ish = m->is, ieh = m->ie, nz = m->nk;
    size_t L = (size_t)N1 + 2;
    double *du0 = zalloc(L), *duL = zalloc(L), *duR = zalloc(L), *zeros = zalloc(L),
           *du_CFL = zalloc(L), *u_L = zalloc(L), *u_R = zalloc(L), *u_0 = zalloc(L),
           *duhdu_L = zalloc(L), *duhdu_R = zalloc(L), *duhdu_0 = zalloc(L),
           *uh_L = zalloc(L), *uh_R = zalloc(L), *uh_0 = zalloc(L),
           *FAmt_L = zalloc(L), *FAmt_R = zalloc(L), *FAmt_0 = zalloc(L),
           *uhtot_L = zalloc(L), *uhtot_R = zalloc(L), *vr = zalloc(L), *por = zalloc(L);
    double Idt = 1.0 / dt;
    double min_visc_rem = F32(0.1);
    double CFL_min = F32(1e-6);
    flux_adjust(m, u, h_in, h_W, h_E, zeros, uh_tot_0, duhdu_tot_0, du0,
                du_max_CFL, du_min_CFL, dt, visc_rem, j, do_I, NULL);
    int domore = 0;
    for (int I = ish - 1; I <= ieh; ++I) {
        if (do_I[I]) domore = 1;
        du_CFL[I] = (CFL_min * Idt) * A2(m->dxCu, I, j);
        duR[I] = MIN(0.0, du0[I] - du_CFL[I]);
        duL[I] = MAX(0.0, du0[I] + du_CFL[I]);
    }
    if (!domore) {
        for (int I = ish - 1; I <= ieh; ++I) {
            A2(m->FA_u_W0, I, j) = 0.0; A2(m->FA_u_WW, I, j) = 0.0;
            A2(m->FA_u_E0, I, j) = 0.0; A2(m->FA_u_EE, I, j) = 0.0;
            A2(m->uBT_WW, I, j) = 0.0; A2(m->uBT_EE, I, j) = 0.0;
        }
        goto done;
    }
    for (int k = 1; k <= nz; ++k)
        for (int I = ish - 1; I <= ieh; ++I) {
            if (!do_I[I]) continue;
            double vrk = VR(I, k);
            double visc_rem_lim = MAX(vrk, min_visc_rem * visc_rem_max[I]);
            if (visc_rem_lim > 0.0) {
                double uk = A3(u, I, j, k);
                if (uk + duR[I] * visc_rem_lim > -(du_CFL[I] * vrk))
                    duR[I] = -(uk + du_CFL[I] * vrk) / visc_rem_lim;
                if (uk + duL[I] * visc_rem_lim < du_CFL[I] * vrk)
                    duL[I] = -(uk - du_CFL[I] * vrk) / visc_rem_lim;
            }
        }
    for (int k = 1; k <= nz; ++k) {
        for (int I = ish - 1; I <= ieh; ++I) {
            vr[I] = VR(I, k);
            por[I] = A3(m->por_face_areaU, I, j, k);
            if (do_I[I]) {
                u_L[I] = A3(u, I, j, k) + duL[I] * vr[I];
                u_R[I] = A3(u, I, j, k) + duR[I] * vr[I];
                u_0[I] = A3(u, I, j, k) + du0[I] * vr[I];
            }
        }
        flux_layer(m, u_0, h_in, h_W, h_E, uh_0, duhdu_0, vr, dt, j, k, do_I, por);
        flux_layer(m, u_L, h_in, h_W, h_E, uh_L, duhdu_L, vr, dt, j, k, do_I, por);
        flux_layer(m, u_R, h_in, h_W, h_E, uh_R, duhdu_R, vr, dt, j, k, do_I, por);
        for (int I = ish - 1; I <= ieh; ++I) {
            if (!do_I[I]) continue;
            FAmt_0[I] = FAmt_0[I] + duhdu_0[I];
            FAmt_L[I] = FAmt_L[I] + duhdu_L[I];
            FAmt_R[I] = FAmt_R[I] + duhdu_R[I];
            uhtot_L[I] = uhtot_L[I] + uh_L[I];
            uhtot_R[I] = uhtot_R[I] + uh_R[I];
        }
    }
    for (int I = ish - 1; I <= ieh; ++I) {
        if (do_I[I]) {
            double FA_0 = FAmt_0[I], FA_avg = FAmt_0[I];
            if ((duL[I] - du0[I]) != 0.0) FA_avg = uhtot_L[I] / (duL[I] - du0[I]);
            if (FA_avg > MAX(FA_0, FAmt_L[I])) FA_avg = MAX(FA_0, FAmt_L[I]);
            else if (FA_avg < MIN(FA_0, FAmt_L[I])) FA_0 = FA_avg;
            A2(m->FA_u_W0, I, j) = FA_0;
            A2(m->FA_u_WW, I, j) = FAmt_L[I];
            if (fabs(FA_0 - FAmt_L[I]) <= F32(1e-12) * FA_0)
                A2(m->uBT_WW, I, j) = 0.0;
            else
                A2(m->uBT_WW, I, j) = (1.5 * (duL[I] - du0[I])) *
                                      ((FAmt_L[I] - FA_avg) / (FAmt_L[I] - FA_0));
            FA_0 = FAmt_0[I]; FA_avg = FAmt_0[I];
            if ((duR[I] - du0[I]) != 0.0) FA_avg = uhtot_R[I] / (duR[I] - du0[I]);
            if (FA_avg > MAX(FA_0, FAmt_R[I])) FA_avg = MAX(FA_0, FAmt_R[I]);
            else if (FA_avg < MIN(FA_0, FAmt_R[I])) FA_0 = FA_avg;
            A2(m->FA_u_E0, I, j) = FA_0;
            A2(m->FA_u_EE, I, j) = FAmt_R[I];
            if (fabs(FAmt_R[I] - FA_0) <= F32(1e-12) * FA_0)
                A2(m->uBT_EE, I, j) = 0.0;
            else
                A2(m->uBT_EE, I, j) = (1.5 * (duR[I] - du0[I])) *
                                      ((FAmt_R[I] - FA_avg) / (FAmt_R[I] - FA_0));
        } else {
            A2(m->FA_u_W0, I, j) = 0.0; A2(m->FA_u_WW, I, j) = 0.0;
            A2(m->FA_u_E0, I, j) = 0.0; A2(m->FA_u_EE, I, j) = 0.0;
            A2(m->uBT_WW, I, j) = 0.0; A2(m->uBT_EE, I, j) = 0.0;
        }
    }
done:
    free(du0); free(duL); free(duR); free(zeros); free(du_CFL); free(u_L);
    free(u_R); free(u_0); free(duhdu_L); free(duhdu_R); free(duhdu_0);
    free(uh_L); free(uh_R); free(uh_0); free(FAmt_L); free(FAmt_R); free(FAmt_0);
    free(uhtot_L); free(uhtot_R); free(vr); free(por);
}
#undef VR

/* zonal_mass_flux for one row j, :218-499 */
static void mass_flux_row(oracle_model *m, const double *u, const double *h_in,
                          double *uh, double dt, int j) {
    int ish = m->is, ieh = m->ie, nz = m->nk;
    size_t L = (size_t)N1 + 2;
    double *duhdu = zalloc(L * (nz + 1)), *visc_rem = zalloc(L * (nz + 1));
    double *du = zalloc(L), *du_min_CFL = zalloc(L), *du_max_CFL = zalloc(L),
           *duhdu_tot_0 = zalloc(L), *uh_tot_0 = zalloc(L), *visc_rem_max = zalloc(L),
           *urow = zalloc(L), *uhrow = zalloc(L), *vr = zalloc(L), *por = zalloc(L);
    unsigned char *do_I = (unsigned char *)calloc(L, 1);
    double CFL_dt = 0.5 / dt;
    double *h_W = m->hW, *h_E = m->hE;
#define VRk(I, k) visc_rem[(size_t)(k) * L + (size_t)(I)]
#define DHk(I, k) duhdu[(size_t)(k) * L + (size_t)(I)]
    for (int I = ish - 1; I <= ieh; ++I) do_I[I] = 1;
    for (int k = 1; k <= nz; ++k) {
        for (int I = ish - 1; I <= ieh; ++I) {
            VRk(I, k) = A3(m->visc_rem_u, I, j, k);
            urow[I] = A3(u, I, j, k);
            vr[I] = VRk(I, k);
            por[I] = A3(m->por_face_areaU, I, j, k);
        }
        flux_layer(m, urow, h_in, h_W, h_E, uhrow, &DHk(0, k), vr, dt, j, k, do_I, por);
        for (int I = ish - 1; I <= ieh; ++I) A3(uh, I, j, k) = uhrow[I];
    }
    /* use_visc_rem and use_visc_rem_max */
    for (int I = 0; I < (int)L; ++I) visc_rem_max[I] = 0.0;
    for (int k = 1; k <= nz; ++k)
        for (int I = ish - 1; I <= ieh; ++I)
            visc_rem_max[I] = MAX(visc_rem_max[I], VRk(I, k));
    for (int I = ish - 1; I <= ieh; ++I) {
        double I_vrm = 0.0;
        if (visc_rem_max[I] > 0.0) I_vrm = 1.0 / visc_rem_max[I];
        double dx_W = A2(m->dxT, I, j), dx_E = A2(m->dxT, I + 1, j);
        du_max_CFL[I] = 2.0 * (CFL_dt * dx_W) * I_vrm;
        du_min_CFL[I] = -(2.0 * (CFL_dt * dx_E) * I_vrm);
        uh_tot_0[I] = 0.0;
        duhdu_tot_0[I] = 0.0;
    }
    for (int k = 1; k <= nz; ++k)
        for (int I = ish - 1; I <= ieh; ++I) {
            duhdu_tot_0[I] = duhdu_tot_0[I] + DHk(I, k);
            uh_tot_0[I] = uh_tot_0[I] + A3(uh, I, j, k);
        }
    for (int k = 1; k <= nz; ++k)
        for (int I = ish - 1; I <= ieh; ++I) {
            double dx_W = A2(m->dxT, I, j), dx_E = A2(m->dxT, I + 1, j);
            double uk = A3(u, I, j, k), vrk = VRk(I, k), mk = A2(m->mask2dCu, I, j);
            if (du_max_CFL[I] * vrk > dx_W * CFL_dt - uk * mk)
                du_max_CFL[I] = (dx_W * CFL_dt - uk) / vrk;
            if (du_min_CFL[I] * vrk < -(dx_E * CFL_dt) - uk * mk)
                du_min_CFL[I] = -(dx_E * CFL_dt + uk) / vrk;
        }
    for (int I = ish - 1; I <= ieh; ++I) {
        du_max_CFL[I] = MAX(du_max_CFL[I], 0.0);
        du_min_CFL[I] = MIN(du_min_CFL[I], 0.0);
    }
    /* uhbt is present (all zero), u_cor and du_cor are present */
    double *uhbt_row = zalloc(L);
    for (int I = ish - 1; I <= ieh; ++I) uhbt_row[I] = A2(m->c_uhbt, I, j);
    flux_adjust(m, u, h_in, h_W, h_E, uhbt_row, uh_tot_0, duhdu_tot_0, du,
                du_max_CFL, du_min_CFL, dt, visc_rem, j, do_I, uh);
    for (int k = 1; k <= nz; ++k)
        for (int I = ish - 1; I <= ieh; ++I)
            A3(m->u_cor, I, j, k) = A3(u, I, j, k) + du[I] * VRk(I, k);
    for (int I = ish - 1; I <= ieh; ++I) A2(m->du_cor, I, j) = du[I];
    set_bt_cont(m, u, h_in, h_W, h_E, uh_tot_0, duhdu_tot_0, du_max_CFL,
                du_min_CFL, dt, visc_rem, visc_rem_max, j, do_I);
#undef VRk
#undef DHk
    free(uhbt_row);
    free(duhdu); free(visc_rem); free(du); free(du_min_CFL); free(du_max_CFL);
    free(duhdu_tot_0); free(uh_tot_0); free(visc_rem_max); free(urow);
    free(uhrow); free(vr); free(por); free(do_I);
}

/* zonal_flux_thickness, :602-735 (marginal faces, visc_rem_u present) */
static void flux_thickness(oracle_model *m, const double *u, const double *h,
                           double dt) {
    double *h_W = m->hW, *h_E = m->hE, *h_u = m->BT_h_u;
    for (int k = 1; k <= m->nk; ++k)
        for (int j = m->js; j <= m->je; ++j)
            for (int I = m->is - 1; I <= m->ie; ++I) {
                int i = I;
                double uk = A3(u, I, j, k), h_marg;
                if (uk > 0.0) {
                    double CFL = uk * dt * A2(m->IdxT, i, j);
                    double curv_3 = (A3(h_W, i, j, k) + A3(h_E, i, j, k)) - 2.0 * A3(h, i, j, k);
                    h_marg = A3(h_E, i, j, k) +
                             CFL * ((A3(h_W, i, j, k) - A3(h_E, i, j, k)) + 3.0 * curv_3 * (CFL - 1.0));
                } else if (uk < 0.0) {
                    double CFL = -(uk * dt * A2(m->IdxT, i + 1, j));
                    double curv_3 = (A3(h_W, i + 1, j, k) + A3(h_E, i + 1, j, k)) -
                                    2.0 * A3(h, i + 1, j, k);
                    h_marg = A3(h_W, i + 1, j, k) +
                             CFL * ((A3(h_E, i + 1, j, k) - A3(h_W, i + 1, j, k)) +
                                    3.0 * curv_3 * (CFL - 1.0));
                } else {
                    h_marg = 0.5 * (A3(h_W, i + 1, j, k) + A3(h_E, i, j, k));
                }
                A3(h_u, I, j, k) = h_marg;
            }
    for (int k = 1; k <= m->nk; ++k)
        for (int j = m->js; j <= m->je; ++j)
            for (int I = m->is - 1; I <= m->ie; ++I)
                A3(h_u, I, j, k) =
                    A3(h_u, I, j, k) * (A3(m->visc_rem_u, I, j, k) * A3(m->por_face_areaU, I, j, k));
}

void oracle_continuity(oracle_model *m, const double *u, const double *hin,
                       double *h, double *uh, double dt) {
    OMP_FOR
    for (int k = 1; k <= m->nk; ++k) ppm_layer(m, hin, m->hW, m->hE, k);
    OMP_FOR
    for (int j = m->js; j <= m->je; ++j) mass_flux_row(m, u, hin, uh, dt, j);
    flux_thickness(m, m->u_cor, hin, dt);
    /* continuity_zonal_convergence with hin, h_min = 0, :148-176 */
    OMP_FOR
    for (int k = 1; k <= m->nk; ++k)
        for (int j = m->js; j <= m->je; ++j)
            for (int i = m->is; i <= m->ie; ++i)
                A3(h, i, j, k) = MAX(A3(hin, i, j, k) - dt * A2(m->IareaT, i, j) *
                                                           (A3(uh, i, j, k) - A3(uh, i - 1, j, k)),
                                     0.0);
}

/* ------------------------------------------------------------------------ */
/* meridional continuity: MOM6's continuity_PPM follows the zonal pass with   */
/* the meridional one; the mini-app's module is zonal only                    */
/* (mom6_continuity_serial.F90:143).  The pass is the zonal restatement above */
/* applied to the transposed problem and transposed back.                     */
/* ------------------------------------------------------------------------ */
enum { MT_IAREAT, MT_IDXT, MT_DXCU, MT_DXT, MT_DYCU, MT_MASKCU, MT_MASKT, MT_HW, MT_HE,
       MT_UHBT, MT_DUCOR, MT_UCOR, MT_POR, MT_VISC, MT_FAW0, MT_FAWW, MT_FAE0, MT_FAEE,
       MT_UBTWW, MT_UBTEE, MT_BTHU, MT_COUNT };

static void transpose_plane(const double *a, double *at, int n1, int n2) {
    for (int j = 1; j <= n2; ++j)
        for (int i = 1; i <= n1; ++i)
            at[(size_t)(i - 1) * n2 + (j - 1)] = a[(size_t)(j - 1) * n1 + (i - 1)];
}

static void transpose_field(const double *a, double *at, int n1, int n2, int nk) {
    for (int k = 0; k < nk; ++k)
        transpose_plane(a + (size_t)k * n1 * n2, at + (size_t)k * n1 * n2, n1, n2);
}

int oracle_set_coriolis_scheme(oracle_model *m, int scheme) {
    if (scheme < 1 || scheme > 3) return -1;
    m->cor_scheme = scheme;
    return 0;
}

void oracle_set_merid(oracle_model *m, int on) {
    size_t n2d = (size_t)N1 * N2, n3d = n2d * m->nk;
    m->merid = on;
    if (!on || m->hz) return;
    m->hz = zalloc(n3d); m->BT_h_v = zalloc(n3d);
    m->FA_v_S0 = zalloc(n2d); m->FA_v_SS = zalloc(n2d); m->FA_v_N0 = zalloc(n2d);
    m->FA_v_NN = zalloc(n2d); m->vBT_SS = zalloc(n2d); m->vBT_NN = zalloc(n2d);
    m->dv_cor = zalloc(n2d);
    const int is3[MT_COUNT] = {0, 0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 1, 1, 1, 0, 0, 0, 0, 0, 0, 1};
    for (int q = 0; q < MT_COUNT; ++q) m->mt[q] = zalloc(is3[q] ? n3d : n2d);
    for (size_t q = 0; q < n3d; ++q) { m->mt[MT_POR][q] = 1.0; m->mt[MT_VISC][q] = 1.0; }
    /* the y metrics in the places of the x metrics, transposed */
    transpose_plane(m->IareaT, m->mt[MT_IAREAT], N1, N2);
    transpose_plane(m->IdyT, m->mt[MT_IDXT], N1, N2);
    transpose_plane(m->dyCv, m->mt[MT_DXCU], N1, N2);
    transpose_plane(m->dyT, m->mt[MT_DXT], N1, N2);
    transpose_plane(m->dxCv, m->mt[MT_DYCU], N1, N2);
    transpose_plane(m->mask2dCv, m->mt[MT_MASKCU], N1, N2);
    transpose_plane(m->mask2dT, m->mt[MT_MASKT], N1, N2);
}

void oracle_continuity_merid(oracle_model *m, const double *v, const double *hin,
                             double *h, double *vh, double dt) {
    oracle_set_merid(m, 1);
    const int n1 = N1, n2 = N2, nk = m->nk;
    const size_t n3d = (size_t)n1 * n2 * nk;
    oracle_model T = *m;   /* the transposed problem */
    T.n1 = n2; T.n2 = n1; T.ni = m->nj; T.nj = m->ni;
    T.is = m->js; T.ie = m->je; T.js = m->is; T.je = m->ie;
    T.isd = m->jsd; T.ied = m->jed; T.jsd = m->isd; T.jed = m->ied;
    T.IareaT = m->mt[MT_IAREAT]; T.IdxT = m->mt[MT_IDXT]; T.dxCu = m->mt[MT_DXCU];
    T.dxT = m->mt[MT_DXT]; T.dy_Cu = m->mt[MT_DYCU]; T.mask2dCu = m->mt[MT_MASKCU];
    T.mask2dT = m->mt[MT_MASKT]; T.hW = m->mt[MT_HW]; T.hE = m->mt[MT_HE];
    T.c_uhbt = m->mt[MT_UHBT]; T.du_cor = m->mt[MT_DUCOR]; T.u_cor = m->mt[MT_UCOR];
    T.por_face_areaU = m->mt[MT_POR]; T.visc_rem_u = m->mt[MT_VISC];
    T.FA_u_W0 = m->mt[MT_FAW0]; T.FA_u_WW = m->mt[MT_FAWW]; T.FA_u_E0 = m->mt[MT_FAE0];
    T.FA_u_EE = m->mt[MT_FAEE]; T.uBT_WW = m->mt[MT_UBTWW]; T.uBT_EE = m->mt[MT_UBTEE];
    T.BT_h_u = m->mt[MT_BTHU];
    if (m->visc_rem_v) transpose_field(m->visc_rem_v, m->mt[MT_VISC], n1, n2, nk);
    double *vT = (double *)malloc(n3d * sizeof(double)), *hinT = (double *)malloc(n3d * sizeof(double));
    double *hT = (double *)malloc(n3d * sizeof(double)), *vhT = (double *)calloc(n3d, sizeof(double));
    transpose_field(v, vT, n1, n2, nk);
    transpose_field(hin, hinT, n1, n2, nk);
    transpose_field(h, hT, n1, n2, nk);
    oracle_continuity(&T, vT, hinT, hT, vhT, dt);
    /* back: cells [is, ie] x [js, je], faces [is, ie] x [js-1, je] */
    for (int k = 1; k <= nk; ++k)
        for (int j = m->js - 1; j <= m->je; ++j)
            for (int i = m->is; i <= m->ie; ++i) {
                size_t o = (size_t)(k - 1) * n1 * n2 + (size_t)(j - 1) * n1 + (i - 1);
                size_t t = (size_t)(k - 1) * n1 * n2 + (size_t)(i - 1) * n2 + (j - 1);
                if (j >= m->js) h[o] = hT[t];
                vh[o] = vhT[t];
                m->BT_h_v[o] = m->mt[MT_BTHU][t];
            }
    for (int j = m->js - 1; j <= m->je; ++j)
        for (int i = m->is; i <= m->ie; ++i) {
            size_t o = (size_t)(j - 1) * n1 + (i - 1), t = (size_t)(i - 1) * n2 + (j - 1);
            m->FA_v_S0[o] = m->mt[MT_FAW0][t]; m->FA_v_SS[o] = m->mt[MT_FAWW][t];
            m->FA_v_N0[o] = m->mt[MT_FAE0][t]; m->FA_v_NN[o] = m->mt[MT_FAEE][t];
            m->vBT_SS[o] = m->mt[MT_UBTWW][t]; m->vBT_NN[o] = m->mt[MT_UBTEE][t];
            m->dv_cor[o] = m->mt[MT_DUCOR][t];
        }
    free(vT); free(hinT); free(hT); free(vhT);
}

/* continuity of the step: zonal, or zonal then meridional through hz */
static void step_continuity(oracle_model *m, const double *u, const double *v,
                            const double *hin, double *h, double dt) {
    if (!m->merid) {
        oracle_continuity(m, u, hin, h, m->uh, dt);
        return;
    }
    memcpy(m->hz, hin, (size_t)N1 * N2 * m->nk * sizeof(double));
    oracle_continuity(m, u, hin, m->hz, m->uh, dt);
    if (m->cfg.bc_fill) oracle_halo_fill(m, m->hz, m->nk, 0);
    oracle_continuity_merid(m, v, m->hz, h, m->vh, dt);
}

/* ------------------------------------------------------------------------ */
/* the split RK2 iteration, rk2_serial_driver.F90:218-399                   */
/* ------------------------------------------------------------------------ */
static void vel_update(oracle_model *m, const double *ubase, const double *vbase,
                       double *uout, double *vout, double coef) {
    for (int k = 1; k <= m->nk; ++k) {
        OMP_FOR
        for (int j = m->js; j <= m->je; ++j)
            for (int i = m->is; i <= m->ie - 1 + m->ce; ++i)
                A3(uout, i, j, k) = A3(ubase, i, j, k) +
                                    coef * (A3(m->CAu, i, j, k) + A3(m->diffu, i, j, k));
        OMP_FOR
        for (int j = m->js; j <= m->je - 1 + m->cn; ++j)
            for (int i = m->is; i <= m->ie; ++i)
                A3(vout, i, j, k) = A3(vbase, i, j, k) +
                                    coef * (A3(m->CAv, i, j, k) + A3(m->diffv, i, j, k));
    }
}

/* ------------------------------------------------------------------------ */
/* driver diagnostics: post_product_sum_u/v (mom6_diag.F90:274-334) after the */
/* predictor continuity (rk2_serial_driver.F90:299-304), compute_and_post_KE  */
/* and compute_and_post_mass (:664-728) after the last iteration (:385-391).  */
/* ------------------------------------------------------------------------ */
void oracle_diag_enable(oracle_model *m, int on) {
    size_t n2d = (size_t)N1 * N2, n3d = n2d * m->nk;
    m->diag_on = on;
    if (on && !m->diag_work) {
        m->diag_work = zalloc(n2d); m->diag_usum = zalloc(n2d); m->diag_vsum = zalloc(n2d);
        m->diag_KE = zalloc(n3d); m->diag_mass = zalloc(n2d);
    }
}

/* work_2d(i, j) = sum_k a(i, j, k) * b(i, j, k) over [is, ie - iu] x [js, je - jv] */
static void diag_product_sum(oracle_model *m, const double *a, const double *b, int iu, int jv) {
    for (int j = m->js; j <= m->je - jv; ++j)
        for (int i = m->is; i <= m->ie - iu; ++i) A2(m->diag_work, i, j) = 0.0;
    for (int k = 1; k <= m->nk; ++k)
        for (int j = m->js; j <= m->je - jv; ++j)
            for (int i = m->is; i <= m->ie - iu; ++i)
                A2(m->diag_work, i, j) = A2(m->diag_work, i, j) + A3(a, i, j, k) * A3(b, i, j, k);
}

static void diag_end_of_call(oracle_model *m) {
    for (int k = 1; k <= m->nk; ++k)
        for (int j = m->js; j <= m->je; ++j)
            for (int i = m->is; i <= m->ie; ++i) {
                double u0 = A3(m->u, i, j, k), u1 = A3(m->u, i - 1, j, k);
                double v0 = A3(m->v, i, j, k), v1 = A3(m->v, i, j - 1, k);
                A3(m->diag_KE, i, j, k) = 0.5 * (0.5 * (u0 * u0 + u1 * u1) + 0.5 * (v0 * v0 + v1 * v1));
            }
    memset(m->diag_mass, 0, (size_t)N1 * N2 * sizeof(double));
    for (int k = 1; k <= m->nk; ++k)
        for (int j = m->js; j <= m->je; ++j)
            for (int i = m->is; i <= m->ie; ++i)
                A2(m->diag_mass, i, j) = A2(m->diag_mass, i, j) + A3(m->h, i, j, k);
}

/* which: 0 the field posted by the last diffu_sum post, 1 diffv_sum, 2 KE (3-D),
 * 3 mass; the computational domain of each is what the GPU posts */
int oracle_diag_get(const oracle_model *m, int which, double *out) {
    size_t n2d = (size_t)N1 * N2;
    if (!m->diag_on) return -1;
    switch (which) {
    case 0: memcpy(out, m->diag_usum, n2d * sizeof(double)); return 0;
    case 1: memcpy(out, m->diag_vsum, n2d * sizeof(double)); return 0;
    case 2: memcpy(out, m->diag_KE, n2d * m->nk * sizeof(double)); return 0;
    case 3: memcpy(out, m->diag_mass, n2d * sizeof(double)); return 0;
    default: return -1;
    }
}

static void one_step(oracle_model *m) {
    size_t n3d = (size_t)N1 * N2 * m->nk;
    double dt = m->dt;
    memcpy(m->h, m->h0, n3d * sizeof(double));
    /* PREDICTOR */
    oracle_compute_transports(m, m->u, m->v, m->h, m->uh, m->vh);
    oracle_hor_visc(m, m->u, m->v, m->h, m->diffu, m->diffv);
    oracle_coriolis(m, m->u, m->v, m->h, m->uh, m->vh, m->CAu, m->CAv);
    vel_update(m, m->u, m->v, m->up, m->vp, dt);
    oracle_vert_visc(m, m->up, m->vp, m->h, dt);
    if (m->remnant) oracle_vert_visc_remnant(m, dt);
    oracle_btstep(m, m->eta, m->ubt, m->vbt, m->ubt_av, m->vbt_av, m->eta_av);
    if (m->xfn) {   /* rk2_mpi_cuda_c_driver.F90:409-412 */
        m->xfn(m->xctx, m->up, m->nk, 1);
        m->xfn(m->xctx, m->vp, m->nk, 2);
    }
    step_continuity(m, m->up, m->vp, m->h0, m->h, dt);
    if (m->xfn) m->xfn(m->xctx, m->h, m->nk, 0);
    if (m->diag_on) {
        size_t n2d = (size_t)N1 * N2;
        diag_product_sum(m, m->diffu, m->h, 1, 0);
        memcpy(m->diag_usum, m->diag_work, n2d * sizeof(double));
        diag_product_sum(m, m->diffv, m->h, 0, 1);
        memcpy(m->diag_vsum, m->diag_work, n2d * sizeof(double));
    }
    if (m->cfg.bc_fill) {
        oracle_halo_fill(m, m->h, m->nk, 0);
        oracle_halo_fill(m, m->up, m->nk, 1);
        oracle_halo_fill(m, m->vp, m->nk, 2);
        oracle_halo_fill(m, m->eta_av, 1, 0);
        oracle_halo_fill(m, m->ubt_av, 1, 1);
        oracle_halo_fill(m, m->vbt_av, 1, 2);
    }
    /* CORRECTOR */
    oracle_compute_transports(m, m->up, m->vp, m->h, m->uh, m->vh);
    oracle_hor_visc(m, m->up, m->vp, m->h, m->diffu, m->diffv);
    oracle_coriolis(m, m->up, m->vp, m->h, m->uh, m->vh, m->CAu, m->CAv);
    vel_update(m, m->u, m->v, m->u, m->v, 0.5 * dt);
    oracle_vert_visc(m, m->u, m->v, m->h, 0.5 * dt);
    if (m->remnant) oracle_vert_visc_remnant(m, 0.5 * dt);
    oracle_btstep(m, m->eta_av, m->ubt_av, m->vbt_av, m->ubt_av, m->vbt_av, m->eta);
    if (m->xfn) {
        m->xfn(m->xctx, m->u, m->nk, 1);
        m->xfn(m->xctx, m->v, m->nk, 2);
    }
    /* htmp <- h over the data domain; the reference loops i=isd,jed
     * (rk2_serial_driver.F90:375), bounded here by ied as the CUDA C driver
     * does (rk2_cuda_c_driver.F90:471). */
    memcpy(m->htmp, m->h, n3d * sizeof(double));
    step_continuity(m, m->u, m->v, m->htmp, m->h, 0.5 * dt);
    if (m->cfg.bc_fill) {
        oracle_halo_fill(m, m->h, m->nk, 0);
        oracle_halo_fill(m, m->u, m->nk, 1);
        oracle_halo_fill(m, m->v, m->nk, 2);
        oracle_halo_fill(m, m->eta, 1, 0);
    }
}

void oracle_step(oracle_model *m, int nsteps) {
    for (int s = 0; s < nsteps; ++s) one_step(m);
    if (m->diag_on && nsteps > 0) diag_end_of_call(m);
}

/* ------------------------------------------------------------------------ */
/* field access and verification                                            */
/* ------------------------------------------------------------------------ */
static double *field_ptr(const oracle_model *m, int f, int *is3d) {
    *is3d = 1;
    switch (f) {
    case OR_F_U: return m->u;
    case OR_F_V: return m->v;
    case OR_F_H: return m->h;
    case OR_F_H0: return m->h0;
    case OR_F_UH: return m->uh;
    case OR_F_VH: return m->vh;
    case OR_F_UP: return m->up;
    case OR_F_VP: return m->vp;
    case OR_F_HU_BT: return m->BT_h_u;
    case OR_F_RAY_U: return m->Ray_u;
    case OR_F_RAY_V: return m->Ray_v;
    case OR_F_CAU: return m->CAu;
    case OR_F_CAV: return m->CAv;
    case OR_F_DIFFU: return m->diffu;
    case OR_F_DIFFV: return m->diffv;
    case OR_F_HV_BT: return m->BT_h_v;
    case OR_F_VISC_REM_U: return m->visc_rem_u;
    case OR_F_VISC_REM_V: return m->visc_rem_v;
    default: break;
    }
    *is3d = 0;
    switch (f) {
    case OR_F_ETA: return m->eta;
    case OR_F_UBT: return m->ubt;
    case OR_F_VBT: return m->vbt;
    case OR_F_UBT_AV: return m->ubt_av;
    case OR_F_VBT_AV: return m->vbt_av;
    case OR_F_ETA_AV: return m->eta_av;
    case OR_F_FA_U_W0: return m->FA_u_W0;
    case OR_F_FA_U_WW: return m->FA_u_WW;
    case OR_F_FA_U_E0: return m->FA_u_E0;
    case OR_F_FA_U_EE: return m->FA_u_EE;
    case OR_F_UBT_WW: return m->uBT_WW;
    case OR_F_UBT_EE: return m->uBT_EE;
    case OR_F_DU_COR: return m->du_cor;
    case OR_F_FA_V_S0: return m->FA_v_S0;
    case OR_F_FA_V_SS: return m->FA_v_SS;
    case OR_F_FA_V_N0: return m->FA_v_N0;
    case OR_F_FA_V_NN: return m->FA_v_NN;
    case OR_F_VBT_SS: return m->vBT_SS;
    case OR_F_VBT_NN: return m->vBT_NN;
    case OR_F_DV_COR: return m->dv_cor;
    case OR_F_TAUX_BOT: return m->vv_taux_bot;
    case OR_F_TAUY_BOT: return m->vv_tauy_bot;
    case OR_F_TAUX: return m->taux;
    case OR_F_TAUY: return m->tauy;
    default: return NULL;
    }
}

size_t oracle_field_size(const oracle_model *m, int field) {
    int is3d;
    if (!field_ptr(m, field, &is3d)) return 0;
    return (size_t)m->n1 * m->n2 * (is3d ? (size_t)m->nk : 1);
}

int oracle_get(const oracle_model *m, int field, double *out) {
    int is3d;
    double *p = field_ptr(m, field, &is3d);
    if (!p) return -1;
    memcpy(out, p, oracle_field_size(m, field) * sizeof(double));
    return 0;
}

int oracle_set(oracle_model *m, int field, const double *in) {
    int is3d;
    double *p = field_ptr(m, field, &is3d);
    if (!p) return -1;
    memcpy(p, in, oracle_field_size(m, field) * sizeof(double));
    return 0;
}

void oracle_set_bt_extended(oracle_model *m, int on) { m->bt_extended = on ? 1 : 0; }
/* btstep's G%first_direction (mom6_barotropic_serial.F90:250): which velocity
 * component the odd substeps update first */
void oracle_set_bt_first_direction(oracle_model *m, int d) { m->first_direction = d; }
void oracle_set_exchange(oracle_model *m, oracle_exchange_fn fn, void *ctx) {
    m->xfn = fn;
    m->xctx = ctx;
}

/* Copy one of the oracle's grid or control-structure arrays by name (count
 * doubles: n1*n2, or 4*n1*n2 for f_4_u/f_4_v).  Returns 0, or -1 for an
 * unknown name or a count mismatch. */
int oracle_array(const oracle_model *m, const char *name, double *out, size_t count) {
    struct { const char *n; const double *p; size_t k; } tab[] = {
        {"IareaT", m->IareaT, 1}, {"areaT", m->areaT, 1}, {"dxT", m->dxT, 1},
        {"IdxT", m->IdxT, 1}, {"dxCu", m->dxCu, 1}, {"dyCu", m->dyCu, 1},
        {"dy_Cu", m->dy_Cu, 1}, {"IdxCu", m->IdxCu, 1}, {"IdyCu", m->IdyCu, 1},
        {"dxCv", m->dxCv, 1}, {"dyCv", m->dyCv, 1}, {"IdxCv", m->IdxCv, 1},
        {"IdyCv", m->IdyCv, 1}, {"IareaBu", m->IareaBu, 1}, {"CoriolisBu", m->CoriolisBu, 1},
        {"IareaCu", m->IareaCu, 1}, {"IareaCv", m->IareaCv, 1}, {"mask2dT", m->mask2dT, 1},
        {"mask2dBu", m->mask2dBu, 1}, {"mask2dCu", m->mask2dCu, 1},
        {"mask2dCv", m->mask2dCv, 1}, {"Area_q", m->co_Area_q, 1},
        {"dx2h", m->hv_dx2h, 1}, {"dy2h", m->hv_dy2h, 1}, {"dx2q", m->hv_dx2q, 1},
        {"dy2q", m->hv_dy2q, 1}, {"DX_dyT", m->hv_DX_dyT, 1}, {"DY_dxT", m->hv_DY_dxT, 1},
        {"DX_dyBu", m->hv_DX_dyBu, 1}, {"DY_dxBu", m->hv_DY_dxBu, 1},
        {"reduction_xx", m->hv_red_xx, 1}, {"reduction_xy", m->hv_red_xy, 1},
        {"Datu", m->bt_Datu, 1}, {"Datv", m->bt_Datv, 1}, {"gtot_E", m->bt_gtot_E, 1},
        {"gtot_W", m->bt_gtot_W, 1}, {"gtot_N", m->bt_gtot_N, 1},
        {"gtot_S", m->bt_gtot_S, 1}, {"f_4_u", m->bt_f_4_u, 4}, {"f_4_v", m->bt_f_4_v, 4},
        {"bt_rem_u", m->bt_rem_u, 1}, {"bt_rem_v", m->bt_rem_v, 1}};
    for (size_t t = 0; t < sizeof(tab) / sizeof(tab[0]); ++t)
        if (strcmp(tab[t].n, name) == 0) {
            size_t n = (size_t)N1 * N2 * tab[t].k;
            if (count != n || !tab[t].p) return -1;
            memcpy(out, tab[t].p, n * sizeof(double));
            return 0;
        }
    return -1;
}

void oracle_dims(const oracle_model *m, int *o) {
    o[0] = m->n1; o[1] = m->n2; o[2] = m->nk;
    o[3] = m->is; o[4] = m->ie; o[5] = m->js; o[6] = m->je; o[7] = m->nstep;
}

/* verify_state, rk2_serial_driver.F90:563-623 */
void oracle_verify(const oracle_model *m, double *out) {
    double mass_init = 0.0, mass_final = 0.0, max_u = 0.0, max_v = 0.0,
           max_eta = 0.0, ke_total = 0.0;
    for (int k = 1; k <= m->nk; ++k)
        for (int j = m->js; j <= m->je; ++j)
            for (int i = m->is; i <= m->ie; ++i) {
                double a = A2(m->areaT, i, j);
                mass_init = mass_init + A3(m->h0, i, j, k) * a;
                mass_final = mass_final + A3(m->h, i, j, k) * a;
                max_u = MAX(max_u, fabs(A3(m->u, i, j, k)));
                max_v = MAX(max_v, fabs(A3(m->v, i, j, k)));
                double uu = A3(m->u, i, j, k), vv = A3(m->v, i, j, k);
                ke_total = ke_total + 0.5 * (uu * uu + vv * vv) * A3(m->h, i, j, k) * a;
            }
    for (int j = m->js; j <= m->je; ++j)
        for (int i = m->is; i <= m->ie; ++i) max_eta = MAX(max_eta, fabs(A2(m->eta, i, j)));
    out[0] = mass_init; out[1] = mass_final;
    out[2] = fabs(mass_final - mass_init) / mass_init;
    out[3] = max_u; out[4] = max_v; out[5] = max_eta; out[6] = ke_total;
}
