/*
 * mom6_cuda_c.h -- the reference-compatible C ABI of libmom6b.so.
 *
 * These are the entry points the reference's src/cuda_c backend exports and
 * its Fortran wrappers bind with iso_c_binding (one `bind(c, name=...)`
 * interface each).  A build that links libmom6b.so instead of the reference's
 * CUDA C objects runs the unchanged Fortran wrappers and rk2_cuda_c_driver on
 * this library's kernels.
 *
 * Conventions, as in the reference:
 *  - every array is a device pointer to the element (isd, jsd[, 1]) of a
 *    Fortran column-major, 1-based array of doubles, dimensions (n1, n2[, n3]);
 *    f_4_u / f_4_v are (4, n1, n2);
 *  - is_l..je_l are the 1-based local compute bounds;
 *  - integer flags are 0 / 1; a pointer whose flag is 0 is never read (the
 *    wrappers pass aliases of other arrays there);
 *  - launch_* return nothing and check nothing; they are enqueued on `stream`
 *    (a cudaStream_t, NULL for the legacy default stream) and do not
 *    synchronize.  The grid_* / block_* arguments are accepted and ignored:
 *    each entry point covers exactly the index ranges of the reference kernel
 *    with a launch geometry of its own;
 *  - scratch arguments the reference kernels write (hvel / z_i of vertical
 *    viscosity) are outputs in the reference but pure scratch for the caller;
 *    this library leaves them untouched.
 *
 * Every result is bit-identical to the reference kernel built without FMA
 * contraction (nvcc --fmad=false), which is how the parity tests check them.
 */
#ifndef MOM6_CUDA_C_H
#define MOM6_CUDA_C_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- runtime helpers: cuda_helpers.h:10-17, mom6_cuda_c_common.F90:19-65 ----
 * Return (int)cudaError_t; cuda_malloc_c returns NULL on failure. */
int   cuda_set_device_c(int device);                                   /* cuda_helpers.cu:8  */
int   cuda_device_synchronize_c(void);                                 /* cuda_helpers.cu:13 */
void *cuda_malloc_c(size_t bytes);                                     /* cuda_helpers.cu:18 */
void  cuda_free_c(void *ptr);                                          /* cuda_helpers.cu:25 */
int   cuda_memcpy_h2d_c(void *dst, const void *src, size_t bytes);     /* cuda_helpers.cu:30 */
int   cuda_memcpy_d2h_c(void *dst, const void *src, size_t bytes);     /* cuda_helpers.cu:35 */
int   cuda_memcpy_d2d_c(void *dst, const void *src, size_t bytes);     /* cuda_helpers.cu:40 */
int   cuda_memset_c(void *ptr, int value, size_t bytes);               /* cuda_helpers.cu:45 */

/* ---- barotropic substep kernels: mom6_barotropic_kernels.cu:347-523,
 *      Fortran bindings mom6_barotropic_cuda_c.F90:76-211 (2-D grids) ---- */
void launch_bt_init_kernel(double *eta, double *ubt, double *vbt, double *ubt_av,
                           double *vbt_av, double *uhbt_av, double *vhbt_av,
                           double *eta_in, double *ubt_in, double *vbt_in, int n1, int n2,
                           int grid_x, int grid_y, int block_x, int block_y, void *stream);
void launch_bt_store_prev_u_kernel(double *ubt_prev, double *ubt, int n1, int n2, int is_l,
                                   int ie_l, int js_l, int je_l, int grid_x, int grid_y,
                                   int block_x, int block_y, void *stream);
void launch_bt_store_prev_v_kernel(double *vbt_prev, double *vbt, int n1, int n2, int is_l,
                                   int ie_l, int js_l, int je_l, int grid_x, int grid_y,
                                   int block_x, int block_y, void *stream);
void launch_bt_eta_pred_kernel(double *eta_pred, double *eta, double *ubt, double *vbt,
                               double *Datu, double *Datv, double *IareaT, int n1, int n2,
                               int is_l, int ie_l, int js_l, int je_l, double dtbt, int grid_x,
                               int grid_y, int block_x, int block_y, void *stream);
void launch_bt_pressure_force_u_kernel(double *PFu, double *eta_pred, double *gtot_E,
                                       double *gtot_W, double *IdxCu, int n1, int n2, int is_l,
                                       int ie_l, int js_l, int je_l, double dgeo_de,
                                       int grid_x, int grid_y, int block_x, int block_y,
                                       void *stream);
void launch_bt_pressure_force_v_kernel(double *PFv, double *eta_pred, double *gtot_N,
                                       double *gtot_S, double *IdyCv, int n1, int n2, int is_l,
                                       int ie_l, int js_l, int je_l, double dgeo_de,
                                       int grid_x, int grid_y, int block_x, int block_y,
                                       void *stream);
void launch_bt_coriolis_update_u_kernel(double *ubt, double *Cor_u, double *vbt, double *PFu,
                                        double *f_4_u, double *bt_rem_u, int n1, int n2,
                                        int is_l, int ie_l, int js_l, int je_l, double dtbt,
                                        int grid_x, int grid_y, int block_x, int block_y,
                                        void *stream);
void launch_bt_coriolis_update_v_kernel(double *vbt, double *Cor_v, double *ubt, double *PFv,
                                        double *f_4_v, double *bt_rem_v, int n1, int n2,
                                        int is_l, int ie_l, int js_l, int je_l, double dtbt,
                                        int grid_x, int grid_y, int block_x, int block_y,
                                        void *stream);
void launch_bt_transport_eta_accum_kernel(double *uhbt, double *vhbt, double *eta,
                                          double *ubt_av, double *vbt_av, double *uhbt_av,
                                          double *vhbt_av, double *ubt, double *vbt,
                                          double *ubt_prev, double *vbt_prev, double *Datu,
                                          double *Datv, double *IareaT, int n1, int n2,
                                          int is_l, int ie_l, int js_l, int je_l, double dtbt,
                                          double trans_wt1, double trans_wt2, double inv_nstep,
                                          int grid_x, int grid_y, int block_x, int block_y,
                                          void *stream);
void launch_bt_eta_update_kernel(double *eta, double *uhbt, double *vhbt, double *IareaT,
                                 int n1, int n2, int is_l, int ie_l, int js_l, int je_l,
                                 double dtbt, int grid_x, int grid_y, int block_x, int block_y,
                                 void *stream);
void launch_bt_copy_output_kernel(double *u_av_out, double *v_av_out, double *eta_out,
                                  double *ubt_av, double *vbt_av, double *eta, int n1, int n2,
                                  int grid_x, int grid_y, int block_x, int block_y,
                                  void *stream);

/* ---- continuity PPM: mom6_continuity_kernels.cu:1108-1305,
 *      Fortran bindings mom6_continuity_cuda_c.F90:78-253 ---- */
void launch_ppm_reconstruction_3d_kernel(double *h_W, double *h_E, double *h_in,
                                         double *mask2dT, int n1, int n2, int n3, int is_l,
                                         int ie_l, int js_l, int je_l, double h_min,
                                         int monotonic, int upwind_1st_flag,
                                         int simple_2nd_flag, int grid_x, int grid_y,
                                         int grid_z, int block_x, int block_y, int block_z,
                                         void *stream);
void launch_zonal_flux_layer_3d_kernel(double *uh, double *duhdu, double *u, double *h_in,
                                       double *h_W, double *h_E, double *dy_Cu, double *IdxT,
                                       double *IareaT, double *por_face_areaU,
                                       double *visc_rem_u, int n1, int n2, int n3, int is_l,
                                       int ie_l, int js_l, int je_l, double dt,
                                       int vol_CFL_flag, int use_visc_rem_flag,
                                       int use_por_face_flag, int grid_x, int grid_y,
                                       int grid_z, int block_x, int block_y, int block_z,
                                       void *stream);
void launch_zonal_convergence_kernel(double *h, double *hin, double *uh, double *IareaT,
                                     int n1, int n2, int n3, int is_l, int ie_l, int js_l,
                                     int je_l, double dt, int grid_x, int grid_y, int grid_z,
                                     int block_x, int block_y, int block_z, void *stream);
void launch_visc_rem_max_kernel(double *visc_rem_max_out, double *visc_rem_u, int n1, int n2,
                                int n3, int is_l, int ie_l, int js_l, int je_l,
                                int use_vrm_max_flag, int grid_x, int grid_y, int grid_z,
                                int block_x, int block_y, int block_z, void *stream);
void launch_uh_duhdu_tot_kernel(double *uh_tot_0, double *duhdu_tot_0, double *uh,
                                double *duhdu, int n1, int n2, int n3, int is_l, int ie_l,
                                int js_l, int je_l, int grid_x, int grid_y, int grid_z,
                                int block_x, int block_y, int block_z, void *stream);
void launch_zonal_CFL_limits_kernel(double *du_max_CFL_out, double *du_min_CFL_out, double *u,
                                    double *visc_rem_u, double *visc_rem_max_in, double *dxT,
                                    double *areaT, double *dy_Cu, double *mask2dCu, int n1,
                                    int n2, int n3, int is_l, int ie_l, int js_l, int je_l,
                                    double CFL_dt, double I_dt, int vol_CFL_flag,
                                    int use_visc_rem_flag, int aggress_flag, int grid_x,
                                    int grid_y, int grid_z, int block_x, int block_y,
                                    int block_z, void *stream);
void launch_zonal_flux_adjust_kernel(double *uh, double *du_out, double *u, double *h_in,
                                     double *h_W, double *h_E, double *uhbt,
                                     double *visc_rem_u, double *por_face_areaU,
                                     double *IareaT, double *dy_Cu, double *IdxT,
                                     double *du_max_CFL_in, double *du_min_CFL_in,
                                     double *uh_tot_0_in, double *duhdu_tot_0_in, int n1,
                                     int n2, int n3, int is_l, int ie_l, int js_l, int je_l,
                                     double dt, double tol_eta_base, double tol_vel_val,
                                     int vol_CFL_flag, int use_visc_rem_flag,
                                     int better_iter_flag, int use_por_face_flag, int grid_x,
                                     int grid_y, int grid_z, int block_x, int block_y,
                                     int block_z, void *stream);
void launch_set_zonal_BT_cont_kernel(double *FA_u_W0, double *FA_u_WW, double *uBT_WW,
                                     double *FA_u_E0, double *FA_u_EE, double *uBT_EE,
                                     double *u, double *h_in, double *h_W, double *h_E,
                                     double *visc_rem_u, double *por_face_areaU,
                                     double *IareaT, double *dy_Cu, double *IdxT, double *dxCu,
                                     double *visc_rem_max_in, double *du_max_CFL_in,
                                     double *du_min_CFL_in, double *uh_tot_0_in,
                                     double *duhdu_tot_0_in, int n1, int n2, int n3, int is_l,
                                     int ie_l, int js_l, int je_l, double dt,
                                     double tol_eta_base, double tol_vel_val, int vol_CFL_flag,
                                     int use_visc_rem_flag, int better_iter_flag,
                                     int use_por_face_flag, int grid_x, int grid_y, int grid_z,
                                     int block_x, int block_y, int block_z, void *stream);
void launch_zonal_flux_thickness_kernel(double *h_u, double *u, double *h, double *h_W,
                                        double *h_E, double *por_face_areaU,
                                        double *visc_rem_u, double *IareaT, double *IdxT,
                                        double *dy_Cu, int n1, int n2, int n3, int is_l,
                                        int ie_l, int js_l, int je_l, double dt,
                                        int vol_CFL_flag, int marginal_flag,
                                        int has_visc_rem_flag, int use_por_face_flag,
                                        int grid_x, int grid_y, int grid_z, int block_x,
                                        int block_y, int block_z, void *stream);
void launch_u_cor_kernel(double *u_cor, double *u, double *du, double *visc_rem_u, int n1,
                         int n2, int n3, int is_l, int ie_l, int js_l, int je_l,
                         int use_visc_rem_flag, int grid_x, int grid_y, int grid_z,
                         int block_x, int block_y, int block_z, void *stream);

/* ---- Coriolis and momentum advection: mom6_coriolis_kernels.cu:545-708,
 *      Fortran bindings mom6_coriolis_cuda_c.F90:62-147 (phase1_kernel_smem,
 *      phase1a_circ and phase1b_ke are exported by the reference but have no
 *      Fortran binding) ---- */
void launch_phase1_kernel(double *dvdx, double *dudy, double *hArea_u, double *hArea_v,
                          double *KE, double *u, double *v, double *h, double *dyCv,
                          double *dxCu, double *dyCu, double *dxCv, double *areaT, int n1,
                          int n2, int n3, int is_l, int ie_l, int js_l, int je_l, int grid_x,
                          int grid_y, int grid_z, int block_x, int block_y, int block_z,
                          void *stream);
void launch_phase1_kernel_smem(double *dvdx, double *dudy, double *hArea_u, double *hArea_v,
                               double *KE, double *u, double *v, double *h, double *dyCv,
                               double *dxCu, double *dyCu, double *dxCv, double *areaT, int n1,
                               int n2, int n3, int is_l, int ie_l, int js_l, int je_l,
                               int grid_x, int grid_y, int grid_z, int block_x, int block_y,
                               int block_z, void *stream);
void launch_phase1a_circ_kernel(double *dvdx, double *dudy, double *hArea_u, double *hArea_v,
                                double *u, double *v, double *h, double *dyCv, double *dxCu,
                                double *areaT, int n1, int n2, int n3, int is_l, int ie_l,
                                int js_l, int je_l, int grid_x, int grid_y, int grid_z,
                                int block_x, int block_y, int block_z, void *stream);
void launch_phase1b_ke_kernel(double *KE, double *u, double *v, double *dyCu, double *dxCv,
                              double *areaT, int n1, int n2, int n3, int is_l, int ie_l,
                              int js_l, int je_l, int grid_x, int grid_y, int grid_z,
                              int block_x, int block_y, int block_z, void *stream);
void launch_vorticity_pv_kernel(double *rel_vort, double *abs_vort, double *q, double *Ih_q,
                                double *dvdx, double *dudy, double *hArea_u, double *hArea_v,
                                double *Area_q, double *IareaBu, double *CoriolisBu,
                                double *mask2dBu, int n1, int n2, int n3, int is_l, int ie_l,
                                int js_l, int je_l, int grid_x, int grid_y, int grid_z,
                                int block_x, int block_y, int block_z, void *stream);
void launch_arakawa_hsu90_coef_kernel(double *a, double *b, double *c, double *d, double *q,
                                      int n1, int n2, int n3, int is_l, int ie_l, int js_l,
                                      int je_l, int grid_x, int grid_y, int grid_z,
                                      int block_x, int block_y, int block_z, void *stream);
void launch_arakawa_lamb81_coef_kernel(double *a, double *b, double *c, double *d, double *q,
                                       int n1, int n2, int n3, int is_l, int ie_l, int js_l,
                                       int je_l, int grid_x, int grid_y, int grid_z,
                                       int block_x, int block_y, int block_z, void *stream);
void launch_coriolis_sadourny_kernel(double *CAu, double *CAv, double *q, double *KE,
                                     double *uh, double *vh, double *IdxCu, double *IdyCv,
                                     int n1, int n2, int n3, int is_l, int ie_l, int js_l,
                                     int je_l, int grid_x, int grid_y, int grid_z, int block_x,
                                     int block_y, int block_z, void *stream);
void launch_coriolis_arakawa_kernel(double *CAu, double *CAv, double *a, double *b, double *c,
                                    double *d, double *KE, double *uh, double *vh,
                                    double *IdxCu, double *IdyCv, int n1, int n2, int n3,
                                    int is_l, int ie_l, int js_l, int je_l, int grid_x,
                                    int grid_y, int grid_z, int block_x, int block_y,
                                    int block_z, void *stream);
void launch_coriolis_fused_sadourny_kernel(double *CAu, double *CAv, double *u, double *v,
                                           double *h, double *uh, double *vh, double *dyCv,
                                           double *dxCu, double *dyCu, double *dxCv,
                                           double *areaT, double *IareaBu, double *CoriolisBu,
                                           double *mask2dBu, double *IdxCu, double *IdyCv,
                                           int n1, int n2, int n3, int is_l, int ie_l,
                                           int js_l, int je_l, int grid_x, int grid_y,
                                           int grid_z, int block_x, int block_y, int block_z,
                                           void *stream);

/* ---- horizontal viscosity: mom6_hor_visc_kernels.cu:157-204,
 *      Fortran bindings mom6_hor_visc_cuda_c.F90:73-96 ---- */
void launch_stress_kernel(double *str_xx, double *str_xy, double *u, double *v, double *h,
                          double *DY_dxT, double *DX_dyT, double *DY_dxBu, double *DX_dyBu,
                          double *IdyCu, double *IdxCu, double *IdyCv, double *IdxCv,
                          double *mask2dBu, double *reduction_xx, double *reduction_xy,
                          double Kh_bg, int n1, int n2, int n3, int is_l, int ie_l, int js_l,
                          int je_l, int grid_x, int grid_y, int grid_z, int block_x,
                          int block_y, int block_z, void *stream);
void launch_divergence_kernel(double *diffu, double *diffv, double *str_xx, double *str_xy,
                              double *h, double *mask2dT, double *IdyCu, double *IdxCu,
                              double *IdyCv, double *IdxCv, double *IareaCu, double *IareaCv,
                              double *dy2h, double *dx2h, double *dy2q, double *dx2q,
                              double h_neglect, int n1, int n2, int n3, int is_l, int ie_l,
                              int js_l, int je_l, int grid_x, int grid_y, int grid_z,
                              int block_x, int block_y, int block_z, void *stream);

/* ---- vertical viscosity: mom6_vert_visc_kernels.cu:301-345,
 *      Fortran bindings mom6_vert_visc_cuda_c.F90:54-72 ---- */
void launch_vert_visc_cra_u_kernel(double *u, double *h, double *mask2dCu, double *visc_rem_u,
                                   double *taux_bot, double *taux, double Kv, double Kv_ml,
                                   double Kv_extra_bbl, double Hmix, double Hbbl, double dt,
                                   double dt_Rho0, double h_neglect, double I_Hbbl, int n1,
                                   int n2, int nz, int is_l, int ie_l, int js_l, int je_l,
                                   double *hvel, double *z_i, int grid_x, int grid_y,
                                   int block_x, int block_y, void *stream);
void launch_vert_visc_cra_v_kernel(double *v, double *h, double *mask2dCv, double *visc_rem_v,
                                   double *tauy_bot, double *tauy, double Kv, double Kv_ml,
                                   double Kv_extra_bbl, double Hmix, double Hbbl, double dt,
                                   double dt_Rho0, double h_neglect, double I_Hbbl, int n1,
                                   int n2, int nz, int is_l, int ie_l, int js_l, int je_l,
                                   double *hvel, double *z_i, int grid_x, int grid_y,
                                   int block_x, int block_y, void *stream);

#ifdef __cplusplus
}
#endif
#endif
