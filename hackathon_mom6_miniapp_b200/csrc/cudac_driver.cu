// cudac_driver.cu -- C++ mirror of the reference's CUDA C host side.
//
// rk2_cuda_c_driver.F90 calls Fortran wrappers (continuity_PPM_cuda_c,
// btstep_cuda_c, CorAdCalc_cuda_c, vert_visc_cra_cuda_c, hor_visc_cuda_c in
// src/cuda_c/*_cuda_c.F90) that own the device control structures and issue
// the launch_* entry points of the ABI in a fixed order, each phase ending
// with a device synchronisation.  This file restates that host side in C++:
// the same control-structure arrays, the same launch sequence and arguments,
// and the driver's inline OpenMP loops (h reset, compute_transports, the
// velocity updates, the htmp copy) as small kernels of its own.
//
// Every launch goes through an AbiTable.  By default it points at this
// library's own launch_* entry points, so the mirror is the drop-in path a
// Fortran build would take; given the path of another shared object that
// exports the same symbols (the reference's CUDA C kernels built from their
// sources), it drives those instead, which is how the reference backend is
// run and timed on the same GPU.
#include <dlfcn.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mom6_cuda_c.h"
#include "../../include/mom6b.h"
#include "abi_common.cuh"
#include "host_init.h"

using namespace mom6b;

int mom6b_internal_fail(int code, const std::string& msg);

namespace {

// ---- the entry points the Fortran wrappers call ---------------------------
struct AbiTable {
    decltype(&launch_phase1_kernel) phase1;
    decltype(&launch_vorticity_pv_kernel) vorticity_pv;
    decltype(&launch_coriolis_sadourny_kernel) sadourny;
    decltype(&launch_stress_kernel) stress;
    decltype(&launch_divergence_kernel) divergence;
    decltype(&launch_vert_visc_cra_u_kernel) vv_u;
    decltype(&launch_vert_visc_cra_v_kernel) vv_v;
    decltype(&launch_bt_init_kernel) bt_init;
    decltype(&launch_bt_store_prev_u_kernel) bt_prev_u;
    decltype(&launch_bt_store_prev_v_kernel) bt_prev_v;
    decltype(&launch_bt_eta_pred_kernel) bt_eta_pred;
    decltype(&launch_bt_pressure_force_u_kernel) bt_pf_u;
    decltype(&launch_bt_pressure_force_v_kernel) bt_pf_v;
    decltype(&launch_bt_coriolis_update_u_kernel) bt_cor_u;
    decltype(&launch_bt_coriolis_update_v_kernel) bt_cor_v;
    decltype(&launch_bt_transport_eta_accum_kernel) bt_accum;
    decltype(&launch_bt_eta_update_kernel) bt_eta_update;
    decltype(&launch_bt_copy_output_kernel) bt_copy;
    decltype(&launch_ppm_reconstruction_3d_kernel) ppm;
    decltype(&launch_zonal_flux_layer_3d_kernel) flux_layer;
    decltype(&launch_visc_rem_max_kernel) vrm;
    decltype(&launch_uh_duhdu_tot_kernel) tot;
    decltype(&launch_zonal_CFL_limits_kernel) cfl;
    decltype(&launch_zonal_flux_adjust_kernel) adjust;
    decltype(&launch_set_zonal_BT_cont_kernel) bt_cont;
    decltype(&launch_zonal_flux_thickness_kernel) thickness;
    decltype(&launch_zonal_convergence_kernel) convergence;
};

AbiTable own_table()
{
    return AbiTable{launch_phase1_kernel,
                    launch_vorticity_pv_kernel,
                    launch_coriolis_sadourny_kernel,
                    launch_stress_kernel,
                    launch_divergence_kernel,
                    launch_vert_visc_cra_u_kernel,
                    launch_vert_visc_cra_v_kernel,
                    launch_bt_init_kernel,
                    launch_bt_store_prev_u_kernel,
                    launch_bt_store_prev_v_kernel,
                    launch_bt_eta_pred_kernel,
                    launch_bt_pressure_force_u_kernel,
                    launch_bt_pressure_force_v_kernel,
                    launch_bt_coriolis_update_u_kernel,
                    launch_bt_coriolis_update_v_kernel,
                    launch_bt_transport_eta_accum_kernel,
                    launch_bt_eta_update_kernel,
                    launch_bt_copy_output_kernel,
                    launch_ppm_reconstruction_3d_kernel,
                    launch_zonal_flux_layer_3d_kernel,
                    launch_visc_rem_max_kernel,
                    launch_uh_duhdu_tot_kernel,
                    launch_zonal_CFL_limits_kernel,
                    launch_zonal_flux_adjust_kernel,
                    launch_set_zonal_BT_cont_kernel,
                    launch_zonal_flux_thickness_kernel,
                    launch_zonal_convergence_kernel};
}

template <class F>
bool sym(void* dl, const char* name, F& out, std::string& err)
{
    void* p = dlsym(dl, name);
    if (!p) {
        err = std::string("missing symbol ") + name;
        return false;
    }
    out = reinterpret_cast<F>(p);
    return true;
}

bool load_table(void* dl, AbiTable& T, std::string& err)
{
    return sym(dl, "launch_phase1_kernel", T.phase1, err) &&
           sym(dl, "launch_vorticity_pv_kernel", T.vorticity_pv, err) &&
           sym(dl, "launch_coriolis_sadourny_kernel", T.sadourny, err) &&
           sym(dl, "launch_stress_kernel", T.stress, err) &&
           sym(dl, "launch_divergence_kernel", T.divergence, err) &&
           sym(dl, "launch_vert_visc_cra_u_kernel", T.vv_u, err) &&
           sym(dl, "launch_vert_visc_cra_v_kernel", T.vv_v, err) &&
           sym(dl, "launch_bt_init_kernel", T.bt_init, err) &&
           sym(dl, "launch_bt_store_prev_u_kernel", T.bt_prev_u, err) &&
           sym(dl, "launch_bt_store_prev_v_kernel", T.bt_prev_v, err) &&
           sym(dl, "launch_bt_eta_pred_kernel", T.bt_eta_pred, err) &&
           sym(dl, "launch_bt_pressure_force_u_kernel", T.bt_pf_u, err) &&
           sym(dl, "launch_bt_pressure_force_v_kernel", T.bt_pf_v, err) &&
           sym(dl, "launch_bt_coriolis_update_u_kernel", T.bt_cor_u, err) &&
           sym(dl, "launch_bt_coriolis_update_v_kernel", T.bt_cor_v, err) &&
           sym(dl, "launch_bt_transport_eta_accum_kernel", T.bt_accum, err) &&
           sym(dl, "launch_bt_eta_update_kernel", T.bt_eta_update, err) &&
           sym(dl, "launch_bt_copy_output_kernel", T.bt_copy, err) &&
           sym(dl, "launch_ppm_reconstruction_3d_kernel", T.ppm, err) &&
           sym(dl, "launch_zonal_flux_layer_3d_kernel", T.flux_layer, err) &&
           sym(dl, "launch_visc_rem_max_kernel", T.vrm, err) &&
           sym(dl, "launch_uh_duhdu_tot_kernel", T.tot, err) &&
           sym(dl, "launch_zonal_CFL_limits_kernel", T.cfl, err) &&
           sym(dl, "launch_zonal_flux_adjust_kernel", T.adjust, err) &&
           sym(dl, "launch_set_zonal_BT_cont_kernel", T.bt_cont, err) &&
           sym(dl, "launch_zonal_flux_thickness_kernel", T.thickness, err) &&
           sym(dl, "launch_zonal_convergence_kernel", T.convergence, err);
}

// ---- the driver's inline loops --------------------------------------------
// compute_transports (rk2_cuda_c_driver.F90:637-652) over the data domain
__global__ void k_transports(const double* u, const double* v, const double* h,
                             const double* dyCu, const double* dxCv, double* uh, double* vh,
                             int n1, int n2, int nk)
{
    const size_t plane = (size_t)n1 * n2, n = plane * nk;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % n1) + 1, j = (int)((t / n1) % n2) + 1;
        const size_t p2 = t % plane;
        const size_t ip = (i + 1 <= n1) ? t + 1 : t;          // min(i + 1, ied)
        const size_t jp = (j + 1 <= n2) ? t + n1 : t;         // min(j + 1, jed)
        uh[t] = u[t] * 0.5 * (h[t] + h[ip]) * dyCu[p2];
        vh[t] = v[t] * 0.5 * (h[t] + h[jp]) * dxCv[p2];
    }
}

// out = base + c (CAx + diffx) on [i0, i1] x [j0, j1] (:313-328, :420-435)
__global__ void k_vel_update(double* out, const double* base, const double* CA,
                             const double* diff, double c, int n1, int n2, int nk, int i0,
                             int i1, int j0, int j1)
{
    const int w = i1 - i0 + 1, hgt = j1 - j0 + 1;
    const size_t n = (size_t)w * hgt * nk;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int i = i0 + (int)(t % w), j = j0 + (int)((t / w) % hgt), k = 1 + (int)(t / ((size_t)w * hgt));
        const size_t p = ((size_t)(k - 1) * n2 + (j - 1)) * n1 + (i - 1);
        out[p] = base[p] + c * (CA[p] + diff[p]);
    }
}

unsigned blocks_for(size_t n)
{
    size_t b = (n + 255) / 256;
    return (unsigned)(b > 8192 ? 8192 : b);
}

} // namespace

struct mom6b_cudac {
    std::unique_ptr<HostGrid> grid;
    AbiTable T;
    void* dl = nullptr;
    int n1, n2, nk, is_l, ie_l, js_l, je_l, nstep;
    double dt;
    std::vector<void*> allocs;
    // driver state (rk2_cuda_c_driver.F90:176-197)
    double *u, *v, *h, *h0, *htmp, *uh, *vh, *CAu, *CAv, *up, *vp, *diffu, *diffv;
    double *eta, *ubt, *vbt, *uhbt, *ubt_av, *vbt_av, *eta_av, *taux, *tauy;
    // metrics (one device copy per distinct array; the wrappers keep one per CS)
    double *IareaT, *IdxT, *dy_Cu, *mask2dT, *dxT, *areaT, *dxCu, *mask2dCu, *mask2dCv;
    double *IareaBu, *CoriolisBu, *mask2dBu, *dyCv, *dyCu, *dxCv, *IdxCu, *IdyCv, *Area_q3;
    double *DY_dxT, *DX_dyT, *DY_dxBu, *DX_dyBu, *IdyCu, *IdxCv, *IareaCu, *IareaCv, *red_xx,
        *red_xy, *dy2h, *dx2h, *dy2q, *dx2q;
    double *Datu, *Datv, *gtot_E, *gtot_W, *gtot_N, *gtot_S, *f_4_u, *f_4_v, *bt_rem_u,
        *bt_rem_v;
    // control-structure scratch
    double *cont_s3d[3], *cont_s2d[6];
    double *FA_u_W0, *FA_u_WW, *FA_u_E0, *FA_u_EE, *uBT_WW, *uBT_EE, *h_u;
    double* cor_scratch[9];
    double *hv_str_xx, *hv_str_xy;
    double *vv_hvel, *vv_z_i, *vv_visc_rem, *vv_tau_bot;
    double *bt_eta, *bt_eta_pred, *bt_ubt, *bt_vbt, *bt_ubt_prev, *bt_vbt_prev, *bt_uhbt,
        *bt_vhbt, *bt_ubt_av, *bt_vbt_av, *bt_uhbt_av, *bt_vhbt_av, *bt_PFu, *bt_PFv, *bt_Cor_u,
        *bt_Cor_v;

    ~mom6b_cudac()
    {
        for (void* p : allocs) cudaFree(p);
        if (dl) dlclose(dl);
    }
};

namespace {

double* dalloc(mom6b_cudac* m, size_t n, cudaError_t* err)
{
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(double));
    if (e != cudaSuccess) {
        *err = e;
        return nullptr;
    }
    m->allocs.push_back(p);
    cudaMemset(p, 0, n * sizeof(double));
    return (double*)p;
}

// ---- the Fortran wrappers --------------------------------------------------
constexpr int BX = 32, BY4 = 4, BY8 = 8;

// hor_visc_cuda_c (mom6_hor_visc_cuda_c.F90:240-297)
void hor_visc(mom6b_cudac* m, double* u, double* v, double* h, double* diffu, double* diffv)
{
    const int gx = (m->n1 + BX - 1) / BX, gy = (m->n2 + BY4 - 1) / BY4;
    m->T.stress(m->hv_str_xx, m->hv_str_xy, u, v, h, m->DY_dxT, m->DX_dyT, m->DY_dxBu,
                m->DX_dyBu, m->IdyCu, m->IdxCu, m->IdyCv, m->IdxCv, m->mask2dBu, m->red_xx,
                m->red_xy, m->grid->cfg.Kh, m->n1, m->n2, m->nk, m->is_l, m->ie_l, m->js_l,
                m->je_l, gx, gy, m->nk, BX, BY4, 1, nullptr);
    m->T.divergence(diffu, diffv, m->hv_str_xx, m->hv_str_xy, h, m->mask2dT, m->IdyCu, m->IdxCu,
                    m->IdyCv, m->IdxCv, m->IareaCu, m->IareaCv, m->dy2h, m->dx2h, m->dy2q,
                    m->dx2q, 1.0e-3, m->n1, m->n2, m->nk, m->is_l, m->ie_l, m->js_l, m->je_l,
                    gx, gy, m->nk, BX, BY4, 1, nullptr);
    cudaDeviceSynchronize();
}

// CorAdCalc_cuda_c, Sadourny scheme (mom6_coriolis_cuda_c.F90:246-317)
void cor_ad_calc(mom6b_cudac* m, double* u, double* v, double* h, double* uh, double* vh,
                 double* CAu, double* CAv)
{
    const int gx = (m->n1 + BX - 1) / BX, gy = (m->n2 + BY8 - 1) / BY8;
    double** s = m->cor_scratch;
    m->T.phase1(s[0], s[1], s[2], s[3], s[4], u, v, h, m->dyCv, m->dxCu, m->dyCu, m->dxCv,
                m->areaT, m->n1, m->n2, m->nk, m->is_l, m->ie_l, m->js_l, m->je_l, gx, gy,
                m->nk, BX, BY8, 1, nullptr);
    m->T.vorticity_pv(s[5], s[6], s[7], s[8], s[0], s[1], s[2], s[3], m->Area_q3, m->IareaBu,
                      m->CoriolisBu, m->mask2dBu, m->n1, m->n2, m->nk, m->is_l, m->ie_l,
                      m->js_l, m->je_l, gx, gy, m->nk, BX, BY8, 1, nullptr);
    m->T.sadourny(CAu, CAv, s[7], s[4], uh, vh, m->IdxCu, m->IdyCv, m->n1, m->n2, m->nk,
                  m->is_l, m->ie_l, m->js_l, m->je_l, gx, gy, m->nk, BX, BY8, 1, nullptr);
    cudaDeviceSynchronize();
}

// vert_visc_cra_cuda_c (mom6_vert_visc_cuda_c.F90:134-187)
void vert_visc(mom6b_cudac* m, double* u, double* v, double* h, double dt)
{
    const mom6b_config& c = m->grid->cfg;
    const double h_neglect = 1.0e-30, I_Hbbl = 1.0 / (c.Hbbl + h_neglect);
    const double dt_Rho0 = dt / 1035.0;
    const int gx = (m->n1 + BX - 1) / BX, gy = (m->n2 + BY4 - 1) / BY4;
    m->T.vv_u(u, h, m->mask2dCu, m->vv_visc_rem, m->vv_tau_bot, m->taux, c.Kv, c.Kv_ml,
              c.Kv_extra_bbl, c.Hmix, c.Hbbl, dt, dt_Rho0, h_neglect, I_Hbbl, m->n1, m->n2,
              m->nk, m->is_l, m->ie_l, m->js_l, m->je_l, m->vv_hvel, m->vv_z_i, gx, gy, BX, BY4,
              nullptr);
    m->T.vv_v(v, h, m->mask2dCv, m->vv_visc_rem, m->vv_tau_bot, m->tauy, c.Kv, c.Kv_ml,
              c.Kv_extra_bbl, c.Hmix, c.Hbbl, dt, dt_Rho0, h_neglect, I_Hbbl, m->n1, m->n2,
              m->nk, m->is_l, m->ie_l, m->js_l, m->je_l, m->vv_hvel, m->vv_z_i, gx, gy, BX, BY4,
              nullptr);
    cudaDeviceSynchronize();
}

// btstep_cuda_c (mom6_barotropic_cuda_c.F90:305-431)
void btstep(mom6b_cudac* m, double* eta_in, double* ubt_in, double* vbt_in, double* u_av,
            double* v_av, double* eta_av)
{
    const int n1 = m->n1, n2 = m->n2, is = m->is_l, ie = m->ie_l, js = m->js_l, je = m->je_l;
    const int gx = (n1 + BX - 1) / BX, gy = (n2 + BY4 - 1) / BY4;
    const double bebt = 0.2, dtbt = m->dt / (double)m->nstep, dgeo_de = 1.0;
    const double trans_wt1 = 1.0 + bebt, trans_wt2 = -bebt;
    const double inv_nstep = 1.0 / (double)m->nstep;
    const int first_direction = 0;
    m->T.bt_init(m->bt_eta, m->bt_ubt, m->bt_vbt, m->bt_ubt_av, m->bt_vbt_av, m->bt_uhbt_av,
                 m->bt_vhbt_av, eta_in, ubt_in, vbt_in, n1, n2, gx, gy, BX, BY4, nullptr);
    for (int n = 1; n <= m->nstep; ++n) {
        m->T.bt_prev_u(m->bt_ubt_prev, m->bt_ubt, n1, n2, is, ie, js, je, gx, gy, BX, BY4,
                       nullptr);
        m->T.bt_prev_v(m->bt_vbt_prev, m->bt_vbt, n1, n2, is, ie, js, je, gx, gy, BX, BY4,
                       nullptr);
        m->T.bt_eta_pred(m->bt_eta_pred, m->bt_eta, m->bt_ubt, m->bt_vbt, m->Datu, m->Datv,
                         m->IareaT, n1, n2, is, ie, js, je, dtbt, gx, gy, BX, BY4, nullptr);
        m->T.bt_pf_u(m->bt_PFu, m->bt_eta_pred, m->gtot_E, m->gtot_W, m->IdxCu, n1, n2, is, ie,
                     js, je, dgeo_de, gx, gy, BX, BY4, nullptr);
        m->T.bt_pf_v(m->bt_PFv, m->bt_eta_pred, m->gtot_N, m->gtot_S, m->IdyCv, n1, n2, is, ie,
                     js, je, dgeo_de, gx, gy, BX, BY4, nullptr);
        auto cor_u = [&] {
            m->T.bt_cor_u(m->bt_ubt, m->bt_Cor_u, m->bt_vbt, m->bt_PFu, m->f_4_u, m->bt_rem_u,
                          n1, n2, is, ie, js, je, dtbt, gx, gy, BX, BY4, nullptr);
        };
        auto cor_v = [&] {
            m->T.bt_cor_v(m->bt_vbt, m->bt_Cor_v, m->bt_ubt, m->bt_PFv, m->f_4_v, m->bt_rem_v,
                          n1, n2, is, ie, js, je, dtbt, gx, gy, BX, BY4, nullptr);
        };
        if (((n + first_direction) % 2) == 1) {
            cor_v();
            cor_u();
        } else {
            cor_u();
            cor_v();
        }
        m->T.bt_accum(m->bt_uhbt, m->bt_vhbt, m->bt_eta, m->bt_ubt_av, m->bt_vbt_av,
                      m->bt_uhbt_av, m->bt_vhbt_av, m->bt_ubt, m->bt_vbt, m->bt_ubt_prev,
                      m->bt_vbt_prev, m->Datu, m->Datv, m->IareaT, n1, n2, is, ie, js, je, dtbt,
                      trans_wt1, trans_wt2, inv_nstep, gx, gy, BX, BY4, nullptr);
        m->T.bt_eta_update(m->bt_eta, m->bt_uhbt, m->bt_vhbt, m->IareaT, n1, n2, is, ie, js,
                           je, dtbt, gx, gy, BX, BY4, nullptr);
    }
    m->T.bt_copy(u_av, v_av, eta_av, m->bt_ubt_av, m->bt_vbt_av, m->bt_eta, n1, n2, gx, gy, BX,
                 BY4, nullptr);
    cudaDeviceSynchronize();
}

// continuity_PPM_cuda_c with uhbt and BT_cont present (mom6_continuity_cuda_c.F90:423-616)
void continuity(mom6b_cudac* m, double* u, double* hin, double* h, double* uh, double dt)
{
    const int n1 = m->n1, n2 = m->n2, n3 = m->nk;
    const int is = m->is_l, ie = m->ie_l, js = m->js_l, je = m->je_l;
    const int gx = (n1 + BX - 1) / BX, gy = (n2 + BY4 - 1) / BY4;
    const double h_min = 2.0e-10, CFL_dt = 0.5 / dt, I_dt = 1.0 / dt;
    const int mono = 1, upwind = 0, simple = 0, vol_CFL = 0, aggress = 0, better = 1,
              marginal = 1;
    double** s3 = m->cont_s3d;
    double** s2 = m->cont_s2d;
    m->T.ppm(s3[0], s3[1], hin, m->mask2dT, n1, n2, n3, is, ie, js, je, h_min, mono, upwind,
             simple, gx, gy, n3, BX, BY4, 1, nullptr);
    m->T.flux_layer(uh, s3[2], u, hin, s3[0], s3[1], m->dy_Cu, m->IdxT, m->IareaT, s3[0], s3[0],
                    n1, n2, n3, is, ie, js, je, dt, vol_CFL, 0, 0, gx, gy, n3, BX, BY4, 1,
                    nullptr);
    m->T.vrm(s2[5], s3[0], n1, n2, n3, is, ie, js, je, 0, gx, gy, 1, BX, BY4, 1, nullptr);
    m->T.tot(s2[4], s2[3], uh, s3[2], n1, n2, n3, is, ie, js, je, gx, gy, 1, BX, BY4, 1,
             nullptr);
    m->T.cfl(s2[1], s2[2], u, s3[0], s2[5], m->dxT, m->areaT, m->dy_Cu, m->mask2dCu, n1, n2, n3,
             is, ie, js, je, CFL_dt, I_dt, vol_CFL, 0, aggress, gx, gy, 1, BX, BY4, 1, nullptr);
    m->T.adjust(uh, s2[0], u, hin, s3[0], s3[1], m->uhbt, s3[0], s3[0], m->IareaT, m->dy_Cu,
                m->IdxT, s2[1], s2[2], s2[4], s2[3], n1, n2, n3, is, ie, js, je, dt, 1.0e-12,
                3.0e8, vol_CFL, 0, better, 0, gx, gy, 1, BX, BY4, 1, nullptr);
    m->T.bt_cont(m->FA_u_W0, m->FA_u_WW, m->uBT_WW, m->FA_u_E0, m->FA_u_EE, m->uBT_EE, u, hin,
                 s3[0], s3[1], s3[0], s3[0], m->IareaT, m->dy_Cu, m->IdxT, m->dxCu, s2[5],
                 s2[1], s2[2], s2[4], s2[3], n1, n2, n3, is, ie, js, je, dt, 1.0e-12, 3.0e8,
                 vol_CFL, 0, better, 0, gx, gy, 1, BX, BY4, 1, nullptr);
    m->T.thickness(m->h_u, u, hin, s3[0], s3[1], s3[0], s3[0], m->IareaT, m->IdxT, m->dy_Cu, n1,
                   n2, n3, is, ie, js, je, dt, vol_CFL, marginal, 0, 0, gx, gy, n3, BX, BY4, 1,
                   nullptr);
    m->T.convergence(h, hin, uh, m->IareaT, n1, n2, n3, is, ie, js, je, dt, gx, gy, n3, BX, BY4,
                     1, nullptr);
    cudaDeviceSynchronize();
}

void transports(mom6b_cudac* m, double* u, double* v, double* h)
{
    const size_t n = (size_t)m->n1 * m->n2 * m->nk;
    k_transports<<<blocks_for(n), 256>>>(u, v, h, m->dyCu, m->dxCv, m->uh, m->vh, m->n1, m->n2,
                                         m->nk);
    cudaDeviceSynchronize();
}

void vel_update(mom6b_cudac* m, double* up, double* vp, double* u, double* v, double c)
{
    const HostGrid& g = *m->grid;
    // up on [isc, iec-1] x [jsc, jec], vp on [isc, iec] x [jsc, jec-1]
    size_t nu = (size_t)(g.ie - 1 - g.is + 1) * (g.je - g.js + 1) * m->nk;
    k_vel_update<<<blocks_for(nu), 256>>>(up, u, m->CAu, m->diffu, c, m->n1, m->n2, m->nk, g.is,
                                          g.ie - 1, g.js, g.je);
    size_t nv = (size_t)(g.ie - g.is + 1) * (g.je - 1 - g.js + 1) * m->nk;
    k_vel_update<<<blocks_for(nv), 256>>>(vp, v, m->CAv, m->diffv, c, m->n1, m->n2, m->nk, g.is,
                                          g.ie, g.js, g.je - 1);
    cudaDeviceSynchronize();
}

// one iteration of rk2_cuda_c_driver.F90:263-481
void rk2_step(mom6b_cudac* m)
{
    const double dt = m->dt;
    const size_t n3b = (size_t)m->n1 * m->n2 * m->nk * sizeof(double);
    cudaMemcpy(m->h, m->h0, n3b, cudaMemcpyDeviceToDevice);             // h = h0
    // predictor
    transports(m, m->u, m->v, m->h);
    hor_visc(m, m->u, m->v, m->h, m->diffu, m->diffv);
    cor_ad_calc(m, m->u, m->v, m->h, m->uh, m->vh, m->CAu, m->CAv);
    vel_update(m, m->up, m->vp, m->u, m->v, dt);
    vert_visc(m, m->up, m->vp, m->h, dt);
    btstep(m, m->eta, m->ubt, m->vbt, m->ubt_av, m->vbt_av, m->eta_av);
    continuity(m, m->up, m->h0, m->h, m->uh, dt);
    // corrector
    transports(m, m->up, m->vp, m->h);
    hor_visc(m, m->up, m->vp, m->h, m->diffu, m->diffv);
    cor_ad_calc(m, m->up, m->vp, m->h, m->uh, m->vh, m->CAu, m->CAv);
    vel_update(m, m->u, m->v, m->u, m->v, 0.5 * dt);
    vert_visc(m, m->u, m->v, m->h, 0.5 * dt);
    btstep(m, m->eta_av, m->ubt_av, m->vbt_av, m->ubt_av, m->vbt_av, m->eta);
    cudaMemcpy(m->htmp, m->h, n3b, cudaMemcpyDeviceToDevice);          // htmp = h
    continuity(m, m->u, m->htmp, m->h, m->uh, 0.5 * dt);
}

double* field_ptr(mom6b_cudac* m, int f, bool* three_d)
{
    *three_d = true;
    switch (f) {
    case MOM6B_F_U: return m->u;
    case MOM6B_F_V: return m->v;
    case MOM6B_F_H: return m->h;
    case MOM6B_F_H0: return m->h0;
    case MOM6B_F_UH: return m->uh;
    case MOM6B_F_VH: return m->vh;
    case MOM6B_F_UP: return m->up;
    case MOM6B_F_VP: return m->vp;
    case MOM6B_F_HU_BT: return m->h_u;
    default: break;
    }
    *three_d = false;
    switch (f) {
    case MOM6B_F_ETA: return m->eta;
    case MOM6B_F_UBT: return m->ubt;
    case MOM6B_F_VBT: return m->vbt;
    case MOM6B_F_UBT_AV: return m->ubt_av;
    case MOM6B_F_VBT_AV: return m->vbt_av;
    case MOM6B_F_ETA_AV: return m->eta_av;
    case MOM6B_F_FA_U_W0: return m->FA_u_W0;
    case MOM6B_F_FA_U_WW: return m->FA_u_WW;
    case MOM6B_F_FA_U_E0: return m->FA_u_E0;
    case MOM6B_F_FA_U_EE: return m->FA_u_EE;
    case MOM6B_F_UBT_WW: return m->uBT_WW;
    case MOM6B_F_UBT_EE: return m->uBT_EE;
    case MOM6B_F_TAUX_BOT: return m->vv_tau_bot;
    case MOM6B_F_TAUX: return m->taux;
    case MOM6B_F_TAUY: return m->tauy;
    default: return nullptr;
    }
}

} // namespace

extern "C" int mom6b_cudac_create(int ni, int nj, int nk, int bt_nsteps, double dt,
                                  const char* kernel_lib, mom6b_cudac** out)
{
    mom6b_config c;
    mom6b_config_default(&c, MOM6B_INIT_REF);
    c.ni = ni; c.nj = nj; c.nk = nk; c.bt_nsteps = bt_nsteps; c.dt = dt;
    return mom6b_cudac_create_cfg(&c, kernel_lib, out);
}

extern "C" int mom6b_cudac_create_cfg(const mom6b_config* cfg, const char* kernel_lib,
                                      mom6b_cudac** out)
{
    if (!out || !cfg) return mom6b_internal_fail(MOM6B_ERR_ARG, "bad argument");
    const int ni = cfg->ni, nj = cfg->nj, nk = cfg->nk, bt_nsteps = cfg->bt_nsteps;
    const double dt = cfg->dt;
    if (ni < 8 || nj < 8 || nk < 1 || bt_nsteps < 1 || !(dt > 0.0) ||
        (cfg->init_mode != MOM6B_INIT_REF && cfg->init_mode != MOM6B_INIT_CFG))
        return mom6b_internal_fail(MOM6B_ERR_ARG, "bad argument");
    *out = nullptr;
    std::unique_ptr<mom6b_cudac> m(new mom6b_cudac());
    if (kernel_lib && kernel_lib[0]) {
        m->dl = dlopen(kernel_lib, RTLD_NOW | RTLD_LOCAL);
        if (!m->dl) return mom6b_internal_fail(MOM6B_ERR_ARG, std::string("dlopen: ") + dlerror());
        std::string err;
        if (!load_table(m->dl, m->T, err)) return mom6b_internal_fail(MOM6B_ERR_ARG, err);
    } else {
        m->T = own_table();
    }
    mom6b_config c = *cfg;
    m->grid = std::make_unique<HostGrid>(c);
    HostGrid& g = *m->grid;
    if (c.init_mode == MOM6B_INIT_REF)
        g.pi_init = 3.14159265358979323846;   // PI, rk2_cuda_c_driver.F90:477-542
    g.build();
    m->n1 = g.n1; m->n2 = g.n2; m->nk = nk; m->nstep = bt_nsteps; m->dt = dt;
    // local 1-based bounds: is - isd + 1 with isd = 1
    m->is_l = g.is; m->ie_l = g.ie; m->js_l = g.js; m->je_l = g.je;

    const size_t n2 = g.plane, n3 = g.plane * nk;
    cudaError_t err = cudaSuccess;
    mom6b_cudac* M = m.get();
    auto A2 = [&] { return dalloc(M, n2, &err); };
    auto A3 = [&] { return dalloc(M, n3, &err); };
    auto up2 = [&](const std::vector<double>& src) {
        double* d = dalloc(M, src.size(), &err);
        if (d) cudaMemcpy(d, src.data(), src.size() * sizeof(double), cudaMemcpyHostToDevice);
        return d;
    };
    m->u = A3(); m->v = A3(); m->h = A3(); m->h0 = A3(); m->htmp = A3(); m->uh = A3();
    m->vh = A3(); m->CAu = A3(); m->CAv = A3(); m->up = A3(); m->vp = A3(); m->diffu = A3();
    m->diffv = A3();
    m->eta = A2(); m->ubt = A2(); m->vbt = A2(); m->uhbt = A2(); m->ubt_av = A2();
    m->vbt_av = A2(); m->eta_av = A2();
    m->taux = up2(g.taux); m->tauy = up2(g.tauy);
    m->IareaT = up2(g.IareaT); m->IdxT = up2(g.IdxT); m->dy_Cu = up2(g.dy_Cu);
    m->mask2dT = up2(g.mask2dT); m->dxT = up2(g.dxT); m->areaT = up2(g.areaT);
    m->dxCu = up2(g.dxCu); m->mask2dCu = up2(g.mask2dCu); m->mask2dCv = up2(g.mask2dCv);
    m->IareaBu = up2(g.IareaBu); m->CoriolisBu = up2(g.CoriolisBu);
    m->mask2dBu = up2(g.mask2dBu); m->dyCv = up2(g.dyCv); m->dyCu = up2(g.dyCu);
    m->dxCv = up2(g.dxCv); m->IdxCu = up2(g.IdxCu); m->IdyCv = up2(g.IdyCv);
    {
        std::vector<double> aq(n3);
        for (int k = 0; k < nk; ++k)
            std::memcpy(aq.data() + (size_t)k * n2, g.Area_q.data(), n2 * sizeof(double));
        m->Area_q3 = up2(aq);
    }
    m->DY_dxT = up2(g.DY_dxT); m->DX_dyT = up2(g.DX_dyT); m->DY_dxBu = up2(g.DY_dxBu);
    m->DX_dyBu = up2(g.DX_dyBu); m->IdyCu = up2(g.IdyCu); m->IdxCv = up2(g.IdxCv);
    m->IareaCu = up2(g.IareaCu); m->IareaCv = up2(g.IareaCv); m->red_xx = up2(g.red_xx);
    m->red_xy = up2(g.red_xy); m->dy2h = up2(g.dy2h); m->dx2h = up2(g.dx2h);
    m->dy2q = up2(g.dy2q); m->dx2q = up2(g.dx2q);
    m->Datu = up2(g.Datu); m->Datv = up2(g.Datv); m->gtot_E = up2(g.gtot_E);
    m->gtot_W = up2(g.gtot_W); m->gtot_N = up2(g.gtot_N); m->gtot_S = up2(g.gtot_S);
    m->f_4_u = up2(g.f_4_u); m->f_4_v = up2(g.f_4_v); m->bt_rem_u = up2(g.bt_rem_u);
    m->bt_rem_v = up2(g.bt_rem_v);
    for (auto& p : m->cont_s3d) p = A3();
    for (auto& p : m->cont_s2d) p = A2();
    m->FA_u_W0 = A2(); m->FA_u_WW = A2(); m->FA_u_E0 = A2(); m->FA_u_EE = A2();
    m->uBT_WW = A2(); m->uBT_EE = A2(); m->h_u = A3();
    for (auto& p : m->cor_scratch) p = A3();
    m->hv_str_xx = A3(); m->hv_str_xy = A3();
    m->vv_hvel = A3(); m->vv_z_i = dalloc(M, g.plane * (nk + 1), &err);
    m->vv_visc_rem = A3(); m->vv_tau_bot = A2();
    m->bt_eta = A2(); m->bt_eta_pred = A2(); m->bt_ubt = A2(); m->bt_vbt = A2();
    m->bt_ubt_prev = A2(); m->bt_vbt_prev = A2(); m->bt_uhbt = A2(); m->bt_vhbt = A2();
    m->bt_ubt_av = A2(); m->bt_vbt_av = A2(); m->bt_uhbt_av = A2(); m->bt_vhbt_av = A2();
    m->bt_PFu = A2(); m->bt_PFv = A2(); m->bt_Cor_u = A2(); m->bt_Cor_v = A2();
    if (err != cudaSuccess)
        return mom6b_internal_fail(MOM6B_ERR_NOMEM, std::string("cudaMalloc: ") +
                                                        cudaGetErrorString(err));
    // initial state (rk2_cuda_c_driver.F90:216-218), uhbt = 0
    std::vector<double> u, v, h0, eta, ubt, vbt;
    g.initial_state(u, v, h0, eta, ubt, vbt);
    auto cp = [&](double* d, const std::vector<double>& s) {
        cudaMemcpy(d, s.data(), s.size() * sizeof(double), cudaMemcpyHostToDevice);
    };
    cp(m->u, u); cp(m->v, v); cp(m->h0, h0); cp(m->h, h0); cp(m->eta, eta); cp(m->ubt, ubt);
    cp(m->vbt, vbt);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
        return mom6b_internal_fail(MOM6B_ERR_CUDA, std::string("init: ") + cudaGetErrorString(e));
    *out = m.release();
    return MOM6B_OK;
}

extern "C" int mom6b_cudac_step(mom6b_cudac* m, int nsteps)
{
    if (!m || nsteps < 0) return mom6b_internal_fail(MOM6B_ERR_ARG, "bad argument");
    for (int n = 0; n < nsteps; ++n) rk2_step(m);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return mom6b_internal_fail(MOM6B_ERR_CUDA, std::string("step: ") + cudaGetErrorString(e));
    return MOM6B_OK;
}

extern "C" int mom6b_cudac_get_field(mom6b_cudac* m, int field, double* host, size_t count)
{
    if (!m || !host) return mom6b_internal_fail(MOM6B_ERR_ARG, "bad argument");
    bool three_d = false;
    double* d = field_ptr(m, field, &three_d);
    if (!d) return mom6b_internal_fail(MOM6B_ERR_ARG, "unknown field");
    size_t n = (size_t)m->n1 * m->n2 * (three_d ? m->nk : 1);
    if (count != n) return mom6b_internal_fail(MOM6B_ERR_ARG, "count mismatch");
    cudaError_t e = cudaMemcpy(host, d, n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return mom6b_internal_fail(MOM6B_ERR_CUDA, std::string("get: ") + cudaGetErrorString(e));
    return MOM6B_OK;
}

extern "C" size_t mom6b_cudac_field_size(const mom6b_cudac* m, int field)
{
    if (!m) return 0;
    bool three_d = false;
    if (!field_ptr(const_cast<mom6b_cudac*>(m), field, &three_d)) return 0;
    return (size_t)m->n1 * m->n2 * (three_d ? m->nk : 1);
}

extern "C" int mom6b_cudac_destroy(mom6b_cudac* m)
{
    delete m;
    return MOM6B_OK;
}
