// abi_barotropic.cu -- launch_bt_* of the reference-compatible ABI.
//
// One entry point per barotropic substep kernel of the reference's CUDA C
// backend (mom6_barotropic_kernels.cu:12-334, launchers :347-523).  Each
// covers the index ranges of the reference kernel and evaluates the same
// arithmetic in the same order, so results are bit-identical to that kernel
// built without FMA contraction.  The fused persistent barotropic loop of the
// high-level API (k_btstep.cu) is the fast path; these entry points exist so
// the reference's Fortran btstep_cuda_c runs unchanged on this library.
#include "../../include/mom6_cuda_c.h"
#include "abi_common.cuh"

using namespace mom6b::abi;

extern "C" void launch_bt_init_kernel(double* eta, double* ubt, double* vbt, double* ubt_av,
                                      double* vbt_av, double* uhbt_av, double* vhbt_av,
                                      double* eta_in, double* ubt_in, double* vbt_in, int n1,
                                      int n2, int, int, int, int, void* stream)
{
    run_box(Box{1, n1, 1, n2}, 1, stream, [=] __device__(int i, int j, int) {
        const size_t p = at2(i, j, n1);
        eta[p] = eta_in[p];
        ubt[p] = ubt_in[p];
        vbt[p] = vbt_in[p];
        ubt_av[p] = 0.0;
        vbt_av[p] = 0.0;
        uhbt_av[p] = 0.0;
        vhbt_av[p] = 0.0;
    });
}

extern "C" void launch_bt_store_prev_u_kernel(double* ubt_prev, double* ubt, int n1, int n2,
                                              int is_l, int ie_l, int js_l, int je_l, int, int,
                                              int, int, void* stream)
{
    run_box(clip(Box{is_l - 1, ie_l + 1, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) { ubt_prev[at2(i, j, n1)] = ubt[at2(i, j, n1)]; });
}

extern "C" void launch_bt_store_prev_v_kernel(double* vbt_prev, double* vbt, int n1, int n2,
                                              int is_l, int ie_l, int js_l, int je_l, int, int,
                                              int, int, void* stream)
{
    run_box(clip(Box{is_l, ie_l, js_l - 1, je_l + 1}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) { vbt_prev[at2(i, j, n1)] = vbt[at2(i, j, n1)]; });
}

// eta_pred = eta + (dtbt IareaT) (div of Datu ubt, Datv vbt)   (:86-106)
extern "C" void launch_bt_eta_pred_kernel(double* eta_pred, double* eta, double* ubt,
                                          double* vbt, double* Datu, double* Datv,
                                          double* IareaT, int n1, int n2, int is_l, int ie_l,
                                          int js_l, int je_l, double dtbt, int, int, int, int,
                                          void* stream)
{
    run_box(clip(Box{is_l, ie_l, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p = at2(i, j, n1), pw = at2(i - 1, j, n1), ps = at2(i, j - 1, n1);
                const double xflux = Datu[pw] * ubt[pw] - Datu[p] * ubt[p];
                const double yflux = Datv[ps] * vbt[ps] - Datv[p] * vbt[p];
                eta_pred[p] = eta[p] + (dtbt * IareaT[p]) * (xflux + yflux);
            });
}

// PFu = (eta_pred gtot_E - eta_pred(i+1) gtot_W(i+1)) dgeo_de IdxCu   (:112-131)
extern "C" void launch_bt_pressure_force_u_kernel(double* PFu, double* eta_pred, double* gtot_E,
                                                  double* gtot_W, double* IdxCu, int n1, int n2,
                                                  int is_l, int ie_l, int js_l, int je_l,
                                                  double dgeo_de, int, int, int, int,
                                                  void* stream)
{
    run_box(clip(Box{is_l, ie_l - 1, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p = at2(i, j, n1), pe = at2(i + 1, j, n1);
                const double dp = eta_pred[p] * gtot_E[p] - eta_pred[pe] * gtot_W[pe];
                PFu[p] = dp * dgeo_de * IdxCu[p];
            });
}

extern "C" void launch_bt_pressure_force_v_kernel(double* PFv, double* eta_pred, double* gtot_N,
                                                  double* gtot_S, double* IdyCv, int n1, int n2,
                                                  int is_l, int ie_l, int js_l, int je_l,
                                                  double dgeo_de, int, int, int, int,
                                                  void* stream)
{
    run_box(clip(Box{is_l, ie_l, js_l, je_l - 1}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p = at2(i, j, n1), pn = at2(i, j + 1, n1);
                const double dp = eta_pred[p] * gtot_N[p] - eta_pred[pn] * gtot_S[pn];
                PFv[p] = dp * dgeo_de * IdyCv[p];
            });
}

// Four-point Coriolis on the other component, then the damped update
// (:164-189): the pairing of the four products is part of the result.
extern "C" void launch_bt_coriolis_update_u_kernel(double* ubt, double* Cor_u, double* vbt,
                                                   double* PFu, double* f_4_u, double* bt_rem_u,
                                                   int n1, int n2, int is_l, int ie_l, int js_l,
                                                   int je_l, double dtbt, int, int, int, int,
                                                   void* stream)
{
    run_box(clip(Box{is_l, ie_l - 1, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p = at2(i, j, n1);
                const double east = f_4_u[at4(4, i, j, n1)] * vbt[at2(i + 1, j, n1)] +
                                    f_4_u[at4(1, i, j, n1)] * vbt[at2(i, j - 1, n1)];
                const double west = f_4_u[at4(3, i, j, n1)] * vbt[p] +
                                    f_4_u[at4(2, i, j, n1)] * vbt[at2(i + 1, j - 1, n1)];
                const double cor = east + west;
                Cor_u[p] = cor;
                ubt[p] = bt_rem_u[p] * (ubt[p] + dtbt * (cor + PFu[p]));
            });
}

extern "C" void launch_bt_coriolis_update_v_kernel(double* vbt, double* Cor_v, double* ubt,
                                                   double* PFv, double* f_4_v, double* bt_rem_v,
                                                   int n1, int n2, int is_l, int ie_l, int js_l,
                                                   int je_l, double dtbt, int, int, int, int,
                                                   void* stream)
{
    run_box(clip(Box{is_l, ie_l, js_l, je_l - 1}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p = at2(i, j, n1);
                const double a = f_4_v[at4(1, i, j, n1)] * ubt[at2(i - 1, j, n1)] +
                                 f_4_v[at4(4, i, j, n1)] * ubt[at2(i, j + 1, n1)];
                const double b = f_4_v[at4(2, i, j, n1)] * ubt[p] +
                                 f_4_v[at4(3, i, j, n1)] * ubt[at2(i - 1, j + 1, n1)];
                const double cor = -1.0 * (a + b);
                Cor_v[p] = cor;
                vbt[p] = bt_rem_v[p] * (vbt[p] + dtbt * (cor + PFv[p]));
            });
}

// uhbt/vhbt on the extended ranges and the running averages (:228-271).
extern "C" void launch_bt_transport_eta_accum_kernel(
    double* uhbt, double* vhbt, double*, double* ubt_av, double* vbt_av, double* uhbt_av,
    double* vhbt_av, double* ubt, double* vbt, double* ubt_prev, double* vbt_prev, double* Datu,
    double* Datv, double*, int n1, int n2, int is_l, int ie_l, int js_l, int je_l, double,
    double trans_wt1, double trans_wt2, double inv_nstep, int, int, int, int, void* stream)
{
    run_box(clip(Box{is_l - 1, ie_l, js_l - 1, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p = at2(i, j, n1);
                if (i >= is_l - 1 && j >= js_l) {          // u faces
                    const double t = Datu[p] * (trans_wt1 * ubt[p] + trans_wt2 * ubt_prev[p]);
                    uhbt[p] = t;
                    ubt_av[p] = ubt_av[p] + ubt[p] * inv_nstep;
                    uhbt_av[p] = uhbt_av[p] + t * inv_nstep;
                }
                if (i >= is_l && j >= js_l - 1) {          // v faces
                    const double t = Datv[p] * (trans_wt1 * vbt[p] + trans_wt2 * vbt_prev[p]);
                    vhbt[p] = t;
                    vbt_av[p] = vbt_av[p] + vbt[p] * inv_nstep;
                    vhbt_av[p] = vhbt_av[p] + t * inv_nstep;
                }
            });
}

// eta -= dtbt IareaT div(uhbt, vhbt)   (:279-297)
extern "C" void launch_bt_eta_update_kernel(double* eta, double* uhbt, double* vhbt,
                                            double* IareaT, int n1, int n2, int is_l, int ie_l,
                                            int js_l, int je_l, double dtbt, int, int, int, int,
                                            void* stream)
{
    run_box(clip(Box{is_l, ie_l, js_l, je_l}, n1, n2), 1, stream,
            [=] __device__(int i, int j, int) {
                const size_t p = at2(i, j, n1);
                const double div = (uhbt[p] - uhbt[at2(i - 1, j, n1)]) +
                                   (vhbt[p] - vhbt[at2(i, j - 1, n1)]);
                eta[p] = eta[p] - dtbt * IareaT[p] * div;
            });
}

extern "C" void launch_bt_copy_output_kernel(double* u_av_out, double* v_av_out, double* eta_out,
                                             double* ubt_av, double* vbt_av, double* eta, int n1,
                                             int n2, int, int, int, int, void* stream)
{
    run_box(Box{1, n1, 1, n2}, 1, stream, [=] __device__(int i, int j, int) {
        const size_t p = at2(i, j, n1);
        u_av_out[p] = ubt_av[p];
        v_av_out[p] = vbt_av[p];
        eta_out[p] = eta[p];
    });
}
