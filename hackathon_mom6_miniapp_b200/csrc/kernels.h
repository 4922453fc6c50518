// kernels.h -- parameter blocks and host launchers of the FP64 step kernels.
#pragma once

#include "common.cuh"

namespace mom6b {

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
};

struct BTParams {
    double dtbt, dgeo_de, trans_wt1, trans_wt2, inv_nstep;
    int nstep, first_direction, extended;
    long long spin_budget;     // clock64 cycles a block may wait at one barrier
};

cudaError_t launch_tendency(const Dims& D, const Metrics& M, const double* uin,
                            const double* vin, const double* h, const double* ubase,
                            const double* vbase, double* uout, double* vout,
                            double coef, double h_neglect, cudaStream_t s);
cudaError_t launch_vertvisc(const Dims& D, const Metrics& M, double* u, double* v,
                            const double* h, double dt, const VVParams& P,
                            double* taux_bot, double* tauy_bot, cudaStream_t s);
cudaError_t launch_continuity(const Dims& D, const Metrics& M, const double* u,
                              const double* hin, double* hW, double* hE,
                              const double* uhbt, const ContOut& O, double dt,
                              double h_min, cudaStream_t s);
cudaError_t launch_btstep(const Dims& D, const Metrics& M, const BTWork& W,
                          const BTParams& P, const double* eta_in,
                          const double* ubt_in, const double* vbt_in, double* u_av,
                          double* v_av, double* eta_av, cudaStream_t s);
cudaError_t launch_halo_fill(const Dims& D, double* f, int nz, int kind, cudaStream_t s);

}  // namespace mom6b
