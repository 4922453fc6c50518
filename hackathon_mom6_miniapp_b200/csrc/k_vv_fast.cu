// k_vv_fast.cu -- vertical viscosity, the fast forms (FP64 and mixed).
//
// The staged one-thread-per-column kernel of vertvisc_impl.cuh
// (vert_visc_coef + vert_visc_apply, mom6_vert_visc_serial.F90:138-287 and
// :394-506) instantiated with FAST and built with FMA contraction: quotients
// by Newton-Raphson-refined reciprocals (div_nr), and the bottom-boundary
// function botfn(z_i) formed top-down from the column's total harmonic
// thickness instead of stored by the bottom-up sweep, so the only per-column
// scratch is the elimination multipliers c1.  R = double is the fast FP64
// form (within 1e-12 relative L2 of the exact form, tested); R = float with
// the elimination in double is the mixed form.
#include "vertvisc_impl.cuh"

namespace mom6b {

bool vertvisc_fast_fits(const Dims& D) { return D.nk >= 1; }

cudaError_t launch_vertvisc_fast(const Dims& D, const Metrics& M, double* u, double* v,
                                 const double* h, double dt, const VVParams& P,
                                 double* taux_bot, double* tauy_bot, cudaStream_t s)
{
    return launch_vertvisc_pf_t<double, double, true>(D, M, u, v, h, dt, P, taux_bot, tauy_bot,
                                                      s);
}

cudaError_t launch_vertvisc_fast_f(const Dims& D, const Metrics& M, float* u, float* v,
                                   const float* h, double dt, const VVParams& P,
                                   double* taux_bot, double* tauy_bot, cudaStream_t s)
{
    return launch_vertvisc_pf_t<float, double, true>(D, M, u, v, h, dt, P, taux_bot, tauy_bot,
                                                     s);
}

} // namespace mom6b
