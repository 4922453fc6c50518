// k_vertvisc.cu -- vertical viscosity, one thread per water column (FP64).
//
// Restates vert_visc_coef + vert_visc_apply of the serial module
// (mom6_vert_visc_serial.F90:138-287 and :394-506) as the driver calls them
// (rk2_serial_driver.F90:276-277, :356-357): harmonic/upwind-blended face
// thickness, mixed-layer and bottom-boundary-layer viscosity profile, wind
// stress at the surface, Rayleigh drag, Schopf & Loughe forward elimination
// and back substitution, and the bottom stress output.
//
// Three sweeps per column, all in the reference's order:
//   1. bottom-up: h_harm and the running z_i; h_harm(k) and botfn(z_i(m))
//      are kept per layer/interface (the values the reference recomputes);
//   2. top-down: hvel, a(K) and the forward elimination; the eliminated
//      velocity is written back in place, and c1(k) overwrites the botfn slot
//      k, which is dead by then;
//   3. bottom-up: back substitution.
// The coefficient arrays a_u/h_u of the serial control structure are never
// materialised.  Layers in which the Rayleigh array is identically zero (a
// per-layer flag computed when the model is built) skip the Rayleigh loads;
// adding RHO_0*0*u is exact, so this changes no result.
#include <cstdlib>

#include "vertvisc_impl.cuh"

namespace mom6b {


cudaError_t launch_vertvisc(const Dims& D, const Metrics& M, double* u, double* v,
                            const double* h, double dt, const VVParams& P,
                            double* taux_bot, double* tauy_bot, cudaStream_t s,
                            double* rem_u, double* rem_v)
{
    return launch_vertvisc_pf_t<double>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u,
                                        rem_v);
}

} // namespace mom6b
