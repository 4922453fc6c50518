// hor_visc.h -- the scheme branches of hor_visc (mom6_hor_visc_serial.F90)
// beyond the driver's constant-Kh Laplacian: parameters and launcher.
#pragma once

#include "kernels.h"

namespace mom6b {

// hor_visc_init's configuration (mom6_hor_visc_serial.F90:160-268).  The
// flags are the control structure's after init: smag_kh = Smagorinsky and
// Laplacian, smag_ah = Smagorinsky and biharmonic, leith_kh = Leith,
// leith_ah = Leith and biharmonic; bb stands for better_bound_Kh =
// better_bound_Ah = bound_Kh = bound_Ah, which init sets together.  The
// arrays are (n1, n2); the xx (h-point) and xy (q-point) constants of the
// reference are the same expressions of areaT and share one array each.
struct HorViscGen {
    int lap, bih, smag_kh, smag_ah, leith_kh, leith_ah, no_slip, bb, mod_leith;
    double Kh_bg, Ah_bg, Kh_bg_min, h_neglect;
    const double *Kh_Max, *Ah_Max, *L2c, *Bc, *L3c, *B6c;
    const double *Idx2dyCu, *Idxdy2u, *Idx2dyCv, *Idxdy2v;
    // the same arrays as scalars, when uni = 1 (every one of them and every
    // grid metric uniform over the points the kernel reads)
    int uni;
    double sKh_Max, sAh_Max, sL2c, sBc, sL3c, sB6c, sIdx2dyCu, sIdxdy2u, sIdx2dyCv, sIdxdy2v;
};

// diffu on [is, ie-1] x [js, je] and diffv on [is, ie] x [js, je-1], every
// layer, from u, v, h: the points the velocity update reads.
cudaError_t launch_hor_visc_gen(const Dims& D, const Metrics& M, const UniMetrics& U,
                                const HorViscGen& P, const double* u, const double* v,
                                const double* h, double* diffu, double* diffv, cudaStream_t s);

} // namespace mom6b
