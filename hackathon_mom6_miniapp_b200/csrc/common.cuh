// common.cuh -- shared definitions of the B200 split RK2 kernels.
//
// Layout: every field is the reference's Fortran array (n1, n2[, nk]),
// column-major, 1-based (mom6_types.F90:145-148).  Kernels index with the
// reference's 1-based (i, j, k) so that loop ranges can be compared with the
// Fortran line for line; A2/A3 subtract the 1.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mom6b {

// Grid metrics and static fields on the device.  Every pointer addresses an
// (n1, n2) array of doubles, except f_4_u / f_4_v which are (4, n1, n2)
// (mom6_barotropic_serial.F90:97-98).
struct Metrics {
    const double *IareaT, *areaT, *dxT, *IdxT, *dxCu, *dyCu, *dy_Cu, *IdxCu,
        *IdyCu, *dxCv, *dyCv, *IdxCv, *IdyCv, *IareaBu, *CoriolisBu, *IareaCu,
        *IareaCv, *mask2dT, *mask2dBu, *mask2dCu, *mask2dCv;
    // derived at initialisation exactly as hor_visc_init / coriolis_init do
    const double *Area_q, *DX_dyT, *DY_dxT, *DX_dyBu, *DY_dxBu, *dx2h, *dy2h,
        *dx2q, *dy2q, *red_xx, *red_xy, *Kh_xx, *Kh_xy;
    // barotropic_init (mom6_barotropic_serial.F90:106-133)
    const double *Datu, *Datv, *gtot_E, *gtot_W, *gtot_N, *gtot_S, *f_4_u,
        *f_4_v, *bt_rem_u, *bt_rem_v;
    // forcing (rk2_serial_driver.F90:508-542)
    const double *taux, *tauy, *Ray_u, *Ray_v;
    const unsigned char *ray_layer_u, *ray_layer_v; // 1 where the layer is nonzero
    // meridional continuity
    const double *dyT, *IdyT;
};

struct Dims {
    int n1, n2, nk;
    int is, ie, js, je;   // compute domain, 1-based
    int isd, ied, jsd, jed;
    long long plane;      // n1 * n2
    // sides (west, east, south, north) where a decomposed run's neighbouring
    // subdomain lies: 1 at a cut, 0 at a wall or for the whole domain
    int cw = 0, ce = 0, cs = 0, cn = 0;
};

#define MOM6B_A2(a, i, j, D) (a)[(size_t)((j)-1) * (size_t)(D).n1 + (size_t)((i)-1)]
#define MOM6B_A3(a, i, j, k, D)                                                 \
    (a)[(size_t)((k)-1) * (size_t)(D).plane + (size_t)((j)-1) * (size_t)(D).n1 + \
        (size_t)((i)-1)]
#define MOM6B_F4(a, c, i, j, D)                                                 \
    (a)[(((size_t)((j)-1) * (size_t)(D).n1 + (size_t)((i)-1)) * 4) + (size_t)((c)-1)]

// Physical constants, mom6_types.F90:80-85.
constexpr double kGEarth = 9.80;
constexpr double kRho0 = 1035.0;

// Status flags written by kernels that can give up (grid barrier timeouts).
enum : int { kDevOk = 0, kDevTimeout = 1 };

// One element global -> shared with cp.async (bypasses registers); ok = false
// writes zero (src-size 0) and reads nothing.
template <typename R>
__device__ __forceinline__ void cp_async_elem(R* sdst, const R* gsrc, bool ok)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    if constexpr (sizeof(R) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gsrc),
                     "r"(ok ? 8 : 0)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(gsrc),
                     "r"(ok ? 4 : 0)
                     : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// the calling thread's copies except the most recent group are complete
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }

// a / b in the arithmetic type of a templated kernel: the IEEE quotient in
// double (the bit-exact forms), the fast reciprocal-based quotient (2 ulp) in
// float (the mixed form).
__device__ __forceinline__ double div_r(double a, double b) { return a / b; }
__device__ __forceinline__ float div_r(float a, float b) { return __fdividef(a, b); }

// a / b for the fast forms: the hardware's approximate reciprocal of b refined
// by two Newton-Raphson steps r <- r + r (1 - b r) (each doubles the correct
// bits), then the quotient corrected once by its residual, q <- q + r (a - b q)
// (Markstein's scheme).  Within about an ulp of the IEEE quotient; b must be
// a normal nonzero number (every use here divides by a positive thickness,
// viscosity or pivot).
__device__ __forceinline__ double div_nr(double a, double b)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(b));
    double e = fma(-b, r, 1.0);
    r = fma(r, e, r);
    e = fma(-b, r, 1.0);
    r = fma(r, e, r);
    const double q = a * r;
    return fma(r, fma(-b, q, a), q);
}

} // namespace mom6b
