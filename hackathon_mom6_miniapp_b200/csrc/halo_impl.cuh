// halo_impl.cuh -- the single-GPU halo / boundary fill of one point.
//
// The reference's single-device drivers never fill halos (the MPI driver
// exchanges them, mom6_mpi_domain.F90:58-137); the configured beta-plane
// domain is periodic in i with solid walls in j, halo width 4, and the fill
// is applied to every prognostic field after each stencil phase, identically
// in the oracle.
#pragma once

#include "common.cuh"

namespace mom6b {

// Halo points per layer of a field of the given kind.
__host__ __device__ inline long long halo_points_per_layer(const Dims& D, int kind)
{
    const int lo_x = (kind == 1) ? D.is - 2 : D.is - 1;
    const int lo_y = (kind == 2) ? D.js - 2 : D.js - 1;
    const int nxh = lo_x + (D.n1 - D.ie), nyh = lo_y + (D.n2 - D.je);
    return (long long)nyh * D.n1 + (long long)nxh * (D.n2 - nyh);
}

// kind 0: h point, 1: u point (faces is-1 and ie are the basin walls and keep
// their values), 2: v point (antisymmetric about the wall faces js-1, je).
// Every halo value is read from non-halo points only, so one pass suffices.
template <typename T>
__device__ __forceinline__ void halo_fill_point(const Dims& D, T* f, int nz, int kind,
                                                long long t)
{
    const int is = D.is, ie = D.ie, js = D.js, je = D.je;
    const int P = ie - is + 1;
    const int lo_x = (kind == 1) ? is - 2 : is - 1;   // x halo: i <= lo_x or i > ie
    const int lo_y = (kind == 2) ? js - 2 : js - 1;   // y halo: j <= lo_y or j > je
    const int nxh = lo_x + (D.n1 - ie);               // halo columns
    const int nyh = lo_y + (D.n2 - je);               // halo rows
    // enumerate: halo rows (all i) first, then halo columns of the other rows
    const long long per_layer = (long long)nyh * D.n1 + (long long)nxh * (D.n2 - nyh);
    if (t >= per_layer * nz) return;
    const int k = (int)(t / per_layer) + 1;
    long long r = t % per_layer;
    int i, j;
    if (r < (long long)nyh * D.n1) {
        int row = (int)(r / D.n1);
        i = (int)(r % D.n1) + 1;
        j = row < lo_y ? row + 1 : je + 1 + (row - lo_y);
    } else {
        r -= (long long)nyh * D.n1;
        int col = (int)(r % nxh);
        j = lo_y + 1 + (int)(r / nxh);
        i = col < lo_x ? col + 1 : ie + 1 + (col - lo_x);
    }
    const bool xh = (i <= lo_x) || (i > ie);
    const bool yh = (j <= lo_y) || (j > je);
    int si = xh ? (i < is ? i + P : i - P) : i;
    int sj = j;
    double sgn = 1.0;
    if (yh) {
        if (kind == 2) {
            sj = (j < js) ? 2 * (js - 1) - j : 2 * je - j;
            sgn = -1.0;
        } else {
            sj = (j < js) ? 2 * js - 1 - j : 2 * je + 1 - j;
        }
    }
    T val = MOM6B_A3(f, si, sj, k, D);
    MOM6B_A3(f, i, j, k, D) = (sgn < 0.0) ? -val : val;
}

} // namespace mom6b
