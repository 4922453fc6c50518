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


// One thread per column.  KMAX bounds nk at compile time so that the two
// per-column scratch arrays live in local memory: the hardware interleaves
// local memory across the threads of a warp, so slot m of 32 consecutive
// columns is one contiguous 256-byte segment, cached in L1/L2.  The grid is
// blockDim.x columns along i by one row: blockIdx.y enumerates u rows then
// v rows.
template <int KMAX>
__global__ void __launch_bounds__(256)
k_vertvisc(Dims D, Metrics M, double* __restrict__ u, double* __restrict__ v,
           const double* __restrict__ h, double dt, VVParams P,
           double* __restrict__ taux_bot, double* __restrict__ tauy_bot)
{
    double slot[KMAX + 2];   // botfn(z_i(m)), then c1(m)
    double hh[KMAX + 2];     // h_harm(k) from sweep 1, reused in sweep 2
    const int nz = D.nk;
    const int nrow_u = D.je - D.js + 1;
    bool is_u = (int)blockIdx.y < nrow_u;
    int i, j, di, dj;
    double* vel;
    const double *mask, *tau, *Ray;
    const unsigned char* ray_on;
    double* tbot;
    if (is_u) {  // u columns: I in [is-1, ie], j in [js, je]
        j = D.js + (int)blockIdx.y;
        i = D.is - 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
        if (i > D.ie) return;
        di = 1; dj = 0;
        vel = u; mask = M.mask2dCu; tau = M.taux; Ray = M.Ray_u;
        ray_on = M.ray_layer_u; tbot = taux_bot;
    } else {     // v columns: i in [is, ie], J in [js-1, je]
        j = D.js - 1 + ((int)blockIdx.y - nrow_u);
        i = D.is + (int)(blockIdx.x * blockDim.x + threadIdx.x);
        if (i > D.ie) return;
        di = 0; dj = 1;
        vel = v; mask = M.mask2dCv; tau = M.tauy; Ray = M.Ray_v;
        ray_on = M.ray_layer_v; tbot = tauy_bot;
    }
    const double msk = MOM6B_A2(mask, i, j, D);
    if (!(msk > 0.0)) return;  // vert_visc_apply leaves masked columns alone

    const size_t col = (size_t)(j - 1) * D.n1 + (i - 1);
    const size_t nbr = (size_t)(j - 1 + dj) * D.n1 + (i - 1 + di);
    const size_t plane = (size_t)D.plane;
    const double hn = P.h_neglect;

    // ---- sweep 1: h_harm and z_i bottom-up (vert_visc_coef :160-179) -----
    double z = 0.0;
    slot[nz + 1] = vv_botfn(0.0);
    for (int k = nz; k >= 1; --k) {
        size_t o = (size_t)(k - 1) * plane;
        double h0 = h[o + col], h1 = h[o + nbr];
        double h_harm = 2.0 * h0 * h1 / (h0 + h1 + hn);
        hh[k] = h_harm;
        if (k >= 2) {
            z = z + h_harm * P.I_Hbbl;
            slot[k] = vv_botfn(z);
        }
    }

    // hvel(k): harmonic mean, blended toward the arithmetic mean where the
    // flow opposes the thickness gradient (:162-177)
    auto hvel_of = [&](int k) -> double {
        size_t o = (size_t)(k - 1) * plane;
        double h0 = h[o + col], h1 = h[o + nbr];
        double h_harm = hh[k];
        double hv = h_harm;
        if (vel[o + col] * (h1 - h0) < 0.0) {
            double bf = slot[k + 1];
            double h_arith = 0.5 * (h1 + h0);
            hv = (1.0 - bf) * h_harm + bf * h_arith;
        }
        return hv;
    };
    // a(K2) for K2 in [2, nz] given the running z_top (:185-202)
    auto a_of = [&](int K2, double z_top, double hv_lo, double hv_up) -> double {
        double Kv_tot = P.Kv;
        if (z_top < P.Hmix) {
            double topfn = 1.0 - z_top / P.Hmix;
            Kv_tot = Kv_tot + (P.Kv_ml - P.Kv) * topfn;
        }
        Kv_tot = Kv_tot + P.Kv_extra_bbl * slot[K2];
        double h_shear = 0.5 * (hv_lo + hv_up + hn);
        return Kv_tot / h_shear;
    };
    const double a_bot_num = P.Kv + P.Kv_extra_bbl;

    // ---- sweep 2: coefficients + forward elimination, top-down -----------
    const double dt_Rho0 = dt / kRho0;
    const double sfc_stress = dt_Rho0 * MOM6B_A2(tau, i, j, D) * msk;
    double hv_k = hvel_of(1);
    double z_top = 0.0;
    double hv_next, a_next;
    if (nz >= 2) {
        hv_next = hvel_of(2);
        z_top = z_top + hv_k;
        a_next = a_of(2, z_top, hv_next, hv_k);
    } else {
        hv_next = 0.0;
        a_next = a_bot_num / (0.5 * hv_k + hn);
    }
    double a_k = 0.0;  // a(1) = 0, surface
    double Rayk = ray_on[0] ? Ray[col] : 0.0;
    double h_u = hv_k + hn;
    double b_denom_1 = h_u + dt * (Rayk + a_k);
    double b1 = 1.0 / (b_denom_1 + dt * a_next);
    double d1 = b_denom_1 * b1;
    double u_prev = b1 * (h_u * vel[col] + sfc_stress);
    vel[col] = u_prev;
    for (int k = 2; k <= nz; ++k) {
        a_k = a_next;
        hv_k = hv_next;
        if (k < nz) {
            hv_next = hvel_of(k + 1);
            z_top = z_top + hv_k;
            a_next = a_of(k + 1, z_top, hv_next, hv_k);
        } else {
            a_next = a_bot_num / (0.5 * hv_k + hn);
        }
        size_t o = (size_t)(k - 1) * plane + col;
        Rayk = ray_on[k - 1] ? Ray[o] : 0.0;
        double c1 = dt * a_k * b1;
        slot[k] = c1;
        h_u = hv_k + hn;
        b_denom_1 = h_u + dt * (Rayk + a_k * d1);
        b1 = 1.0 / (b_denom_1 + dt * a_next);
        d1 = b_denom_1 * b1;
        u_prev = (h_u * vel[o] + dt * a_k * u_prev) * b1;
        vel[o] = u_prev;
    }
    const double a_bottom = a_next;

    // ---- sweep 3: back substitution (:447-449) ----------------------------
    double u_below = u_prev;
    for (int k = nz - 1; k >= 1; --k) {
        size_t o = (size_t)(k - 1) * plane + col;
        double uk = vel[o] + slot[k + 1] * u_below;
        vel[o] = uk;
        u_below = uk;
    }
    // bottom stress (:452-458)
    double tb = kRho0 * u_prev * a_bottom;
    for (int k = 1; k <= nz; ++k)
        if (ray_on[k - 1]) {
            size_t o = (size_t)(k - 1) * plane + col;
            tb = tb + kRho0 * Ray[o] * vel[o];
        }
    tbot[col] = tb;
}

template <int KMAX>
static cudaError_t launch_vv(const Dims& D, const Metrics& M, double* u, double* v,
                             const double* h, double dt, const VVParams& P,
                             double* taux_bot, double* tauy_bot, cudaStream_t s)
{
    const int nb = 128;
    int ncol = D.ie - D.is + 2;  // u rows have one more column than v rows
    int nrows = (D.je - D.js + 1) + (D.je - D.js + 2);
    dim3 grid((ncol + nb - 1) / nb, nrows, 1);
    k_vertvisc<KMAX><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    return cudaGetLastError();
}

cudaError_t launch_vertvisc(const Dims& D, const Metrics& M, double* u, double* v,
                            const double* h, double dt, const VVParams& P,
                            double* taux_bot, double* tauy_bot, cudaStream_t s,
                            double* rem_u, double* rem_v)
{
    if (rem_u || !getenv("MOM6B_VV_LOCAL"))
        return launch_vertvisc_pf_t<double>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u,
                                            rem_v);
    if (D.nk <= 80) return launch_vv<80>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
    if (D.nk <= 128) return launch_vv<128>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
    if (D.nk <= 256) return launch_vv<256>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
    return launch_vv<1024>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
}

} // namespace mom6b
