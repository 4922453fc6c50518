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

#include "kernels.h"

namespace mom6b {

__device__ __forceinline__ double vv_botfn(double z2) {
    return 1.0 / (1.0 + 0.09 * z2 * z2 * z2 * z2 * z2 * z2);
}

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

// Prefetching variant (the default): one per-column local array (botfn(z_i(m)),
// then c1(m)); h_harm is recomputed in sweep 2 from the same two thicknesses
// and the same expression, so it is bit-identical to the sweep-1 value.  The
// sweeps are latency-bound chains, so every sweep loads the inputs of CH
// layers into registers before it computes them: one memory latency per CH
// layers instead of one per layer.
// Layers whose inputs one prefetch brings in.
constexpr int kVvChunk = 4;

template <int KMAX, int CH>
__global__ void __launch_bounds__(128)
k_vertvisc_pf(Dims D, Metrics M, double* __restrict__ u, double* __restrict__ v,
              const double* __restrict__ h, double dt, VVParams P,
              double* __restrict__ taux_bot, double* __restrict__ tauy_bot)
{
    double slot[KMAX + 2];   // botfn(z_i(m)), then c1(m)
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

    const size_t plane = (size_t)D.plane;
    const double* hc = h + (size_t)(j - 1) * D.n1 + (i - 1);          // h(i, j, 1)
    const double* hn_ = h + (size_t)(j - 1 + dj) * D.n1 + (i - 1 + di); // neighbour
    double* vc = vel + (size_t)(j - 1) * D.n1 + (i - 1);
    const double* rc = Ray + (size_t)(j - 1) * D.n1 + (i - 1);
    const double hn = P.h_neglect;

    // ---- sweep 1: h_harm and z_i bottom-up (vert_visc_coef :160-179) -----
    double z = 0.0;
    slot[nz + 1] = vv_botfn(0.0);
    for (int kt = nz; kt >= 2; kt -= CH) {
        double a0[CH], a1[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt - c;
            if (k >= 2) {
                a0[c] = hc[(size_t)(k - 1) * plane];
                a1[c] = hn_[(size_t)(k - 1) * plane];
            }
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt - c;
            if (k >= 2) {
                double h_harm = 2.0 * a0[c] * a1[c] / (a0[c] + a1[c] + hn);
                z = z + h_harm * P.I_Hbbl;
                slot[k] = vv_botfn(z);
            }
        }
    }

    // hvel(k): harmonic mean, blended toward the arithmetic mean where the
    // flow opposes the thickness gradient (:162-177)
    auto hvel = [&](int k, double h0, double h1, double vk) -> double {
        double h_harm = 2.0 * h0 * h1 / (h0 + h1 + hn);
        double hv = h_harm;
        if (vk * (h1 - h0) < 0.0) {
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
    const double v1 = vc[0];
    double hv_k = hvel(1, hc[0], hn_[0], v1);
    double z_top = 0.0;
    double hv_next, a_next;
    double vnext = 0.0;                      // vel(k + 1) before elimination
    if (nz >= 2) {
        vnext = vc[plane];
        hv_next = hvel(2, hc[plane], hn_[plane], vnext);
        z_top = z_top + hv_k;
        a_next = a_of(2, z_top, hv_next, hv_k);
    } else {
        hv_next = 0.0;
        a_next = a_bot_num / (0.5 * hv_k + hn);
    }
    double a_k = 0.0;  // a(1) = 0, surface
    double Rayk = ray_on[0] ? rc[0] : 0.0;
    double h_u = hv_k + hn;
    double b_denom_1 = h_u + dt * (Rayk + a_k);
    double b1 = 1.0 / (b_denom_1 + dt * a_next);
    double d1 = b_denom_1 * b1;
    double u_prev = b1 * (h_u * v1 + sfc_stress);
    vc[0] = u_prev;
    for (int kt = 2; kt <= nz; kt += CH) {
        // layers kt .. kt+CH-1 are eliminated; they need h and vel of the
        // layer below each (k + 1) and Ray of k
        double p0[CH], p1[CH], pv[CH], pr[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt + c;
            if (k < nz) {
                p0[c] = hc[(size_t)k * plane];
                p1[c] = hn_[(size_t)k * plane];
                pv[c] = vc[(size_t)k * plane];
            }
            if (k <= nz) pr[c] = ray_on[k - 1] ? rc[(size_t)(k - 1) * plane] : 0.0;
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt + c;
            if (k <= nz) {
                const double vk = vnext;     // vel(k) before elimination
                a_k = a_next;
                hv_k = hv_next;
                if (k < nz) {
                    vnext = pv[c];
                    hv_next = hvel(k + 1, p0[c], p1[c], vnext);
                    z_top = z_top + hv_k;
                    a_next = a_of(k + 1, z_top, hv_next, hv_k);
                } else {
                    a_next = a_bot_num / (0.5 * hv_k + hn);
                }
                Rayk = pr[c];
                double c1 = dt * a_k * b1;
                slot[k] = c1;
                h_u = hv_k + hn;
                b_denom_1 = h_u + dt * (Rayk + a_k * d1);
                b1 = 1.0 / (b_denom_1 + dt * a_next);
                d1 = b_denom_1 * b1;
                u_prev = (h_u * vk + dt * a_k * u_prev) * b1;
                vc[(size_t)(k - 1) * plane] = u_prev;
            }
        }
    }
    const double a_bottom = a_next;

    // ---- sweep 3: back substitution (:447-449) ----------------------------
    double u_below = u_prev;
    for (int kt = nz - 1; kt >= 1; kt -= CH) {
        double pv[CH], pc[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt - c;
            if (k >= 1) {
                pv[c] = vc[(size_t)(k - 1) * plane];
                pc[c] = slot[k + 1];
            }
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt - c;
            if (k >= 1) {
                double uk = pv[c] + pc[c] * u_below;
                vc[(size_t)(k - 1) * plane] = uk;
                u_below = uk;
            }
        }
    }
    // bottom stress (:452-458)
    double tb = kRho0 * u_prev * a_bottom;
    for (int k = 1; k <= nz; ++k)
        if (ray_on[k - 1]) {
            size_t o = (size_t)(k - 1) * plane;
            tb = tb + kRho0 * rc[o] * vc[o];
        }
    tbot[(size_t)(j - 1) * D.n1 + (i - 1)] = tb;
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

template <int KMAX>
static cudaError_t launch_vv_pf(const Dims& D, const Metrics& M, double* u, double* v,
                                const double* h, double dt, const VVParams& P,
                                double* taux_bot, double* tauy_bot, cudaStream_t s)
{
    const int nb = 128;
    int ncol = D.ie - D.is + 2;
    int nrows = (D.je - D.js + 1) + (D.je - D.js + 2);
    dim3 grid((ncol + nb - 1) / nb, nrows, 1);
    static int chunk = -1;
    if (chunk < 0) {
        const char* e = getenv("MOM6B_VV_CHUNK");
        chunk = e ? atoi(e) : kVvChunk;
    }
    if (chunk == 2)
        k_vertvisc_pf<KMAX, 2><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    else if (chunk == 8)
        k_vertvisc_pf<KMAX, 8><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    else
        k_vertvisc_pf<KMAX, 4><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    return cudaGetLastError();
}

cudaError_t launch_vertvisc(const Dims& D, const Metrics& M, double* u, double* v,
                            const double* h, double dt, const VVParams& P,
                            double* taux_bot, double* tauy_bot, cudaStream_t s)
{
    if (!getenv("MOM6B_VV_LOCAL")) {
        if (D.nk <= 80) return launch_vv_pf<80>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
        if (D.nk <= 128) return launch_vv_pf<128>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
        if (D.nk <= 256) return launch_vv_pf<256>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
        return launch_vv_pf<1024>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
    }
    if (D.nk <= 80) return launch_vv<80>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
    if (D.nk <= 128) return launch_vv<128>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
    if (D.nk <= 256) return launch_vv<256>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
    return launch_vv<1024>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s);
}

} // namespace mom6b
