// vertvisc_impl.cuh -- the prefetching vertical viscosity kernel, templated
// on the storage type R of u, v and h, in which the coefficients and the
// tridiagonal elimination are computed: R = double is the bit-exact FP64
// form (k_vertvisc.cu); R = float is the mixed form (k_mixed.cu).  The
// system is diagonally dominant (every pivot is h + dt (Ray + a d1 + a_next)
// with nonnegative terms), so the FP32 elimination loses only a few units in
// the last place per layer; the bottom stress accumulates in double.
//
// Restates vert_visc_coef + vert_visc_apply of the serial module
// (mom6_vert_visc_serial.F90:138-287 and :394-506) as the driver calls them
// (rk2_serial_driver.F90:276-277, :356-357).
#pragma once

#include <cstdlib>

#include "kernels.h"

namespace mom6b {

template <typename C>
__device__ __forceinline__ C vv_botfn(C z2) {
    return div_r(C(1.0), C(1.0) + C(0.09) * z2 * z2 * z2 * z2 * z2 * z2);
}

// Prefetching variant (the default): one per-column local array (botfn(z_i(m)),
// then c1(m)); h_harm is recomputed in sweep 2 from the same two thicknesses
// and the same expression, so it is bit-identical to the sweep-1 value.  The
// sweeps are latency-bound chains, so every sweep loads the inputs of CH
// layers into registers before it computes them: one memory latency per CH
// layers instead of one per layer.
// Layers whose inputs one prefetch brings in.
constexpr int kVvChunk = 4;
// CTAs per SM the registers are held to, by storage type: measured fastest on
// B200 (FP64 6: 2.28 ms per step, no cap 2.50; FP32 10: 1.13 ms, 8: 1.23,
// 12: 1.36).
template <typename R>
constexpr int vv_min_blocks() { return sizeof(R) == 4 ? 10 : 6; }

// The column of thread tx of the CTA with block coordinates (bx, by): row
// by of the interleaved u/v row list, column bx * blockDim.x + tx.
// REM (FP64): also the remnant of vert_visc_remnant (mom6_vert_visc_serial.F90
// :295-387) of every column into rem_u / rem_v -- the same elimination with
// h_u as the right-hand side, sharing b1, d1 and c1 with the velocity's;
// 1 in masked columns.
// ASYNC: sweeps 1 and 2 stage the next chunk's h, h(neighbour) and velocity
// in shared memory with cp.async (per-thread slots of stage, [2][CH][3][128])
// while the current chunk is computed, instead of loading each chunk into
// registers before computing it.  The arithmetic is unchanged.
template <int KMAX, int CH, typename R, bool REM = false, bool ASYNC = false>
__device__ __forceinline__ void
vertvisc_column(const Dims& D, const Metrics& M, R* __restrict__ u, R* __restrict__ v,
                const R* __restrict__ h, double dt, const VVParams& P,
                double* __restrict__ taux_bot, double* __restrict__ tauy_bot, int bx, int by,
                double* __restrict__ rem_u = nullptr, double* __restrict__ rem_v = nullptr,
                R* stage = nullptr)
{
    // Coefficients (h_harm, z_i, botfn, hvel, a(K)) and the tridiagonal
    // elimination (b1, d1, c1, the eliminated velocity and the back
    // substitution) are computed in the storage type R; the bottom stress
    // accumulates in double.
    using C = R;
    using E = R;
    E slot[KMAX + 2];   // botfn(z_i(m)), then c1(m)
    const int nz = D.nk;
    // Rows are interleaved so that the u row j and the v rows j-1, j, which
    // read the same rows of h, run close together: by = 0 is the v
    // row js-1, then u row js+q at 1+2q and v row js+q at 2+2q.
    const int yb = by;
    const bool is_u = yb >= 1 && ((yb - 1) & 1) == 0;
    const int q = yb >= 1 ? (yb - 1) >> 1 : -1;
    int i, j, di, dj;
    R* vel;
    const double *mask, *tau, *Ray;
    const unsigned char* ray_on;
    double* tbot;
    if (is_u) {  // u columns: I in [is-1, ie], j in [js, je]
        j = D.js + q;
        i = D.is - 1 + bx * (int)blockDim.x + (int)threadIdx.x;
        if (i > D.ie) return;
        di = 1; dj = 0;
        vel = u; mask = M.mask2dCu; tau = M.taux; Ray = M.Ray_u;
        ray_on = M.ray_layer_u; tbot = taux_bot;
    } else {     // v columns: i in [is, ie], J in [js-1, je]
        j = D.js + q;
        i = D.is + bx * (int)blockDim.x + (int)threadIdx.x;
        if (i > D.ie) return;
        di = 0; dj = 1;
        vel = v; mask = M.mask2dCv; tau = M.tauy; Ray = M.Ray_v;
        ray_on = M.ray_layer_v; tbot = tauy_bot;
    }
    const double msk = MOM6B_A2(mask, i, j, D);
    const size_t plane = (size_t)D.plane;
    double* rcol = nullptr;
    if constexpr (REM) rcol = (is_u ? rem_u : rem_v) + (size_t)(j - 1) * D.n1 + (i - 1);
    if (!(msk > 0.0)) {  // vert_visc_apply leaves masked columns alone
        if constexpr (REM)
            for (int k = 1; k <= D.nk; ++k) rcol[(size_t)(k - 1) * plane] = 1.0;
        return;
    }

    const R* hc = h + (size_t)(j - 1) * D.n1 + (i - 1);               // h(i, j, 1)
    const R* hn_ = h + (size_t)(j - 1 + dj) * D.n1 + (i - 1 + di);     // neighbour
    R* vc = vel + (size_t)(j - 1) * D.n1 + (i - 1);
    const double* rc = Ray + (size_t)(j - 1) * D.n1 + (i - 1);
    const C hn = (C)P.h_neglect, I_Hbbl = (C)P.I_Hbbl, Kv = (C)P.Kv, Kv_ml = (C)P.Kv_ml;
    const C Kv_extra_bbl = (C)P.Kv_extra_bbl, Hmix = (C)P.Hmix;

    // ---- sweep 1: h_harm and z_i bottom-up (vert_visc_coef :160-179) -----
    // stage slot (b, c, f) of this thread
    const int tid = (int)threadIdx.x;
    auto ST = [&](int b, int c, int f) -> R& { return stage[((b * CH + c) * 3 + f) * 128 + tid]; };
    C z = C(0.0);
    slot[nz + 1] = vv_botfn(C(0.0));
    auto stage1 = [&](int kt, int b) {
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int k = kt - c;
            const bool ok = k >= 2;
            const size_t o = ok ? (size_t)(k - 1) * plane : 0;
            cp_async_elem(&ST(b, c, 0), hc + o, ok);
            cp_async_elem(&ST(b, c, 1), hn_ + o, ok);
        }
        cp_async_commit();
    };
    if constexpr (ASYNC) {
        if (nz >= 2) stage1(nz, 0);
    }
    for (int kt = nz, it = 0; kt >= 2; kt -= CH, ++it) {
        C a0[CH], a1[CH];
        if constexpr (ASYNC) {
            const int b = it & 1;
            if (kt - CH >= 2) {
                stage1(kt - CH, b ^ 1);
                cp_async_wait_prior();
            } else {
                cp_async_wait_all();
            }
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                a0[c] = ST(b, c, 0);
                a1[c] = ST(b, c, 1);
            }
        } else {
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt - c;
            if (k >= 2) {
                a0[c] = hc[(size_t)(k - 1) * plane];
                a1[c] = hn_[(size_t)(k - 1) * plane];
            }
        }
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt - c;
            if (k >= 2) {
                C h_harm = div_r(C(2.0) * a0[c] * a1[c], a0[c] + a1[c] + hn);
                z = z + h_harm * I_Hbbl;
                slot[k] = vv_botfn(z);
            }
        }
    }

    // hvel(k): harmonic mean, blended toward the arithmetic mean where the
    // flow opposes the thickness gradient (:162-177)
    // bf_up = botfn(z_i(k+1)) (slot k+1 of sweep 1)
    auto hvel = [&](C bf_up, C h0, C h1, C vk) -> C {
        C h_harm = div_r(C(2.0) * h0 * h1, h0 + h1 + hn);
        C hv = h_harm;
        if (vk * (h1 - h0) < C(0.0)) {
            C bf = bf_up;
            C h_arith = C(0.5) * (h1 + h0);
            hv = (C(1.0) - bf) * h_harm + bf * h_arith;
        }
        return hv;
    };
    // a(K2) for K2 in [2, nz] given the running z_top (:185-202)
    // bf_K2 = botfn(z_i(K2)) (slot K2 of sweep 1)
    auto a_of = [&](C bf_K2, C z_top, C hv_lo, C hv_up) -> C {
        C Kv_tot = Kv;
        if (z_top < Hmix) {
            C topfn = C(1.0) - div_r(z_top, Hmix);
            Kv_tot = Kv_tot + (Kv_ml - Kv) * topfn;
        }
        Kv_tot = Kv_tot + Kv_extra_bbl * bf_K2;
        C h_shear = C(0.5) * (hv_lo + hv_up + hn);
        return div_r(Kv_tot, h_shear);
    };
    const C a_bot_num = Kv + Kv_extra_bbl;

    // ---- sweep 2: coefficients + forward elimination, top-down -----------
    const E dtE = (E)dt;
    const E sfc_stress = (E)(dt / kRho0 * MOM6B_A2(tau, i, j, D) * msk);
    const E v1 = vc[0];
    C hv_k = hvel((C)slot[2], hc[0], hn_[0], (C)v1);
    C z_top = C(0.0);
    C hv_next, a_next;
    E vnext = E(0.0);                        // vel(k + 1) before elimination
    if (nz >= 2) {
        vnext = vc[plane];
        hv_next = hvel((C)slot[3], hc[plane], hn_[plane], (C)vnext);
        z_top = z_top + hv_k;
        a_next = a_of((C)slot[2], z_top, hv_next, hv_k);
    } else {
        hv_next = C(0.0);
        a_next = div_r(a_bot_num, C(0.5) * hv_k + hn);
    }
    E a_k = E(0.0);  // a(1) = 0, surface
    E Rayk = ray_on[0] ? (E)rc[0] : E(0.0);
    E h_u = (E)(hv_k + hn);
    E b_denom_1 = h_u + dtE * (Rayk + a_k);
    E b1 = div_r(E(1.0), b_denom_1 + dtE * (E)a_next);
    E d1 = b_denom_1 * b1;
    E u_prev = b1 * (h_u * v1 + sfc_stress);
    vc[0] = (R)u_prev;
    E r_prev = E(0.0);   // the remnant's eliminated value (REM)
    if constexpr (REM) {
        r_prev = b1 * h_u;
        rcol[0] = r_prev;
    }
    // sweep 2 stages h, h(neighbour) and vel of layer k + 1 for k in the
    // chunk; every staged layer is read before this thread overwrites it
    auto stage2 = [&](int kt, int b) {
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int k = kt + c;
            const bool ok = k < nz;
            const size_t o = ok ? (size_t)k * plane : 0;
            cp_async_elem(&ST(b, c, 0), hc + o, ok);
            cp_async_elem(&ST(b, c, 1), hn_ + o, ok);
            cp_async_elem(&ST(b, c, 2), (const R*)vc + o, ok);
        }
        cp_async_commit();
    };
    if constexpr (ASYNC) {
        if (nz >= 2) stage2(2, 0);
    }
    for (int kt = 2, it = 0; kt <= nz; kt += CH, ++it) {
        // layers kt .. kt+CH-1 are eliminated; they need h and vel of the
        // layer below each (k + 1) and Ray of k
        // and botfn of interfaces k+1, k+2 (slots kt+1 .. kt+CH+1, read
        // before this chunk overwrites slots kt .. kt+CH-1 with c1)
        C p0[CH], p1[CH], pb[CH + 1];
        E pv[CH], pr[CH];
        if constexpr (ASYNC) {
            const int b = it & 1;
            if (kt + CH <= nz) {
                stage2(kt + CH, b ^ 1);
                cp_async_wait_prior();
            } else {
                cp_async_wait_all();
            }
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const int k = kt + c;
                p0[c] = ST(b, c, 0);
                p1[c] = ST(b, c, 1);
                pv[c] = (E)ST(b, c, 2);
                if (k <= nz) pr[c] = ray_on[k - 1] ? (E)rc[(size_t)(k - 1) * plane] : E(0.0);
            }
        } else {
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt + c;
            if (k < nz) {
                p0[c] = hc[(size_t)k * plane];
                p1[c] = hn_[(size_t)k * plane];
                pv[c] = vc[(size_t)k * plane];
            }
            if (k <= nz) pr[c] = ray_on[k - 1] ? (E)rc[(size_t)(k - 1) * plane] : E(0.0);
        }
        }
#pragma unroll
        for (int c = 0; c <= CH; ++c)
            if (kt + 1 + c <= nz + 1) pb[c] = (C)slot[kt + 1 + c];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt + c;
            if (k <= nz) {
                const E vk = vnext;          // vel(k) before elimination
                a_k = (E)a_next;
                hv_k = hv_next;
                if (k < nz) {
                    vnext = pv[c];
                    hv_next = hvel(pb[c + 1], p0[c], p1[c], (C)vnext);
                    z_top = z_top + hv_k;
                    a_next = a_of(pb[c], z_top, hv_next, hv_k);
                } else {
                    a_next = div_r(a_bot_num, C(0.5) * hv_k + hn);
                }
                Rayk = pr[c];
                E c1 = dtE * a_k * b1;
                slot[k] = c1;
                h_u = (E)(hv_k + hn);
                b_denom_1 = h_u + dtE * (Rayk + a_k * d1);
                b1 = div_r(E(1.0), b_denom_1 + dtE * (E)a_next);
                d1 = b_denom_1 * b1;
                u_prev = (h_u * vk + dtE * a_k * u_prev) * b1;
                vc[(size_t)(k - 1) * plane] = (R)u_prev;
                if constexpr (REM) {
                    r_prev = (h_u + dtE * a_k * r_prev) * b1;
                    rcol[(size_t)(k - 1) * plane] = r_prev;
                }
            }
        }
    }
    const double a_bottom = (double)a_next;

    // ---- sweep 3: back substitution (:447-449) ----------------------------
    E u_below = u_prev;
    E r_below = r_prev;
    for (int kt = nz - 1; kt >= 1; kt -= CH) {
        E pv[CH], pc[CH], pr2[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt - c;
            if (k >= 1) {
                pv[c] = vc[(size_t)(k - 1) * plane];
                pc[c] = slot[k + 1];
                if constexpr (REM) pr2[c] = rcol[(size_t)(k - 1) * plane];
            }
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt - c;
            if (k >= 1) {
                E uk = pv[c] + pc[c] * u_below;
                vc[(size_t)(k - 1) * plane] = (R)uk;
                u_below = uk;
                if constexpr (REM) {
                    const E rk = pr2[c] + pc[c] * r_below;
                    rcol[(size_t)(k - 1) * plane] = rk;
                    r_below = rk;
                }
            }
        }
    }
    // bottom stress (:452-458)
    double tb = kRho0 * (double)u_prev * a_bottom;
    for (int k = 1; k <= nz; ++k)
        if (ray_on[k - 1]) {
            size_t o = (size_t)(k - 1) * plane;
            tb = tb + kRho0 * rc[o] * (double)vc[o];
        }
    tbot[(size_t)(j - 1) * D.n1 + (i - 1)] = tb;
}

// MINB: the CTAs per SM the register allocation is held to.
template <int KMAX, int CH, typename R, int MINB = 1, bool REM = false, bool ASYNC = false>
__global__ void __launch_bounds__(128, MINB)
k_vertvisc_pf(Dims D, Metrics M, R* __restrict__ u, R* __restrict__ v,
              const R* __restrict__ h, double dt, VVParams P,
              double* __restrict__ taux_bot, double* __restrict__ tauy_bot,
              double* __restrict__ rem_u = nullptr, double* __restrict__ rem_v = nullptr)
{
    __shared__ R stage[ASYNC ? 2 * CH * 3 * 128 : 1];
    vertvisc_column<KMAX, CH, R, REM, ASYNC>(D, M, u, v, h, dt, P, taux_bot, tauy_bot,
                                             (int)blockIdx.x, (int)blockIdx.y, rem_u, rem_v,
                                             stage);
}

template <int KMAX, typename R>
static cudaError_t launch_vv_pf(const Dims& D, const Metrics& M, R* u, R* v, const R* h,
                                double dt, const VVParams& P, double* taux_bot,
                                double* tauy_bot, cudaStream_t s, double* rem_u = nullptr,
                                double* rem_v = nullptr)
{
    const int nb = 128;
    int ncol = D.ie - D.is + 2;
    int nrows = (D.je - D.js + 1) + (D.je - D.js + 2);
    dim3 grid((ncol + nb - 1) / nb, nrows, 1);
    static int chunk = -1, minb = -1, async = -1;
    if (chunk < 0) {
        const char* e = getenv("MOM6B_VV_CHUNK");
        chunk = e ? atoi(e) : kVvChunk;
        const char* b = getenv("MOM6B_VV_MINB");
        minb = b ? atoi(b) : vv_min_blocks<R>();
        // staged sweeps: FP64 2.215 ms per step against 2.285 loaded into
        // registers (chunks of 6 layers: 3.11, spilling); the FP32 form is
        // faster loading into registers (1.02 against 1.10-1.14 ms)
        const char* a = getenv("MOM6B_VV_ASYNC");
        async = a ? atoi(a) : (sizeof(R) == 8 ? 6 : 0);
    }
    if (async && !rem_u) {
        // staged sweeps, the register cap by the async minb
        if (async == 8)
            k_vertvisc_pf<KMAX, 4, R, 8, false, true><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P,
                                                                        taux_bot, tauy_bot);
        else if (async == 4)
            k_vertvisc_pf<KMAX, 4, R, 4, false, true><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P,
                                                                        taux_bot, tauy_bot);
        else if (async == 10 && sizeof(R) == 4)
            k_vertvisc_pf<KMAX, 4, R, 10, false, true><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P,
                                                                         taux_bot, tauy_bot);
        else
            k_vertvisc_pf<KMAX, 4, R, 6, false, true><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P,
                                                                        taux_bot, tauy_bot);
        return cudaGetLastError();
    }
    if constexpr (sizeof(R) == 8) {
        if (rem_u) {   // with the remnant (the FP64 form's register cap)
            if (async)
                k_vertvisc_pf<KMAX, 4, R, 6, true, true><<<grid, nb, 0, s>>>(
                    D, M, u, v, h, dt, P, taux_bot, tauy_bot, rem_u, rem_v);
            else
                k_vertvisc_pf<KMAX, 4, R, 6, true><<<grid, nb, 0, s>>>(
                    D, M, u, v, h, dt, P, taux_bot, tauy_bot, rem_u, rem_v);
            return cudaGetLastError();
        }
    }
    if (chunk == 2)
        k_vertvisc_pf<KMAX, 2, R><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    else if (chunk == 8)
        k_vertvisc_pf<KMAX, 8, R><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    else if (minb == 6)
        k_vertvisc_pf<KMAX, 4, R, 6><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    else if (minb == 8)
        k_vertvisc_pf<KMAX, 4, R, 8><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    else if (minb == 10 && sizeof(R) == 4)
        k_vertvisc_pf<KMAX, 4, R, 10><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    else if (minb == 12 && sizeof(R) == 4)
        k_vertvisc_pf<KMAX, 4, R, 12><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    else
        k_vertvisc_pf<KMAX, 4, R><<<grid, nb, 0, s>>>(D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    return cudaGetLastError();
}

// rem_u, rem_v (FP64, both or neither): also the vertical-viscosity remnant.
template <typename R>
cudaError_t launch_vertvisc_pf_t(const Dims& D, const Metrics& M, R* u, R* v, const R* h,
                                 double dt, const VVParams& P, double* taux_bot,
                                 double* tauy_bot, cudaStream_t s, double* rem_u = nullptr,
                                 double* rem_v = nullptr)
{
    if ((rem_u == nullptr) != (rem_v == nullptr)) return cudaErrorInvalidValue;
    if (D.nk <= 80) return launch_vv_pf<80>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u, rem_v);
    if (D.nk <= 128) return launch_vv_pf<128>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u, rem_v);
    if (D.nk <= 256) return launch_vv_pf<256>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u, rem_v);
    return launch_vv_pf<1024>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u, rem_v);
}

} // namespace mom6b
