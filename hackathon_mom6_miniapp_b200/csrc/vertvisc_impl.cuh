// vertvisc_impl.cuh -- the prefetching vertical viscosity kernel, templated
// on the storage type R of u, v and h, in which the coefficients are
// computed, and on the type E of the tridiagonal elimination: R = E = double
// is the bit-exact FP64 form (k_vertvisc.cu); R = float, E = double is the
// mixed form (k_mixed.cu: FP32 state and coefficients, FP64 elimination);
// R = E = float is the mixed form's opt-in all-FP32 variant.  The system is
// diagonally dominant (every pivot is h + dt (Ray + a d1 + a_next) with
// nonnegative terms), so even an FP32 elimination loses only a few units in
// the last place per layer; the bottom stress accumulates in double.
//
// Restates vert_visc_coef + vert_visc_apply of the serial module
// (mom6_vert_visc_serial.F90:138-287 and :394-506) as the driver calls them
// (rk2_serial_driver.F90:276-277, :356-357).
#pragma once

#include <cstdlib>

#include "kernels.h"

namespace mom6b {

template <bool FAST = false>
__device__ __forceinline__ double vv_div(double a, double b) {
    if constexpr (FAST) return div_nr(a, b);
    else return a / b;
}
template <bool FAST = false>
__device__ __forceinline__ float vv_div(float a, float b) { return div_r(a, b); }

template <bool FAST = false, typename C>
__device__ __forceinline__ C vv_botfn(C z2) {
    if constexpr (FAST) {
        const C zz = z2 * z2;
        return vv_div<true>(C(1.0), C(1.0) + C(0.09) * (zz * zz * zz));
    } else {
        return div_r(C(1.0), C(1.0) + C(0.09) * z2 * z2 * z2 * z2 * z2 * z2);
    }
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
template <typename R, typename E>
constexpr int vv_min_blocks() { return sizeof(R) == 8 ? 6 : (sizeof(E) == 8 ? 8 : 10); }

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
// FAST: the fast forms' arithmetic (built with FMA contraction): quotients
// by div_nr, and botfn(z_i) formed top-down from the column total Z = z_i(2)
// (z_i(K) = Z - the harmonic thickness above K; z_i(nz+1) = 0) instead of
// being stored by sweep 1, so the per-column local array holds c1 only.
template <int KMAX, int CH, typename R, typename E, bool REM = false, bool ASYNC = false,
          bool FAST = false>
__device__ __forceinline__ void
vertvisc_column(const Dims& D, const Metrics& M, R* __restrict__ u, R* __restrict__ v,
                const R* __restrict__ h, double dt, const VVParams& P,
                double* __restrict__ taux_bot, double* __restrict__ tauy_bot, int bx, int by,
                double* __restrict__ rem_u = nullptr, double* __restrict__ rem_v = nullptr,
                R* stage = nullptr)
{
    // Coefficients (h_harm, z_i, botfn, hvel, a(K)) are computed in the
    // storage type R, the tridiagonal elimination (b1, d1, c1, the
    // eliminated velocity and the back substitution) in E; the bottom stress
    // accumulates in double.
    using C = R;
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
    if constexpr (!FAST) slot[nz + 1] = vv_botfn(C(0.0));
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
                C h_harm = vv_div<FAST>(C(2.0) * a0[c] * a1[c], a0[c] + a1[c] + hn);
                z = z + h_harm * I_Hbbl;
                if constexpr (!FAST) slot[k] = vv_botfn(z);
            }
        }
    }

    // hvel(k): harmonic mean, blended toward the arithmetic mean where the
    // flow opposes the thickness gradient (:162-177)
    // bf_up = botfn(z_i(k+1)) (slot k+1 of sweep 1)
    auto harm = [&](C h0, C h1) -> C { return vv_div<FAST>(C(2.0) * h0 * h1, h0 + h1 + hn); };
    auto hvel_h = [&](C bf_up, C h_harm, C h0, C h1, C vk) -> C {
        C hv = h_harm;
        if (vk * (h1 - h0) < C(0.0)) {
            C bf = bf_up;
            C h_arith = C(0.5) * (h1 + h0);
            hv = (C(1.0) - bf) * h_harm + bf * h_arith;
        }
        return hv;
    };
    auto hvel = [&](C bf_up, C h0, C h1, C vk) -> C {
        return hvel_h(bf_up, harm(h0, h1), h0, h1, vk);
    };
    // a(K2) for K2 in [2, nz] given the running z_top (:185-202)
    // bf_K2 = botfn(z_i(K2)) (slot K2 of sweep 1)
    auto a_of = [&](C bf_K2, C z_top, C hv_lo, C hv_up) -> C {
        C Kv_tot = Kv;
        if (z_top < Hmix) {
            C topfn = C(1.0) - vv_div<FAST>(z_top, Hmix);
            Kv_tot = Kv_tot + (Kv_ml - Kv) * topfn;
        }
        Kv_tot = Kv_tot + Kv_extra_bbl * bf_K2;
        C h_shear = C(0.5) * (hv_lo + hv_up + hn);
        return vv_div<FAST>(Kv_tot, h_shear);
    };
    const C a_bot_num = Kv + Kv_extra_bbl;

    // ---- sweep 2: coefficients + forward elimination, top-down -----------
    const E dtE = (E)dt;
    const E sfc_stress = (E)(dt / kRho0 * MOM6B_A2(tau, i, j, D) * msk);
    const E v1 = vc[0];
    // FAST: zi is z_i(m) of the deepest interface m whose botfn is formed,
    // bf_cur = botfn(z_i(k + 1)) for the layer k about to be eliminated
    C zi = z, bf_cur = C(0.0);
    const C bf2 = FAST ? vv_botfn<FAST>(zi) : C(0.0);
    C bf_first;
    if constexpr (FAST) bf_first = bf2;
    else bf_first = (C)slot[2];
    C hv_k = hvel(bf_first, hc[0], hn_[0], (C)v1);
    C z_top = C(0.0);
    C hv_next, a_next;
    E vnext = E(0.0);                        // vel(k + 1) before elimination
    if (nz >= 2) {
        vnext = vc[plane];
        if constexpr (FAST) {
            const C h0 = hc[plane], h1 = hn_[plane];
            const C hh = harm(h0, h1);
            zi = nz >= 3 ? zi - hh * I_Hbbl : C(0.0);          // z_i(3)
            bf_cur = vv_botfn<FAST>(zi);
            hv_next = hvel_h(bf_cur, hh, h0, h1, (C)vnext);
            z_top = z_top + hv_k;
            a_next = a_of(bf2, z_top, hv_next, hv_k);
        } else {
            hv_next = hvel((C)slot[3], hc[plane], hn_[plane], (C)vnext);
            z_top = z_top + hv_k;
            a_next = a_of((C)slot[2], z_top, hv_next, hv_k);
        }
    } else {
        hv_next = C(0.0);
        a_next = vv_div<FAST>(a_bot_num, C(0.5) * hv_k + hn);
    }
    E a_k = E(0.0);  // a(1) = 0, surface
    E Rayk = ray_on[0] ? (E)rc[0] : E(0.0);
    E h_u = (E)(hv_k + hn);
    E b_denom_1 = h_u + dtE * (Rayk + a_k);
    E b1 = vv_div<FAST>(E(1.0), b_denom_1 + dtE * (E)a_next);
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
        if constexpr (!FAST) {
#pragma unroll
            for (int c = 0; c <= CH; ++c)
                if (kt + 1 + c <= nz + 1) pb[c] = (C)slot[kt + 1 + c];
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            int k = kt + c;
            if (k <= nz) {
                const E vk = vnext;          // vel(k) before elimination
                a_k = (E)a_next;
                hv_k = hv_next;
                if (k < nz) {
                    vnext = pv[c];
                    if constexpr (FAST) {
                        // botfn(z_i(k + 1)) is bf_cur; z_i(k + 2) drops layer k + 1
                        const C hh = harm(p0[c], p1[c]);
                        const C bf_k1 = bf_cur;
                        zi = k + 2 <= nz ? zi - hh * I_Hbbl : C(0.0);
                        bf_cur = vv_botfn<FAST>(zi);
                        hv_next = hvel_h(bf_cur, hh, p0[c], p1[c], (C)vnext);
                        z_top = z_top + hv_k;
                        a_next = a_of(bf_k1, z_top, hv_next, hv_k);
                    } else {
                        hv_next = hvel(pb[c + 1], p0[c], p1[c], (C)vnext);
                        z_top = z_top + hv_k;
                        a_next = a_of(pb[c], z_top, hv_next, hv_k);
                    }
                } else {
                    a_next = vv_div<FAST>(a_bot_num, C(0.5) * hv_k + hn);
                }
                Rayk = pr[c];
                E c1 = dtE * a_k * b1;
                slot[k] = c1;
                h_u = (E)(hv_k + hn);
                b_denom_1 = h_u + dtE * (Rayk + a_k * d1);
                b1 = vv_div<FAST>(E(1.0), b_denom_1 + dtE * (E)a_next);
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

// The fast forms' column in two sweeps: the tridiagonal system is eliminated
// bottom-up and back-substituted top-down (the serial code's elimination
// mirrored), so that z_i, the bottom-up sum of the harmonic thicknesses that
// botfn(z_i) needs, is formed on the way up instead of by a sweep of its own.
// The mixed-layer taper 1 - z_top / Hmix needs z_top, the sum of hvel from the
// surface, which the upward sweep only has at the end; it applies only to the
// interfaces with z_top < Hmix.  hvel >= h_harm, so when the harmonic
// thicknesses of the top MTOP layers already sum to Hmix (checked first, with
// a relative margin for rounding) every interface below layer MTOP is untapered:
// the sweep runs up to layer MTOP + 1 without z_top, then forms z_i, hvel,
// z_top and a(K) of the top MTOP layers and eliminates them.  Returns false,
// having written nothing, for a column where the check fails (thin surface
// layers, or nz <= MTOP + 1); the caller then runs vertvisc_column.
// Per layer: h, h(neighbour) and the velocity are read once by the upward
// sweep (staged in shared memory, CH layers ahead, with cp.async), the
// eliminated velocity and the multiplier once by the downward one.
// Within a few units in the last place of the top-down elimination (the
// system is diagonally dominant); each coefficient follows the serial
// expressions with vv_div quotients, and z_i is summed bottom-up as the serial
// code sums it.
constexpr int kVvTop = 4;

// NT: the threads of the CTA (the stride of stage, [2][CH][3][NT]).
template <int KMAX, int CH, typename R, typename E, int NT = 128, int MTOP = kVvTop>
__device__ __forceinline__ bool
vertvisc_column_up(const Dims& D, const Metrics& M, R* __restrict__ u, R* __restrict__ v,
                   const R* __restrict__ h, double dt, const VVParams& P,
                   double* __restrict__ taux_bot, double* __restrict__ tauy_bot, int bx, int by,
                   R* stage)
{
    using C = R;
    const int nz = D.nk;
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
        if (i > D.ie) return true;
        di = 1; dj = 0;
        vel = u; mask = M.mask2dCu; tau = M.taux; Ray = M.Ray_u;
        ray_on = M.ray_layer_u; tbot = taux_bot;
    } else {     // v columns: i in [is, ie], J in [js-1, je]
        j = D.js + q;
        i = D.is + bx * (int)blockDim.x + (int)threadIdx.x;
        if (i > D.ie) return true;
        di = 0; dj = 1;
        vel = v; mask = M.mask2dCv; tau = M.tauy; Ray = M.Ray_v;
        ray_on = M.ray_layer_v; tbot = tauy_bot;
    }
    const double msk = MOM6B_A2(mask, i, j, D);
    if (!(msk > 0.0)) return true;   // vert_visc_apply leaves masked columns alone
    if (nz <= MTOP + 1) return false;
    const size_t plane = (size_t)D.plane;
    const R* hc = h + (size_t)(j - 1) * D.n1 + (i - 1);               // h(i, j, 1)
    const R* hn_ = h + (size_t)(j - 1 + dj) * D.n1 + (i - 1 + di);     // neighbour
    R* vc = vel + (size_t)(j - 1) * D.n1 + (i - 1);
    const double* rc = Ray + (size_t)(j - 1) * D.n1 + (i - 1);
    const C hn = (C)P.h_neglect, I_Hbbl = (C)P.I_Hbbl, Kv = (C)P.Kv, Kv_ml = (C)P.Kv_ml;
    const C Kv_extra_bbl = (C)P.Kv_extra_bbl, Hmix = (C)P.Hmix;
    auto harm = [&](C h0, C h1) -> C { return vv_div<true>(C(2.0) * h0 * h1, h0 + h1 + hn); };
    // hvel(k) from botfn(z_i(k + 1)) (vert_visc_coef :162-177)
    auto hvel_h = [&](C bf, C hh, C h0, C h1, C vk) -> C {
        C hv = hh;
        if (vk * (h1 - h0) < C(0.0)) hv = (C(1.0) - bf) * hh + bf * (C(0.5) * (h1 + h0));
        return hv;
    };

    // the top MTOP layers' harmonic thicknesses must reach Hmix
    {
        C h0[MTOP], h1[MTOP];
#pragma unroll
        for (int k = 0; k < MTOP; ++k) {
            h0[k] = hc[(size_t)k * plane];
            h1[k] = hn_[(size_t)k * plane];
        }
        C top = C(0.0);
#pragma unroll
        for (int k = 0; k < MTOP; ++k) top = top + harm(h0[k], h1[k]);
        const C margin = sizeof(C) == 8 ? C(1.0e-12) : C(1.0e-5);
        if (!(top >= Hmix + Hmix * margin)) return false;
    }

    E slot[KMAX + 2];   // c1r(L) = dt a(L) b1(L), the downward sweep's multipliers
    const E dtE = (E)dt;
    const E sfc_stress = (E)(dt / kRho0 * MOM6B_A2(tau, i, j, D) * msk);
    const int tid = (int)threadIdx.x;
    auto ST = [&](int b, int c, int f) -> R& { return stage[((b * CH + c) * 3 + f) * NT + tid]; };

    // ---- upward sweep: layer nz ----------------------------------------------
    C hhL, hvL;           // harm and hvel of the layer L being eliminated
    E vL;                 // its velocity
    {
        const C h0 = hc[(size_t)(nz - 1) * plane], h1 = hn_[(size_t)(nz - 1) * plane];
        vL = (E)vc[(size_t)(nz - 1) * plane];
        hhL = harm(h0, h1);
        hvL = hvel_h(vv_botfn<true>(C(0.0)), hhL, h0, h1, (C)vL);   // z_i(nz + 1) = 0
    }
    // a(nz + 1), the bottom interface (:205-206)
    const C a_bot = vv_div<true>(Kv + Kv_extra_bbl, C(0.5) * hvL + hn);
    // FP64 storage: with a(L) = Kv_tot / h_shear, the step's products of
    // dt a(L + 1) are carried instead of a(L + 1): Pd = dt a(L + 1) d1(L + 1)
    // and Pu = dt a(L + 1) u'(L + 1) (at the bottom d1 = 1 and u' = 0: the
    // zero-velocity bottom).  With K = dt Kv_tot(L), S = h_shear(L) and r =
    // 1 / (bd S + K), b1 = S r, dt a(L) b1 = K r, dt a(L) d1 = K bd r and
    // dt a(L) u' = K rhs r, so a layer takes one quotient instead of two (a(L)
    // and b1).  FP32 storage (the mixed form, whose kernels are held to 64
    // registers) keeps a(L) and the two quotients.
    E Pd = dtE * (E)a_bot, Pu = E(0.0);
    E a_below = (E)a_bot, d1 = E(1.0);
    E up = E(0.0);               // the eliminated velocity of the last layer
    C zL = C(0.0);               // z_i(L + 1)
    // eliminate layer L with a(L) = Kv_tot / h_shear above it (u'(L) ->
    // vel(L), c1r(L) -> slot); Kv_tot = 0, h_shear = 1 at the surface (a(1) = 0)
    auto eliminate = [&](int L, C hv, C Kv_tot, C h_shear, E vk, E Rayk, E rhs_extra) {
        const E hu = (E)(hv + hn);
        if constexpr (sizeof(R) == 8) {
            const E K = dtE * (E)Kv_tot, S = (E)h_shear;
            const E bd = hu + (dtE * Rayk + Pd);
            const E r = vv_div<true>(E(1.0), bd * S + K);
            const E rhs = hu * vk + rhs_extra + Pu;
            up = rhs * (S * r);
            slot[L] = K * r;
            Pd = K * bd * r;
            Pu = K * rhs * r;
        } else {
            const E aL = (E)vv_div<true>(Kv_tot, h_shear);
            const E bd = hu + dtE * (Rayk + a_below * d1);
            const E b1 = vv_div<true>(E(1.0), bd + dtE * aL);
            d1 = bd * b1;
            up = (hu * vk + rhs_extra + dtE * a_below * up) * b1;
            slot[L] = dtE * aL * b1;
            a_below = aL;
        }
        vc[(size_t)(L - 1) * plane] = (R)up;
    };
    // lookahead layers L - 1 of the chunk's layers L = Lt .. Lt - CH + 1 (those
    // with L >= MTOP + 1) into buffer b; every staged velocity is read before
    // this thread overwrites it
    auto stage_up = [&](int Lt, int b) {
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int L = Lt - c;
            const bool ok = L >= MTOP + 1;
            const size_t o = ok ? (size_t)(L - 2) * plane : 0;
            cp_async_elem(&ST(b, c, 0), hc + o, ok);
            cp_async_elem(&ST(b, c, 1), hn_ + o, ok);
            cp_async_elem(&ST(b, c, 2), (const R*)vc + o, ok);
        }
        cp_async_commit();
    };
    stage_up(nz, 0);
    for (int Lt = nz, it = 0; Lt >= MTOP + 1; Lt -= CH, ++it) {
        const int b = it & 1;
        if (Lt - CH >= MTOP + 1) {
            stage_up(Lt - CH, b ^ 1);
            cp_async_wait_prior();
        } else {
            cp_async_wait_all();
        }
        C p0[CH], p1[CH];
        E pv[CH], pr[CH];
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int L = Lt - c;
            p0[c] = ST(b, c, 0);
            p1[c] = ST(b, c, 1);
            pv[c] = (E)ST(b, c, 2);
            pr[c] = (L >= MTOP + 1 && ray_on[L - 1]) ? (E)rc[(size_t)(L - 1) * plane] : E(0.0);
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
            const int L = Lt - c;
            if (L >= MTOP + 1) {
                const C z_L = zL + hhL * I_Hbbl;                 // z_i(L)
                const C hhu = harm(p0[c], p1[c]);                // layer L - 1
                const C bfL = vv_botfn<true>(z_L);
                const C hvu = hvel_h(bfL, hhu, p0[c], p1[c], (C)pv[c]);
                // a(L) below the untapered depth (:185-202), as Kv_tot / h_shear
                eliminate(L, hvL, Kv + Kv_extra_bbl * bfL, C(0.5) * (hvL + hvu + hn), vL,
                          pr[c], E(0.0));
                zL = z_L; hhL = hhu; hvL = hvu; vL = pv[c];
            }
        }
    }

    // ---- the top MTOP layers ------------------------------------------------
    // hvel(MTOP) = hvL, harm(MTOP) = hhL, z_i(MTOP + 1) = zL
    C hvT[MTOP + 1], zT[MTOP + 2];
    E vT[MTOP + 1];
    hvT[MTOP] = hvL;
    vT[MTOP] = vL;
    zT[MTOP + 1] = zL;
    {
        C hh = hhL;
#pragma unroll
        for (int k = MTOP; k >= 2; --k) {
            zT[k] = zT[k + 1] + hh * I_Hbbl;                     // z_i(k)
            const C h0 = hc[(size_t)(k - 2) * plane], h1 = hn_[(size_t)(k - 2) * plane];
            const E vk = (E)vc[(size_t)(k - 2) * plane];
            hh = harm(h0, h1);
            hvT[k - 1] = hvel_h(vv_botfn<true>(zT[k]), hh, h0, h1, (C)vk);
            vT[k - 1] = vk;
        }
    }
    C ztop[MTOP + 1];   // z_top(K) = hvel(1) + ... + hvel(K - 1)
    ztop[1] = C(0.0);
#pragma unroll
    for (int K = 2; K <= MTOP; ++K) ztop[K] = ztop[K - 1] + hvT[K - 1];
#pragma unroll
    for (int L = MTOP; L >= 1; --L) {
        C Kv_tot = C(0.0), h_shear = C(1.0);   // a(1) = 0, the surface
        if (L >= 2) {
            Kv_tot = Kv;
            if (ztop[L] < Hmix) Kv_tot = Kv_tot + (Kv_ml - Kv) * (C(1.0) - vv_div<true>(ztop[L], Hmix));
            Kv_tot = Kv_tot + Kv_extra_bbl * vv_botfn<true>(zT[L]);
            h_shear = C(0.5) * (hvT[L] + hvT[L - 1] + hn);
        }
        const E Rayk = ray_on[L - 1] ? (E)rc[(size_t)(L - 1) * plane] : E(0.0);
        eliminate(L, hvT[L], Kv_tot, h_shear, vT[L], Rayk, L == 1 ? sfc_stress : E(0.0));
    }

    // ---- downward sweep: back substitution u(L) = u'(L) + c1r(L) u(L - 1) ----
    // one multiply-add per layer: the loads of 2 CH layers are issued together
    // The Rayleigh part of the bottom stress (:452-458) is summed in the serial
    // order of the layers from the stored velocities: on the way down for FP64
    // storage, by a pass of its own for FP32 storage (64 registers).
    constexpr bool RAY_DOWN = sizeof(R) == 8;
    constexpr int CHD = 2 * CH;
    E u_above = up;   // u(1) = u'(1), already in place
    double tray = (RAY_DOWN && ray_on[0]) ? kRho0 * rc[0] * (double)(R)up : 0.0;
    for (int kt = 2; kt <= nz; kt += CHD) {
        E pv[CHD], pc[CHD];
        double pr[RAY_DOWN ? CHD : 1];
#pragma unroll
        for (int c = 0; c < CHD; ++c) {
            const int L = kt + c;
            if (L <= nz) {
                pv[c] = (E)vc[(size_t)(L - 1) * plane];
                pc[c] = slot[L];
                if constexpr (RAY_DOWN)
                    pr[c] = ray_on[L - 1] ? rc[(size_t)(L - 1) * plane] : 0.0;
            }
        }
#pragma unroll
        for (int c = 0; c < CHD; ++c) {
            const int L = kt + c;
            if (L <= nz) {
                const E uk = pv[c] + pc[c] * u_above;
                vc[(size_t)(L - 1) * plane] = (R)uk;
                u_above = uk;
                if constexpr (RAY_DOWN)
                    if (pr[c] != 0.0) tray = tray + kRho0 * pr[c] * (double)(R)uk;
            }
        }
    }
    if constexpr (!RAY_DOWN) {
        for (int k = 1; k <= nz; ++k)
            if (ray_on[k - 1]) {
                const size_t o = (size_t)(k - 1) * plane;
                tray = tray + kRho0 * rc[o] * (double)vc[o];
            }
    }
    tbot[(size_t)(j - 1) * D.n1 + (i - 1)] = kRho0 * (double)u_above * (double)a_bot + tray;
    return true;
}

// The fast forms' kernel: the two-sweep column where it applies, else the
// three-sweep one.
template <int KMAX, int CH, typename R, typename E, int MINB, bool ASYNC>
__global__ void __launch_bounds__(128, MINB)
k_vertvisc_up(Dims D, Metrics M, R* __restrict__ u, R* __restrict__ v, const R* __restrict__ h,
              double dt, VVParams P, double* __restrict__ taux_bot,
              double* __restrict__ tauy_bot)
{
    __shared__ R stage[2 * CH * 3 * 128];
    if (!vertvisc_column_up<KMAX, CH, R, E>(D, M, u, v, h, dt, P, taux_bot, tauy_bot,
                                             (int)blockIdx.x, (int)blockIdx.y, stage))
        vertvisc_column<KMAX, CH, R, E, false, ASYNC, true>(D, M, u, v, h, dt, P, taux_bot,
                                                            tauy_bot, (int)blockIdx.x,
                                                            (int)blockIdx.y, nullptr, nullptr,
                                                            stage);
}

// MINB: the CTAs per SM the register allocation is held to.
template <int KMAX, int CH, typename R, typename E, int MINB = 1, bool REM = false,
          bool ASYNC = false, bool FAST = false>
__global__ void __launch_bounds__(128, MINB)
k_vertvisc_pf(Dims D, Metrics M, R* __restrict__ u, R* __restrict__ v,
              const R* __restrict__ h, double dt, VVParams P,
              double* __restrict__ taux_bot, double* __restrict__ tauy_bot,
              double* __restrict__ rem_u = nullptr, double* __restrict__ rem_v = nullptr)
{
    __shared__ R stage[ASYNC ? 2 * CH * 3 * 128 : 1];
    vertvisc_column<KMAX, CH, R, E, REM, ASYNC, FAST>(D, M, u, v, h, dt, P, taux_bot,
                                                      tauy_bot, (int)blockIdx.x,
                                                      (int)blockIdx.y, rem_u, rem_v, stage);
}

// Launch shapes measured fastest on B200 at 720x720x75: the fast FP64 and
// mixed forms run the two-sweep kernel; the exact FP64 form stages sweeps 1
// and 2 with cp.async and holds registers to 6 CTAs per SM (2.215 ms per step
// against 2.285 loaded into registers); the other FP32-storage forms load
// 4-layer chunks into registers (staging measured slower there), held to
// vv_min_blocks CTAs per SM.
template <int KMAX, typename R, typename E, bool FAST>
static cudaError_t launch_vv_pf(const Dims& D, const Metrics& M, R* u, R* v, const R* h,
                                double dt, const VVParams& P, double* taux_bot,
                                double* tauy_bot, cudaStream_t s, double* rem_u = nullptr,
                                double* rem_v = nullptr)
{
    const int nb = 128;
    int ncol = D.ie - D.is + 2;
    int nrows = (D.je - D.js + 1) + (D.je - D.js + 2);
    dim3 grid((ncol + nb - 1) / nb, nrows, 1);
    constexpr int MB = vv_min_blocks<R, E>();
    if constexpr (FAST) {
        // the fast FP64 and mixed forms: the two-sweep column (three sweeps
        // where it does not apply); no remnant in these forms
        if (rem_u) return cudaErrorInvalidValue;
        k_vertvisc_up<KMAX, kVvChunk, R, E, MB, (sizeof(R) == 8)><<<grid, nb, 0, s>>>(
            D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    } else if constexpr (sizeof(R) == 8) {
        if (rem_u)
            k_vertvisc_pf<KMAX, kVvChunk, R, E, MB, true, true, FAST><<<grid, nb, 0, s>>>(
                D, M, u, v, h, dt, P, taux_bot, tauy_bot, rem_u, rem_v);
        else
            k_vertvisc_pf<KMAX, kVvChunk, R, E, MB, false, true, FAST><<<grid, nb, 0, s>>>(
                D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    } else {
        k_vertvisc_pf<KMAX, kVvChunk, R, E, MB, false, false, FAST><<<grid, nb, 0, s>>>(
            D, M, u, v, h, dt, P, taux_bot, tauy_bot);
    }
    return cudaGetLastError();
}

// rem_u, rem_v (FP64, both or neither): also the vertical-viscosity remnant.
template <typename R, typename E = R, bool FAST = false>
cudaError_t launch_vertvisc_pf_t(const Dims& D, const Metrics& M, R* u, R* v, const R* h,
                                 double dt, const VVParams& P, double* taux_bot,
                                 double* tauy_bot, cudaStream_t s, double* rem_u = nullptr,
                                 double* rem_v = nullptr)
{
    if ((rem_u == nullptr) != (rem_v == nullptr)) return cudaErrorInvalidValue;
    if (D.nk <= 80)
        return launch_vv_pf<80, R, E, FAST>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u,
                                            rem_v);
    if (D.nk <= 128)
        return launch_vv_pf<128, R, E, FAST>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u,
                                             rem_v);
    if (D.nk <= 256)
        return launch_vv_pf<256, R, E, FAST>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u,
                                             rem_v);
    return launch_vv_pf<1024, R, E, FAST>(D, M, u, v, h, dt, P, taux_bot, tauy_bot, s, rem_u,
                                          rem_v);
}

} // namespace mom6b
