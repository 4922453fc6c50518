// tendency_impl.cuh -- the fused momentum tendency kernel, templated on the
// state/arithmetic type R.  R = double is the bit-exact FP64 form (built
// without FMA contraction in k_tendency.cu); R = float is the mixed form's
// stencil arithmetic (k_mixed.cu).  Metrics are read as double and rounded
// to R; literals are written R(...) so the float instantiation never
// promotes to double.
//
// One kernel replaces four phases of the serial driver for one half of the
// RK2 step:
//   compute_transports   rk2_serial_driver.F90:544-561
//   hor_visc             mom6_hor_visc_serial.F90:464-1109 (Laplacian path)
//   CorAdCalc            mom6_coriolis_serial.F90:112-252 (Sadourny scheme)
//   velocity update      rk2_serial_driver.F90:257-270 / :337-350
// so uh, vh, diffu, diffv, CAu and CAv never reach HBM.  Per layer a CTA
// stages u, v, h on a (TX+2) x (TY+2) tile in shared memory, evaluates the
// q/str_xy (corner), KE/str_xx (centre) and uh/vh intermediates the tile
// needs, and writes
//   uout(I,j) = ubase(I,j) + coef * (CAu + diffu)   I in [is, ie-1], j in [js, je]
//   vout(i,J) = vbase(i,J) + coef * (CAv + diffv)   i in [is, ie],   J in [js, je-1]
// Each intermediate is evaluated with the reference's operation order, so
// the FP64 result equals the serial Fortran bit for bit.  Two reference
// quirks are reproduced: hArea_u(:, js-1) and hArea_v(is-1, :) are never
// written by CorAdCalc and enter q as zero (mom6_coriolis_serial.F90:142-152
// vs :162-168).  In a subdomain of a decomposed run (Dims' cut flags) the
// points on a cut are interior: there hArea exists, and the u (v) update
// reaches ie (je) at an east (north) cut.
#pragma once

#include "kernels.h"
#include "tma.cuh"

namespace mom6b {

// UNI selects the uniform-metric instantiation (metrics as scalars, Coriolis
// per row); otherwise every metric is read from its 2-D array.  The CTA with
// block coordinates (bx, by, bz) owns the tile i0 = is + bx TX, j0 = js + by TY
// and walks the KC consecutive layers from k0 + bz KC.
// UNI selects the uniform-metric instantiation (metrics as scalars, Coriolis
// per row); otherwise every metric is read from its 2-D array.  The CTA with
// block coordinates (bx, by, bz) owns the tile i0 = is + bx TX, j0 = js + by TY
// and walks the KC consecutive layers from k0 + bz KC.  The u, v, h tiles are
// double-buffered: layer k+1 is copied into shared memory (cp.async) while
// layer k is evaluated, so the loads' latency leaves the layer loop and each
// layer takes two barriers.
// DIAG: also store the horizontal-viscosity accelerations diffu, diffv of the
// updated points in dfu, dfv (the driver's diffu_sum / diffv_sum diagnostics).
// The Arakawa coefficients of the u point (I, j) (mom6_coriolis_serial.F90
// :171-193) from q at its corners: a and d from the east pair of columns,
// q00 = q(I, j), qp0 = q(I+1, j), q0m = q(I, j-1), qpm = q(I+1, j-1); b and
// c from the west pair, qm0 = q(I-1, j), qmm = q(I-1, j-1).  LAMB81 writes a
// and d at I = i - 1 of its loop; the values are the same expressions.
template <int COR, typename R>
__device__ __forceinline__ void arakawa_ad(R q00, R qp0, R q0m, R qpm, R& a, R& d)
{
    if constexpr (COR == 2) {
        const R c12 = R(1.0) / R(12.0);
        a = (q00 + (qp0 + q0m)) * c12;
        d = ((q00 + qpm) + q0m) * c12;
    } else {
        const R c24 = R(1.0) / R(24.0);
        a = (R(2.0) * (qp0 + q0m) + (q00 + qpm)) * c24;
        d = ((qp0 + q0m) + R(2.0) * (q00 + qpm)) * c24;
    }
}

template <int COR, typename R>
__device__ __forceinline__ void arakawa_bc(R q00, R qm0, R q0m, R qmm, R& b, R& c)
{
    if constexpr (COR == 2) {
        const R c12 = R(1.0) / R(12.0);
        b = (q00 + (qm0 + q0m)) * c12;
        c = ((q00 + qmm) + q0m) * c12;
    } else {
        const R c24 = R(1.0) / R(24.0);
        b = ((q00 + qmm) + R(2.0) * (qm0 + q0m)) * c24;
        c = (R(2.0) * (q00 + qmm) + (qm0 + q0m)) * c24;
    }
}

// Multiply-add in the stencil type (the folded stencils of the fast FP64 and
// the mixed forms).
__device__ __forceinline__ double td_fma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float td_fma(float a, float b, float c) { return fmaf(a, b, c); }

// Quotients of the tendency: div_nr in the fast FP64 form, IEEE division in
// the exact form, div_r in float.
template <bool FAST>
__device__ __forceinline__ double td_div(double a, double b)
{
    if constexpr (FAST) return div_nr(a, b);
    else return a / b;
}
template <bool FAST>
__device__ __forceinline__ float td_div(float a, float b) { return div_r(a, b); }

// EXTV: diffu, diffv come from dfu, dfv (the general hor_visc kernel's
// outputs) and the stresses are not evaluated.
// COR: the Coriolis scheme of CorAdCalc (mom6_coriolis_serial.F90:19-21):
// 1 SADOURNY75_ENERGY (the driver's), 2 ARAKAWA_HSU90, 3 ARAKAWA_LAMB81.  The
// Arakawa schemes' coefficients a, b, c, d (:171-193) reach q one corner
// further east and north, so their tiles stage and evaluate one more column
// and row; the coefficients are formed where CAu / CAv need them (:228-248).
// FAST: the fast FP64 form's arithmetic (built with FMA contraction in
// k_tendency_fast.cu): quotients by div_nr.
// TMA: the u, v, h tiles of a layer arrive as three TMA box loads
// ({SX, SY, 1} of the fields' tensor maps tmaps[0..2]) issued by one thread
// into 128-byte-aligned double buffers, completing on one mbarrier per
// buffer; a load that does not land within the wait budget records
// kDevTimeout in *status and the CTA returns.  FP64 Sadourny tiles only: the
// box row (SX doubles) and its x origin i0 - 2 = is - 2 + TX bx (even) meet
// the unit's 16-byte rules.  Otherwise every thread copies its share of the
// tile element by element with cp.async.
template <int TX, int TY, bool UNI, typename R, bool DIAG = false, int COR = 1,
          bool EXTV = false, bool FAST = false, bool TMA = false>
__device__ __forceinline__ void
tendency_tile(const Dims& D, const Metrics& M, const UniMetrics& U, const R* __restrict__ uin,
              const R* __restrict__ vin, const R* __restrict__ h,
              const R* ubase, const R* vbase, R* uout, R* vout,
              R coef, R h_neglect, int k0, int KC, int bx, int by, int bz,
              R* dfu = nullptr, R* dfv = nullptr, const CUtensorMap* tmaps = nullptr,
              int* status = nullptr)
{
    // FU: the fast FP64 form and the mixed form on uniform metrics, whose
    // Sadourny stencils multiply by the folded products of U.tf (the exact
    // form keeps the serial expressions)
    constexpr bool FU = (FAST || sizeof(R) == 4) && UNI && COR == 1 && !EXTV && !DIAG;
    constexpr int W = COR >= 2 ? 1 : 0;      // the Arakawa schemes' extra column and row
    constexpr int SX = TX + 2 + W, SY = TY + 2 + W;  // staged: [i0-1, i0+TX+W] x [j0-1, j0+TY+W]
    constexpr int CX = TX + 1 + W, CY = TY + 1 + W;  // intermediates
    constexpr int NT = TX * TY;
    constexpr int NS = (SX * SY + NT - 1) / NT;  // staged elements per thread
    static_assert(!TMA || (sizeof(R) == 8 && COR <= 1 && (SX * sizeof(R)) % 16 == 0 && TX % 2 == 0),
                  "TMA tiles need 16-byte rows and even x origins");
    // the element-wise staging buffers, and the TMA buffers (each tile a
    // multiple of 128 bytes so that every TMA destination is 128-byte aligned)
    constexpr int AX = TMA ? 1 : SX, AY = TMA ? 1 : SY, AB = TMA ? 1 : 2;
    constexpr int TPAD = ((SX * SY + 15) / 16) * 16;
    __shared__ R s_u[AB][AY][AX], s_v[AB][AY][AX], s_h[AB][AY][AX];
    __shared__ __align__(128) R s_t[TMA ? 2 * 3 * TPAD : 1];
    __shared__ __align__(8) uint64_t s_tbar[2];
    // the intermediates; with TMA tiles two sets, layer k in set k & 1, so
    // that layer k + 1's intermediates never overwrite what layer k's outputs
    // still read and one barrier per layer suffices
    constexpr int IB = TMA ? 2 : 1;
    __shared__ R s_q[IB][CY][CX], s_sxy[IB][CY][CX];   // corners  [i0-1, i0+TX-1] x [j0-1, j0+TY-1]
    __shared__ R s_ke[IB][CY][CX], s_sxx[IB][CY][CX];  // centres  [i0, i0+TX] x [j0, j0+TY]
    __shared__ R s_uh[IB][CY][CX];                     // u-faces  [i0-1, i0+TX-1] x [j0, j0+TY]
    __shared__ R s_vh[IB][CY][CX];                     // v-faces  [i0, i0+TX] x [j0-1, j0+TY-1]

    const int i0 = D.is + bx * TX;
    const int j0 = D.js + by * TY;
    const int tid = (int)threadIdx.y * TX + (int)threadIdx.x;
    const int kb = k0 + bz * KC;
    const int ke = (kb + KC - 1 < D.nk) ? kb + KC - 1 : D.nk;

    // this thread's staged elements: shared index, offset in a layer, in range
    int sp[NS];
    size_t go[NS];
    bool gok[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        const int p = tid + q * NT;
        const int r = p / SX, c = p - r * SX;
        const int i = i0 - 1 + c, j = j0 - 1 + r;
        sp[q] = p < SX * SY ? p : -1;
        gok[q] = p < SX * SY && i <= D.n1 && j <= D.n2;
        go[q] = gok[q] ? (size_t)(j - 1) * D.n1 + (size_t)(i - 1) : 0;
    }
    auto stage = [&](int k, int b) {
        if constexpr (TMA) {
            if (tid == 0) {
                tma_bar_expect(&s_tbar[b], (uint32_t)(3 * SX * SY * sizeof(R)));
#pragma unroll
                for (int f = 0; f < 3; ++f)
                    tma_load_3d(&s_t[(b * 3 + f) * TPAD], &tmaps[f], i0 - 2, j0 - 2, k - 1,
                                &s_tbar[b]);
            }
        } else {
            const size_t koff = (size_t)(k - 1) * (size_t)D.plane;
#pragma unroll
            for (int q = 0; q < NS; ++q) {
                if (sp[q] >= 0) {
                    const size_t o = gok[q] ? koff + go[q] : 0;
                    cp_async_elem(&s_u[b][0][0] + sp[q], uin + o, gok[q]);
                    cp_async_elem(&s_v[b][0][0] + sp[q], vin + o, gok[q]);
                    cp_async_elem(&s_h[b][0][0] + sp[q], h + o, gok[q]);
                }
            }
            cp_async_commit();
        }
    };
    if constexpr (TMA) {
        if (tid == 0) {
            tma_prefetch_map(&tmaps[0]);
            tma_prefetch_map(&tmaps[1]);
            tma_prefetch_map(&tmaps[2]);
            tma_bar_init(&s_tbar[0], 1);
            tma_bar_init(&s_tbar[1], 1);
        }
        __syncthreads();
    }
    // TMA: layers kb and kb + 1 are requested up front and layer k + 2 as soon
    // as every thread is done with layer k's tile (after its intermediates);
    // the element-wise staging requests layer k + 1 at the top of layer k
    if (kb <= ke) stage(kb, 0);
    if (TMA && kb + 1 <= ke) stage(kb + 1, 1);
    // buffer b's n-th use (layer kb + 2 n + b) completes its phase of parity n & 1
    auto parity = [&](int k) { return (uint32_t)(((k - kb) >> 1) & 1); };
  for (int k = kb; k <= ke; ++k) {
    const size_t koff = (size_t)(k - 1) * (size_t)D.plane;
    const int b = (k - kb) & 1;
    const int ib = TMA ? b : 0;
    bool late = false;
    if constexpr (TMA) {
        // layer k's tiles; no barrier: the intermediates' set ib was last read
        // by layer k - 2's outputs, which every thread finished before layer
        // k - 1's barrier
        late = !tma_bar_wait(&s_tbar[b], parity(k), kBtDefaultWait);
    } else {
        // layer k's tiles are visible to all threads, and every thread is done
        // with layer k-1 (its outputs read buffer b^1 and the intermediates)
        cp_async_wait_all();
        __syncthreads();
        if (k < ke) stage(k + 1, b ^ 1);
    }
    const R* t_u = TMA ? &s_t[(b * 3 + 0) * TPAD] : &s_u[b][0][0];
    const R* t_v = TMA ? &s_t[(b * 3 + 1) * TPAD] : &s_v[b][0][0];
    const R* t_h = TMA ? &s_t[(b * 3 + 2) * TPAD] : &s_h[b][0][0];

    // this thread's bases, loaded before the intermediates are evaluated
    const int Io = i0 + (int)threadIdx.x;
    const int jo = j0 + (int)threadIdx.y;
    // at an east / north cut the face on it is interior and updated
    const bool do_u = Io <= D.ie - 1 + D.ce && jo <= D.je;
    const bool do_v = Io <= D.ie && jo <= D.je - 1 + D.cn;
    const size_t oo = koff + (size_t)(jo - 1) * D.n1 + (Io - 1);
    const R ub = do_u ? ubase[oo] : R(0.0);
    const R vb = do_v ? vbase[oo] : R(0.0);

#define SU(i, j) t_u[((j) - (j0 - 1)) * SX + ((i) - (i0 - 1))]
#define SV(i, j) t_v[((j) - (j0 - 1)) * SX + ((i) - (i0 - 1))]
#define SH(i, j) t_h[((j) - (j0 - 1)) * SX + ((i) - (i0 - 1))]
#define G2(a, i, j) ((R)(UNI ? U.a : MOM6B_A2(M.a, i, j, D)))
#define COR(i, j) ((R)(UNI ? U.cor_row[(j) - 1] : MOM6B_A2(M.CoriolisBu, i, j, D)))

    // ---- intermediates ----------------------------------------------------
    // The items of intermediate point p = r CX + c: bit 0 the corner (q,
    // str_xy), bit 1 the centre (KE, str_xx), bit 2 uh, bit 3 vh.  Every thread
    // evaluates all items of its own point; with uniform metrics the CX CY -
    // TX TY fringe points' items are then spread one per thread, so that no
    // thread evaluates a second whole point while the rest of the CTA waits at
    // the barrier.
    auto interm = [&](int p, unsigned items) {
        int r = p / CX, c = p - r * CX;
        // corner point (I, J) = (i0-1+c, j0-1+r): q and str_xy
        if (items & 1u) {
            int I = i0 - 1 + c, J = j0 - 1 + r;
            R qv = R(0.0), sxy = R(0.0);
            if (FU && I + 1 <= D.n1 && J + 1 <= D.n2) {
                // the same expressions with the uniform metrics factored out
                const R dv = SV(I + 1, J) - SV(I, J), du = SU(I, J + 1) - SU(I, J);
                const R h00 = SH(I, J), h10 = SH(I + 1, J), h01 = SH(I, J + 1),
                        h11 = SH(I + 1, J + 1);
                const R a = h00 + h10, b = h01 + h11;
                const R absv = COR(I, J) + td_fma(R(U.tf.kRv), dv, -(R(U.tf.kRu) * du));
                const R S = ((J >= D.js - D.cs ? a : R(0.0)) + b) +
                            ((I >= D.is - D.cw ? h00 + h01 : R(0.0)) + (h10 + h11));
                qv = td_div<FAST>(absv * R(U.tf.kQn), S + R(U.tf.kQe));
                sxy = td_fma(R(U.tf.kSv), dv, R(U.tf.kSu) * du) * (a + b);
            } else if (I + 1 <= D.n1 && J + 1 <= D.n2) {
                R v0 = SV(I, J), v1 = SV(I + 1, J);
                R u0 = SU(I, J), u1 = SU(I, J + 1);
                R h00 = SH(I, J), h10 = SH(I + 1, J), h01 = SH(I, J + 1),
                       h11 = SH(I + 1, J + 1);
                // CorAdCalc: circulation, areas, PV (mom6_coriolis_serial.F90:134-168)
                R dvdx = (v1 * G2(dyCv, I + 1, J)) - (v0 * G2(dyCv, I, J));
                R dudy = (u1 * G2(dxCu, I, J + 1)) - (u0 * G2(dxCu, I, J));
                R rel = G2(mask2dBu, I, J) * (dvdx - dudy) * G2(IareaBu, I, J);
                R absv = COR(I, J) + rel;
                R aT00 = G2(areaT, I, J), aT10 = G2(areaT, I + 1, J),
                       aT01 = G2(areaT, I, J + 1), aT11 = G2(areaT, I + 1, J + 1);
                R hAu0 = (J >= D.js - D.cs) ? R(0.5) * ((aT00 * h00) + (aT10 * h10)) : R(0.0);
                R hAu1 = R(0.5) * ((aT01 * h01) + (aT11 * h11));
                R hAv0 = (I >= D.is - D.cw) ? R(0.5) * ((aT00 * h00) + (aT01 * h01)) : R(0.0);
                R hAv1 = R(0.5) * ((aT10 * h10) + (aT11 * h11));
                R hArea_q = (hAu0 + hAu1) + (hAv0 + hAv1);
                R Ih_q = td_div<FAST>(G2(Area_q, I, J), hArea_q + R(1.0e-20));
                qv = absv * Ih_q;
                if constexpr (!EXTV) {
                // hor_visc: shearing strain and stress at q-points (:513-520, :544, :579, :964, :1050)
                R dvdx_v = G2(DY_dxBu, I, J) *
                                ((v1 * G2(IdyCv, I + 1, J)) - (v0 * G2(IdyCv, I, J)));
                R dudy_v = G2(DX_dyBu, I, J) *
                                ((u1 * G2(IdxCu, I, J + 1)) - (u0 * G2(IdxCu, I, J)));
                R mBu = G2(mask2dBu, I, J);
                R sh_xy = mBu * (dvdx_v + dudy_v);
                R hq = R(0.25) * ((h00 + h11) + (h10 + h01));
                sxy = -(G2(Kh_xy, I, J) * sh_xy);
                sxy = sxy * (hq * mBu * G2(red_xy, I, J));
                }
            }
            s_q[ib][r][c] = qv;
            s_sxy[ib][r][c] = sxy;
        }
        // centre point (i, j) = (i0+c, j0+r): KE and str_xx
        if (items & 2u) {
            int i = i0 + c, j = j0 + r;
            R ke = R(0.0), sxx = R(0.0);
            if (FU && i <= D.n1 && j <= D.n2) {
                const R uc = SU(i, j), um = SU(i - 1, j), vc = SV(i, j), vm = SV(i, j - 1);
                ke = td_fma(R(U.tf.kKu), td_fma(uc, uc, um * um),
                            R(U.tf.kKv) * td_fma(vc, vc, vm * vm));
                sxx = SH(i, j) * td_fma(R(U.tf.kXv), vc - vm, -(R(U.tf.kXu) * (uc - um)));
            } else if (i <= D.n1 && j <= D.n2) {
                R uc = SU(i, j), um = SU(i - 1, j), vc = SV(i, j), vm = SV(i, j - 1);
                ke = td_div<FAST>(R(0.25) *
                               ((G2(dyCu, i, j) * (uc * uc) + G2(dyCu, i - 1, j) * (um * um)) +
                                (G2(dxCv, i, j) * (vc * vc) + G2(dxCv, i, j - 1) * (vm * vm))),
                           G2(areaT, i, j));
                if constexpr (!EXTV) {
                R dudx = G2(DY_dxT, i, j) *
                              ((G2(IdyCu, i, j) * uc) - (G2(IdyCu, i - 1, j) * um));
                R dvdy = G2(DX_dyT, i, j) *
                              ((G2(IdxCv, i, j) * vc) - (G2(IdxCv, i, j - 1) * vm));
                R sh_xx = dudx - dvdy;
                sxx = -(G2(Kh_xx, i, j) * sh_xx);
                sxx = sxx * (SH(i, j) * G2(red_xx, i, j));
                }
            }
            s_ke[ib][r][c] = ke;
            s_sxx[ib][r][c] = sxx;
        }
        // transports (compute_transports uses min(i+1, ied), min(j+1, jed))
        if (items & 4u) {
            int I = i0 - 1 + c, J = j0 + r;
            R uhv = R(0.0);
            if (I <= D.n1 && J <= D.n2) {
                int Ip = I + 1 < D.ied ? I + 1 : D.ied;
                R hp = (Ip - (i0 - 1) < SX) ? SH(Ip, J) : R(0.0);
                if constexpr (FU) uhv = (R(U.tf.kTu) * SU(I, J)) * (SH(I, J) + hp);
                else uhv = SU(I, J) * R(0.5) * (SH(I, J) + hp) * G2(dyCu, I, J);
            }
            s_uh[ib][r][c] = uhv;
        }
        if (items & 8u) {
            int i = i0 + c, j = j0 - 1 + r;
            R vhv = R(0.0);
            if (i <= D.n1 && j <= D.n2) {
                int Jp = j + 1 < D.jed ? j + 1 : D.jed;
                R hp = (Jp - (j0 - 1) < SY) ? SH(i, Jp) : R(0.0);
                if constexpr (FU) vhv = (R(U.tf.kTv) * SV(i, j)) * (SH(i, j) + hp);
                else vhv = SV(i, j) * R(0.5) * (SH(i, j) + hp) * G2(dxCv, i, j);
            }
            s_vh[ib][r][c] = vhv;
        }
    };
    if constexpr (UNI) {
        interm(tid, 15u);
        constexpr int NF = CX * CY - NT;
        for (int e = tid; e < 4 * NF; e += NT) interm(NT + e % NF, 1u << (e / NF));
    } else {
        // the 2-D metric form (more registers per point): whole points
        for (int p = tid; p < CX * CY; p += NT) interm(p, 15u);
    }
    // the thicknesses the outputs read, so that the tile is free after the barrier
    const R hIj = SH(Io, jo), hIpj = SH(Io + 1, jo), hIjp = SH(Io, jo + 1);
    if constexpr (TMA) {
        if (__syncthreads_or(late)) {
            if (tid == 0) {
                if (status) atomicExch(status, kDevTimeout);
                // the loads still in flight land in this CTA's shared memory:
                // wait for them once more (bounded) before the CTA exits
                tma_bar_wait(&s_tbar[b], parity(k), kBtDefaultWait);
                if (k + 1 <= ke) tma_bar_wait(&s_tbar[b ^ 1], parity(k + 1), kBtDefaultWait);
            }
            __syncthreads();
            return;
        }
        if (k + 2 <= ke) stage(k + 2, b);
    } else {
        __syncthreads();
    }

#define Q(I, J) s_q[ib][(J) - (j0 - 1)][(I) - (i0 - 1)]
#define SXY(I, J) s_sxy[ib][(J) - (j0 - 1)][(I) - (i0 - 1)]
#define KE(i, j) s_ke[ib][(j) - j0][(i) - i0]
#define SXX(i, j) s_sxx[ib][(j) - j0][(i) - i0]
#define UH(I, J) s_uh[ib][(J) - j0][(I) - (i0 - 1)]
#define VH(i, j) s_vh[ib][(j) - (j0 - 1)][(i) - i0]

    const int I = i0 + (int)threadIdx.x;
    const int j = j0 + (int)threadIdx.y;
    // ---- u point (I, j) ---------------------------------------------------
    if (FU && I <= D.ie - 1 + D.ce && j <= D.je) {
        const R CAu = td_fma(R(U.tf.kCu), td_fma(Q(I, j), VH(I + 1, j) + VH(I, j),
                                                 Q(I, j - 1) * (VH(I, j - 1) + VH(I + 1, j - 1))),
                             -(R(U.IdxCu) * (KE(I + 1, j) - KE(I, j))));
        const R diffu =
            td_div<FAST>(td_fma(R(U.tf.kDq), SXY(I, j - 1) - SXY(I, j),
                                R(U.tf.kDh) * (SXX(I, j) - SXX(I + 1, j))),
                         td_fma(R(U.tf.kHm), hIj + hIpj, h_neglect));
        uout[oo] = td_fma(coef, CAu + diffu, ub);
    } else if (I <= D.ie - 1 + D.ce && j <= D.je) {
        R IdxCu = G2(IdxCu, I, j);
        R KEx = (KE(I + 1, j) - KE(I, j)) * IdxCu;
        R CAu;
        if constexpr (COR <= 1) {
            CAu = R(0.25) *
                      ((Q(I, j) * (VH(I + 1, j) + VH(I, j))) +
                       (Q(I, j - 1) * (VH(I, j - 1) + VH(I + 1, j - 1)))) *
                      IdxCu -
                  KEx;
        } else {
            R a, b, c, d;
            arakawa_ad<COR>(Q(I, j), Q(I + 1, j), Q(I, j - 1), Q(I + 1, j - 1), a, d);
            arakawa_bc<COR>(Q(I, j), Q(I - 1, j), Q(I, j - 1), Q(I - 1, j - 1), b, c);
            CAu = (((a * VH(I + 1, j)) + (c * VH(I, j - 1))) +
                   ((b * VH(I, j)) + (d * VH(I + 1, j - 1)))) *
                      IdxCu -
                  KEx;
        }
        R diffu;
        if constexpr (EXTV) {
            diffu = dfu[oo];
        } else {
            R h_u = R(0.5) * (G2(mask2dT, I, j) * hIj + G2(mask2dT, I + 1, j) * hIpj);
            diffu = td_div<FAST>((IdxCu * ((G2(dx2q, I, j - 1) * SXY(I, j - 1)) -
                                    (G2(dx2q, I, j) * SXY(I, j))) +
                           G2(IdyCu, I, j) * ((G2(dy2h, I, j) * SXX(I, j)) -
                                              (G2(dy2h, I + 1, j) * SXX(I + 1, j)))) *
                              G2(IareaCu, I, j),
                          h_u + h_neglect);
        }
        uout[oo] = ub + coef * (CAu + diffu);
        if (DIAG && !EXTV) dfu[oo] = diffu;
    }
    // ---- v point (i, J) = (I, j) -------------------------------------------
    if (FU && I <= D.ie && j <= D.je - 1 + D.cn) {
        const int i = I, J = j;
        const R CAv = -td_fma(R(U.tf.kCv), td_fma(Q(i - 1, J), UH(i - 1, J) + UH(i - 1, J + 1),
                                                  Q(i, J) * (UH(i, J) + UH(i, J + 1))),
                              R(U.IdyCv) * (KE(i, J + 1) - KE(i, J)));
        const R diffv =
            td_div<FAST>(td_fma(R(U.tf.kEq), SXY(i - 1, J) - SXY(i, J),
                                -(R(U.tf.kEh) * (SXX(i, J) - SXX(i, J + 1)))),
                         td_fma(R(U.tf.kHm), hIj + hIjp, h_neglect));
        vout[oo] = td_fma(coef, CAv + diffv, vb);
    } else if (I <= D.ie && j <= D.je - 1 + D.cn) {
        const int i = I, J = j;
        R IdyCv = G2(IdyCv, i, J);
        R KEy = (KE(i, J + 1) - KE(i, J)) * IdyCv;
        R CAv;
        if constexpr (COR <= 1) {
            CAv = R(-0.25) *
                      ((Q(i - 1, J) * (UH(i - 1, J) + UH(i - 1, J + 1))) +
                       (Q(i, J) * (UH(i, J) + UH(i, J + 1)))) *
                      IdyCv -
                  KEy;
        } else {
            // a(i-1, J), d(i-1, J+1) of the u points west of i; b(i, J), c(i, J+1)
            R a, b, c, d, t;
            arakawa_ad<COR>(Q(i - 1, J), Q(i, J), Q(i - 1, J - 1), Q(i, J - 1), a, t);
            arakawa_ad<COR>(Q(i - 1, J + 1), Q(i, J + 1), Q(i - 1, J), Q(i, J), t, d);
            arakawa_bc<COR>(Q(i, J), Q(i - 1, J), Q(i, J - 1), Q(i - 1, J - 1), b, t);
            arakawa_bc<COR>(Q(i, J + 1), Q(i - 1, J + 1), Q(i, J), Q(i - 1, J), t, c);
            CAv = -(((a * UH(i - 1, J)) + (c * UH(i, J + 1))) +
                    ((b * UH(i, J)) + (d * UH(i - 1, J + 1)))) *
                      IdyCv -
                  KEy;
        }
        R diffv;
        if constexpr (EXTV) {
            diffv = dfv[oo];
        } else {
            R h_v = R(0.5) * (G2(mask2dT, i, J) * hIj + G2(mask2dT, i, J + 1) * hIjp);
            diffv = td_div<FAST>((IdyCv * ((G2(dy2q, i - 1, J) * SXY(i - 1, J)) -
                                    (G2(dy2q, i, J) * SXY(i, J))) -
                           G2(IdxCv, i, J) * ((G2(dx2h, i, J) * SXX(i, J)) -
                                              (G2(dx2h, i, J + 1) * SXX(i, J + 1)))) *
                              G2(IareaCv, i, J),
                          h_v + h_neglect);
        }
        vout[oo] = vb + coef * (CAv + diffv);
        if (DIAG && !EXTV) dfv[oo] = diffv;
    }
  }  // layer loop
#undef SU
#undef SV
#undef SH
#undef G2
#undef COR
#undef Q
#undef SXY
#undef KE
#undef SXX
#undef UH
#undef VH
}

template <int TX, int TY, bool UNI, typename R, int MINB = 1, bool DIAG = false, int COR = 1,
          bool EXTV = false, bool FAST = false>
__global__ void __launch_bounds__(TX * TY, MINB)
k_tendency(Dims D, Metrics M, UniMetrics U, const R* __restrict__ uin,
           const R* __restrict__ vin, const R* __restrict__ h,
           const R* ubase, const R* vbase, R* uout, R* vout,
           R coef, R h_neglect, int k0, int KC, R* dfu = nullptr, R* dfv = nullptr)
{
    tendency_tile<TX, TY, UNI, R, DIAG, COR, EXTV, FAST>(D, M, U, uin, vin, h, ubase, vbase,
                                                         uout, vout, coef, h_neglect, k0, KC,
                                                         (int)blockIdx.x, (int)blockIdx.y,
                                                         (int)blockIdx.z, dfu, dfv);
}

// The FP64 Sadourny tendency with TMA-staged tiles; the tensor maps of uin,
// vin, h ride in the parameter bank.
struct TendMaps {
    CUtensorMap m[3];
};

template <int TX, int TY, bool UNI, int MINB, bool FAST>
__global__ void __launch_bounds__(TX * TY, MINB)
k_tendency_tma(Dims D, Metrics M, UniMetrics U, const __grid_constant__ TendMaps T,
               const double* __restrict__ uin, const double* __restrict__ vin,
               const double* __restrict__ h, const double* ubase, const double* vbase,
               double* uout, double* vout, double coef, double h_neglect, int k0, int KC,
               int* status)
{
    tendency_tile<TX, TY, UNI, double, false, 1, false, FAST, true>(
        D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, k0, KC,
        (int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, nullptr, nullptr, T.m, status);
}

// The tensor maps of a tendency's uin, vin, h ({TX + 2, TY + 2, 1} boxes);
// false when a field's layout does not qualify (odd n1, unaligned base).
inline bool tendency_maps(const Dims& D, const double* uin, const double* vin,
                          const double* h, int TX, int TY, TendMaps& T)
{
    return tma_map_cached(uin, D.n1, D.n2, D.nk, TX + 2, TY + 2, 1, &T.m[0]) &&
           tma_map_cached(vin, D.n1, D.n2, D.nk, TX + 2, TY + 2, 1, &T.m[1]) &&
           tma_map_cached(h, D.n1, D.n2, D.nk, TX + 2, TY + 2, 1, &T.m[2]) &&
           (D.is - 2) % 2 == 0;
}

// diffu, diffv from the general hor_visc kernel (EXTV), every Coriolis scheme.
template <typename R, int COR>
void launch_tendency_extv(const Dims& D, const Metrics& M, const UniMetrics& U, dim3 grid,
                          dim3 block, const R* uin, const R* vin, const R* h, const R* ubase,
                          const R* vbase, R* uout, R* vout, R coef, R h_neglect, int KC,
                          cudaStream_t s, R* dfu, R* dfv)
{
    constexpr int TX = 32, TY = 8;
    if (U.valid)
        k_tendency<TX, TY, true, R, 3, false, COR, true><<<grid, block, 0, s>>>(
            D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KC, dfu, dfv);
    else
        k_tendency<TX, TY, false, R, 3, false, COR, true><<<grid, block, 0, s>>>(
            D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KC, dfu, dfv);
}

// The Arakawa schemes (COR = 2, 3): both metric forms, with or without the
// diagnostic outputs, registers held to 3 CTAs/SM.
template <typename R, int COR>
cudaError_t launch_tendency_arakawa(const Dims& D, const Metrics& M, const UniMetrics& U,
                                    dim3 grid, dim3 block, const R* uin, const R* vin,
                                    const R* h, const R* ubase, const R* vbase, R* uout,
                                    R* vout, R coef, R h_neglect, int KC, cudaStream_t s, R* dfu,
                                    R* dfv)
{
    constexpr int TX = 32, TY = 8;
    if (dfu) {
        if (U.valid)
            k_tendency<TX, TY, true, R, 3, true, COR><<<grid, block, 0, s>>>(
                D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KC, dfu, dfv);
        else
            k_tendency<TX, TY, false, R, 3, true, COR><<<grid, block, 0, s>>>(
                D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KC, dfu, dfv);
    } else {
        if (U.valid)
            k_tendency<TX, TY, true, R, 3, false, COR><<<grid, block, 0, s>>>(
                D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KC);
        else
            k_tendency<TX, TY, false, R, 3, false, COR><<<grid, block, 0, s>>>(
                D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KC);
    }
    return cudaGetLastError();
}

constexpr int kTendTX = 32, kTendTY = 8, kTendKC = 15;

// Host launcher: one CTA per (TX x TY) tile of the compute domain and chunk of
// kTendKC layers (with the one-barrier TMA loop, 15 layers per CTA: 1.394 ms
// per step at 720x720x75 against 1.397 for 8 and 1.411 for 5 -- the first two
// layers of a chunk, requested up front, are the only loads a CTA waits for
// unhidden by its own work).
// dfu, dfv (both or neither): also store diffu, diffv (the diagnostic form of
// the kernel; the step's own launches pass neither).  scheme: the Coriolis
// scheme (1 SADOURNY75_ENERGY, 2 ARAKAWA_HSU90, 3 ARAKAWA_LAMB81).  FAST: the
// fast FP64 arithmetic, Sadourny scheme without the diagnostic outputs only.
template <typename R, bool FAST = false>
cudaError_t launch_tendency_t(const Dims& D, const Metrics& M, const UniMetrics& U,
                              const R* uin, const R* vin, const R* h, const R* ubase,
                              const R* vbase, R* uout, R* vout, R coef, R h_neglect,
                              cudaStream_t s, R* dfu = nullptr, R* dfv = nullptr,
                              int scheme = 1, bool ext_visc = false, int* status = nullptr)
{
    constexpr int TY = kTendTY;
    int nx = D.ie - D.is + 1, ny = D.je - D.js + 1;
    dim3 block(kTendTX, TY, 1);
    const int KCh = kTendKC;
    int nchunks = (D.nk + KCh - 1) / KCh;
    dim3 grid((nx + kTendTX - 1) / kTendTX, (ny + TY - 1) / TY, nchunks);
    if ((dfu == nullptr) != (dfv == nullptr)) return cudaErrorInvalidValue;
    if constexpr (FAST) {
        // only the plain Sadourny kernel exists in the fast form; the other
        // kernels are not instantiated here, so the exact translation unit's
        // instances (same template arguments) are the only ones linked
        if (ext_visc || dfu || scheme != 1) return cudaErrorInvalidValue;
        if constexpr (sizeof(R) == 8) {
            TendMaps T;
            if (U.valid && status && tendency_maps(D, uin, vin, h, kTendTX, TY, T)) {
                k_tendency_tma<kTendTX, TY, true, 4, true><<<grid, block, 0, s>>>(
                    D, M, U, T, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KCh,
                    status);
                return cudaGetLastError();
            }
        }
        if (U.valid)
            k_tendency<kTendTX, TY, true, R, 4, false, 1, false, true><<<grid, block, 0, s>>>(
                D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KCh);
        else
            k_tendency<kTendTX, TY, false, R, 3, false, 1, false, true><<<grid, block, 0, s>>>(
                D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KCh);
        return cudaGetLastError();
    } else {
    if (ext_visc) {
        if (!dfu || scheme < 1 || scheme > 3) return cudaErrorInvalidValue;
        if (scheme == 1)
            launch_tendency_extv<R, 1>(D, M, U, grid, block, uin, vin, h, ubase, vbase, uout,
                                       vout, coef, h_neglect, KCh, s, dfu, dfv);
        else if (scheme == 2)
            launch_tendency_extv<R, 2>(D, M, U, grid, block, uin, vin, h, ubase, vbase, uout,
                                       vout, coef, h_neglect, KCh, s, dfu, dfv);
        else
            launch_tendency_extv<R, 3>(D, M, U, grid, block, uin, vin, h, ubase, vbase, uout,
                                       vout, coef, h_neglect, KCh, s, dfu, dfv);
        return cudaGetLastError();
    }
    if (scheme == 2)
        return launch_tendency_arakawa<R, 2>(D, M, U, grid, block, uin, vin, h, ubase, vbase,
                                             uout, vout, coef, h_neglect, KCh, s, dfu, dfv);
    if (scheme == 3)
        return launch_tendency_arakawa<R, 3>(D, M, U, grid, block, uin, vin, h, ubase, vbase,
                                             uout, vout, coef, h_neglect, KCh, s, dfu, dfv);
    if (scheme != 1) return cudaErrorInvalidValue;
    if (dfu || dfv) {
        if (U.valid)
            k_tendency<kTendTX, TY, true, R, 3, true><<<grid, block, 0, s>>>(
                D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KCh,
                dfu, dfv);
        else
            k_tendency<kTendTX, TY, false, R, 3, true><<<grid, block, 0, s>>>(
                D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KCh,
                dfu, dfv);
        return cudaGetLastError();
    }
    // CTAs per SM the registers are held to: 4 (64 registers) is the fastest
    // uniform-metric form on B200 (FP64 tendency 2.01 ms per step against 2.13
    // at 3 and 2.62 uncapped); the 2-D metric form keeps 3 (80 registers).
    if constexpr (sizeof(R) == 8) {
        TendMaps T;
        if (U.valid && status && tendency_maps(D, uin, vin, h, kTendTX, TY, T)) {
            k_tendency_tma<kTendTX, TY, true, 4, false><<<grid, block, 0, s>>>(
                D, M, U, T, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KCh,
                status);
            return cudaGetLastError();
        }
    }
    if (U.valid)
        k_tendency<kTendTX, TY, true, R, 4><<<grid, block, 0, s>>>(
            D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KCh);
    else
        k_tendency<kTendTX, TY, false, R, 3><<<grid, block, 0, s>>>(
            D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef, h_neglect, 1, KCh);
    return cudaGetLastError();
    }
}

} // namespace mom6b
