// k_btstep.cu -- the barotropic substep loop as one persistent kernel (FP64).
//
// Restates btstep + update_u/update_v of mom6_barotropic_serial.F90:178-356:
// nstep substeps of eta prediction, pressure force, alternating Coriolis
// updates of ubt/vbt, bebt-weighted transports, eta update and time averages.
// The reference CUDA C backend issues 9 launches per substep from the host
// (mom6_barotropic_cuda_c.F90:348-422); here one cooperative launch runs the
// whole loop and separates the phases with a grid-wide barrier, three per
// substep:
//   A  ubt_prev/vbt_prev copies and eta_pred            (needs old ubt, vbt, eta)
//   B  PFu, PFv and the first velocity update           (needs eta_pred of neighbours)
//   C  the second update, uhbt/vhbt, the averages       (needs the first update)
//   D  eta update, then phase A of the next substep     (needs uhbt(i-1), vhbt(j-1))
// Every thread owns the same points in every phase, so values a thread both
// writes and reads within a phase need no barrier.  The 2-D state (a few MB)
// stays in L2 across the whole loop.
//
// Two transport ranges are supported: the serial module's (uhbt on
// [is, ie-1], vhbt on [js, je-1], ubt_av/vbt_av likewise; uhbt(is-1),
// uhbt(ie), vhbt(js-1), vhbt(je) stay zero, :263-291) and the extended ranges
// of btstep_do_step and the CUDA C kernels ([is-1, ie] / [js-1, je],
// :443-452).  The barrier spins with a clock64 budget; when it expires the
// kernel records kDevTimeout and every block returns.
#include <cstdlib>

#include "../../include/mom6b.h"
#include "halo_impl.cuh"
#include "kernels.h"

namespace mom6b {

// Global home of the per-point private quantities when they do not fit in
// shared memory.
__device__ __forceinline__ double* priv_global(const BTWork& W, int q, int p)
{
    switch (q) {
    case 0: return W.ubt_prev + p;
    case 1: return W.vbt_prev + p;
    case 2: return W.PFu + p;
    case 3: return W.PFv + p;
    case 4: return W.ubt_av + p;
    default: return W.vbt_av + p;
    }
}

// Sense-counting grid barrier.  Returns false when the wait budget ran out
// (or another block reported a timeout); callers then return.
__device__ __forceinline__ bool grid_barrier(const BTWork& W, unsigned int nblocks,
                                             long long budget)
{
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        volatile unsigned int* gen = W.bar_gen;
        volatile int* st = W.status;
        unsigned int g = *gen;
        __threadfence();
        unsigned int arrived = atomicAdd(W.bar_count, 1u);
        int ok = 1;
        if (arrived == nblocks - 1) {
            atomicExch(W.bar_count, 0u);
            __threadfence();
            atomicAdd(W.bar_gen, 1u);
        } else {
            long long t0 = clock64();
            unsigned int spins = 0;
            while (*gen == g) {
                if ((++spins & 63u) == 0) {
                    if (*st != kDevOk) { ok = 0; break; }
                    if (clock64() - t0 > budget) {
                        atomicExch(W.status, kDevTimeout);
                        ok = 0;
                        break;
                    }
                    if (spins > 4096u) __nanosleep(64);
                }
            }
        }
        __threadfence();
        s_ok = ok && (*st == kDevOk);
    }
    __syncthreads();
    return s_ok != 0;
}

// Points are owned per thread inside the active box [is-1, ie+1] x
// [js-1, je+1] (nothing outside it changes during the loop).  With FAST, a
// thread owns at most kBtMaxR points, caches their (i, j) in registers and
// keeps the quantities only it reads (ubt_prev, vbt_prev, PFu, PFv, ubt_av,
// vbt_av) in shared memory; otherwise indices are recomputed per phase and
// those quantities live in the global work arrays (any grid size).
constexpr int kBtThreads = 1024, kBtMaxR = 4;
enum { PV_PREVU = 0, PV_PREVV, PV_PFU, PV_PFV, PV_AVU, PV_AVV, PV_N };

template <bool FAST>
__global__ void __launch_bounds__(kBtThreads, 1)
k_btstep(Dims D, Metrics M, BTWork W, BTParams P, const double* eta_in,
         const double* ubt_in, const double* vbt_in, double* u_av, double* v_av,
         double* eta_av)
{
    extern __shared__ double s_priv[];  // [PV_N][kBtMaxR][blockDim.x] when FAST
    const unsigned int nblocks = gridDim.x;
    const int npts = D.n1 * D.n2;
    const int gtid = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int gsz = (int)(gridDim.x * blockDim.x);
    const int is = D.is, ie = D.ie, js = D.js, je = D.je;
    // A subdomain of a decomposed run reaches two points into the halo at a
    // cut, so that a substep's values at the owned points need only the halo
    // exchanged before it (a new eta reads the old ubt, vbt, eta up to two
    // points away).  Without cuts these are the serial ranges: cells
    // [ci0, ci1] x [cj0, cj1], u faces to ui1, v faces to vj1.
    const int xw = 2 * D.cw, xe = 2 * D.ce, xs = 2 * D.cs, xn = 2 * D.cn;
    const int ci0 = is - xw, ci1 = ie + xe, cj0 = js - xs, cj1 = je + xn;
    const int ui1 = ie - 1 + xe, vj1 = je - 1 + xn;
    // serial ranges vs. extended ranges for uhbt/vhbt and the averages
    const int iu0 = xw ? ci0 : (P.extended ? is - 1 : is);
    const int iu1 = xe ? ui1 : (P.extended ? ie : ie - 1);
    const int jv0 = xs ? cj0 : (P.extended ? js - 1 : js);
    const int jv1 = xn ? vj1 : (P.extended ? je : je - 1);
    const int bx0 = is - 1 - xw, by0 = js - 1 - xs;   // active box origin
    const int bw = ie - is + 3 + xw + xe;             // active box width
    const int nbox = bw * (je - js + 3 + xs + xn);
    const int nr = FAST ? (nbox - gtid + gsz - 1) / gsz : 0;
#define A(a, ii, jj) MOM6B_A2(a, ii, jj, D)
#define PV(q, r, p) (*(FAST ? &s_priv[((q) * kBtMaxR + (r)) * blockDim.x + threadIdx.x] \
                            : priv_global(W, q, p)))

    int pi[kBtMaxR], pj[kBtMaxR], pp[kBtMaxR];
    if (FAST) {
#pragma unroll
        for (int r = 0; r < kBtMaxR; ++r) {
            int q = gtid + r * gsz;
            pi[r] = bx0 + q % bw;
            pj[r] = by0 + q / bw;
            pp[r] = (pj[r] - 1) * D.n1 + (pi[r] - 1);
#pragma unroll
            for (int v = 0; v < PV_N; ++v)
                s_priv[(v * kBtMaxR + r) * blockDim.x + threadIdx.x] = 0.0;
        }
    }
    // visit every owned point: f(r, i, j, p)
    auto for_points = [&](auto&& f) {
        if (FAST) {
#pragma unroll
            for (int r = 0; r < kBtMaxR; ++r) {
                if (r >= nr) break;
                f(r, pi[r], pj[r], pp[r]);
            }
        } else {
            for (int q = gtid; q < nbox; q += gsz) {
                int i = bx0 + q % bw, j = by0 + q / bw;
                f(0, i, j, (j - 1) * D.n1 + (i - 1));
            }
        }
    };

    // init (:199-207): state copies over the whole data domain
    if (P.substep == 0 || P.substep == kBtInit) {
        for (int p = gtid; p < npts; p += gsz) {
            W.eta[p] = eta_in[p];
            W.ubt[p] = ubt_in[p];
            W.vbt[p] = vbt_in[p];
            if (!FAST) { W.ubt_av[p] = 0.0; W.vbt_av[p] = 0.0; }
        }
        if (!grid_barrier(W, nblocks + (unsigned)P.stall_test, P.spin_budget)) return;
        if (P.substep == kBtInit) return;
    }

    auto phase_A = [&]() {
        for_points([&](int r, int i, int j, int p) {
            if (j >= cj0 && j <= cj1) PV(PV_PREVU, r, p) = W.ubt[p];  // i: the box's
            if (i >= ci0 && i <= ci1) PV(PV_PREVV, r, p) = W.vbt[p];  // j: the box's
            if (i >= ci0 && i <= ci1 && j >= cj0 && j <= cj1)
                W.eta_pred[p] =
                    W.eta[p] + (P.dtbt * A(M.IareaT, i, j)) *
                                   (((A(M.Datu, i - 1, j) * A(W.ubt, i - 1, j)) -
                                     (A(M.Datu, i, j) * W.ubt[p])) +
                                    ((A(M.Datv, i, j - 1) * A(W.vbt, i, j - 1)) -
                                     (A(M.Datv, i, j) * W.vbt[p])));
        });
    };
    auto update_u = [&](int p, int i, int j, double PFu) {
        double Cor_u = (((MOM6B_F4(M.f_4_u, 4, i, j, D) * A(W.vbt, i + 1, j)) +
                         (MOM6B_F4(M.f_4_u, 1, i, j, D) * A(W.vbt, i, j - 1))) +
                        ((MOM6B_F4(M.f_4_u, 3, i, j, D) * W.vbt[p]) +
                         (MOM6B_F4(M.f_4_u, 2, i, j, D) * A(W.vbt, i + 1, j - 1))));
        W.ubt[p] = A(M.bt_rem_u, i, j) * (W.ubt[p] + P.dtbt * (Cor_u + PFu));
    };
    auto update_v = [&](int p, int i, int j, double PFv) {
        double Cor_v = -1.0 * (((MOM6B_F4(M.f_4_v, 1, i, j, D) * A(W.ubt, i - 1, j)) +
                                (MOM6B_F4(M.f_4_v, 4, i, j, D) * A(W.ubt, i, j + 1))) +
                               ((MOM6B_F4(M.f_4_v, 2, i, j, D) * W.ubt[p]) +
                                (MOM6B_F4(M.f_4_v, 3, i, j, D) * A(W.ubt, i - 1, j + 1))));
        W.vbt[p] = A(M.bt_rem_v, i, j) * (W.vbt[p] + P.dtbt * (Cor_v + PFv));
    };

    const int n0 = P.substep > 0 ? P.substep : 1, n1 = P.substep > 0 ? P.substep : P.nstep;
    if (P.substep != kBtFinish) {
    phase_A();
    if (!grid_barrier(W, nblocks, P.spin_budget)) return;

    for (int n = n0; n <= n1; ++n) {
        const bool v_first = ((n + P.first_direction) % 2) == 1;
        // phase B: pressure force (:234-247) and the first update
        for_points([&](int r, int i, int j, int p) {
            if (j >= cj0 && j <= cj1 && i >= ci0 && i <= ui1)
                PV(PV_PFU, r, p) = ((W.eta_pred[p] * A(M.gtot_E, i, j)) -
                                    (A(W.eta_pred, i + 1, j) * A(M.gtot_W, i + 1, j))) *
                                   P.dgeo_de * A(M.IdxCu, i, j);
            if (j >= cj0 && j <= vj1 && i >= ci0 && i <= ci1)
                PV(PV_PFV, r, p) = ((W.eta_pred[p] * A(M.gtot_N, i, j)) -
                                    (A(W.eta_pred, i, j + 1) * A(M.gtot_S, i, j + 1))) *
                                   P.dgeo_de * A(M.IdyCv, i, j);
            if (v_first) {
                if (i >= ci0 && i <= ci1 && j >= cj0 && j <= vj1)
                    update_v(p, i, j, PV(PV_PFV, r, p));
            } else {
                if (i >= ci0 && i <= ui1 && j >= cj0 && j <= cj1)
                    update_u(p, i, j, PV(PV_PFU, r, p));
            }
        });
        if (!grid_barrier(W, nblocks, P.spin_budget)) return;
        // phase C: second update, transports (:263-272), averages (:282-291)
        for_points([&](int r, int i, int j, int p) {
            if (v_first) {
                if (i >= ci0 && i <= ui1 && j >= cj0 && j <= cj1)
                    update_u(p, i, j, PV(PV_PFU, r, p));
            } else {
                if (i >= ci0 && i <= ci1 && j >= cj0 && j <= vj1)
                    update_v(p, i, j, PV(PV_PFV, r, p));
            }
            if (j >= cj0 && j <= cj1 && i >= iu0 && i <= iu1) {
                double ub = W.ubt[p];
                W.uhbt[p] = A(M.Datu, i, j) * (P.trans_wt1 * ub + P.trans_wt2 * PV(PV_PREVU, r, p));
                PV(PV_AVU, r, p) = PV(PV_AVU, r, p) + ub * P.inv_nstep;
            }
            if (j >= jv0 && j <= jv1 && i >= ci0 && i <= ci1) {
                double vb = W.vbt[p];
                W.vhbt[p] = A(M.Datv, i, j) * (P.trans_wt1 * vb + P.trans_wt2 * PV(PV_PREVV, r, p));
                PV(PV_AVV, r, p) = PV(PV_AVV, r, p) + vb * P.inv_nstep;
            }
        });
        if (!grid_barrier(W, nblocks, P.spin_budget)) return;
        // phase D: eta update (:274-279), then phase A of the next substep
        for_points([&](int r, int i, int j, int p) {
            if (i >= ci0 && i <= ci1 && j >= cj0 && j <= cj1)
                W.eta[p] = W.eta[p] - P.dtbt * A(M.IareaT, i, j) *
                                          ((W.uhbt[p] - A(W.uhbt, i - 1, j)) +
                                           (W.vhbt[p] - A(W.vhbt, i, j - 1)));
        });
        // eta_pred(i,j) needs only this thread's new eta(i,j); the velocity
        // neighbours were final before the last barrier
        if (n < n1) phase_A();
        if (!grid_barrier(W, nblocks, P.spin_budget)) return;
    }
    }
    if (P.substep > 0) return;
    // copy output (:296-302); outputs may alias the inputs.  The averages are
    // zero outside their ranges (the init of :204-205).
    if (FAST) {
        for (int p = gtid; p < npts; p += gsz) {
            u_av[p] = 0.0;
            v_av[p] = 0.0;
            eta_av[p] = W.eta[p];
        }
        if (!grid_barrier(W, nblocks, P.spin_budget)) return;
        for_points([&](int r, int i, int j, int p) {
            u_av[p] = PV(PV_AVU, r, p);
            v_av[p] = PV(PV_AVV, r, p);
        });
    } else {
        for (int p = gtid; p < npts; p += gsz) {
            u_av[p] = W.ubt_av[p];
            v_av[p] = W.vbt_av[p];
            eta_av[p] = W.eta[p];
        }
    }
#undef A
#undef PV
}

// ---------------------------------------------------------------------------
// Tiled variant: one grid barrier per substep.
// ---------------------------------------------------------------------------
// The updated box [is-1, ie] x [js-1, je] is split into nbx x nby tiles, one
// per CTA.  Each substep a CTA loads the previous eta/ubt/vbt on its tile
// widened by two points below and one above, recomputes eta_pred, the two
// velocity updates and the transports on the halo it needs, and writes its
// own tile's new state to the other buffer; a single grid barrier then ends
// the substep.  The evaluation order of every point is the serial one.  The
// averages of the owned points stay in registers (at most kBtTileR per
// thread).
constexpr int kBtTileR = 4;

struct BTTiles {
    int nbx, nby, tw, th;  // tiles and tile size
    int nt;                // threads per CTA: 1024 (tiles <= 64 x 64, one CTA per SM)
                           // or 512 (tiles <= 64 x 32, two CTAs per SM)
};

// Wait until every tile in nb[0..nnb) has published substep `target` (its
// tile_flag reached it).  Lanes of warp 0 each watch one neighbour with the
// clock64 budget; false when the budget ran out or another block failed.
__device__ __forceinline__ bool wait_neighbours(const BTWork& W, const int* nb, int nnb,
                                                unsigned int target, long long budget)
{
    __shared__ int s_wok;
    if (threadIdx.x < 32) {
        int ok = 1;
        if ((int)threadIdx.x < nnb) {
            volatile unsigned int* fl = W.tile_flag + nb[threadIdx.x];
            volatile int* st = W.status;
            long long t0 = clock64();
            unsigned int spins = 0;
            while (*fl < target) {
                if ((++spins & 63u) == 0) {
                    if (*st != kDevOk) { ok = 0; break; }
                    if (clock64() - t0 > budget) {
                        atomicExch(W.status, kDevTimeout);
                        ok = 0;
                        break;
                    }
                    if (spins > 4096u) __nanosleep(32);
                }
            }
        }
        ok = __all_sync(0xffffffffu, ok);
        __threadfence();
        if (threadIdx.x == 0) s_wok = ok;
    }
    __syncthreads();
    return s_wok != 0;
}

// TAVG: also accumulate the substep-averaged transports (1/nstep) sum_n
// uhbt_n, vhbt_n of the owned points into W.uhbt / W.vhbt (the surrogate's
// training targets; zero outside their ranges).
template <int NT, bool UNI, bool TAVG>
__global__ void __launch_bounds__(NT, 1024 / NT)
k_btstep_tiled(Dims D, Metrics M, UniMetrics U, BTWork W, BTParams P, BTTiles T,
               const double* eta_in, const double* ubt_in, const double* vbt_in,
               double* u_av, double* v_av, double* eta_av)
{
    extern __shared__ double smem[];
    const unsigned int nblocks = gridDim.x;
    const int tid = (int)threadIdx.x;
    const int txl = tid & 31, tyl = tid >> 5;        // 32 x (NT/32) layout over the tile
    constexpr int TY = NT / 32;
    const int npts = D.n1 * D.n2;
    const int gtid = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int gsz = (int)(gridDim.x * blockDim.x);
    const int is = D.is, ie = D.ie, js = D.js, je = D.je;
    const int iu0 = P.extended ? is - 1 : is, iu1 = P.extended ? ie : ie - 1;
    const int jv0 = P.extended ? js - 1 : js, jv1 = P.extended ? je : je - 1;
    const int tx = (int)blockIdx.x % T.nbx, ty = (int)blockIdx.x / T.nbx;
    const int x0 = is - 1 + tx * T.tw, y0 = js - 1 + ty * T.th;
    const int x1 = min(x0 + T.tw - 1, ie), y1 = min(y0 + T.th - 1, je);
    const int lx0 = x0 - 2, ly0 = y0 - 2;              // local origin
    const int LW = T.tw + 3, LH = T.th + 3;
    const int LN = LW * LH;
    double* Se = smem;            // eta, previous substep
    double* Su = Se + LN;         // ubt, previous substep (= ubt_prev)
    double* Sv = Su + LN;         // vbt, previous substep (= vbt_prev)
    double* Sp = Sv + LN;         // eta_pred
    double* Sun = Sp + LN;        // ubt after this substep
    double* Svn = Sun + LN;       // vbt after this substep
#define L(a, i, j) a[((j) - ly0) * LW + ((i) - lx0)]
#define G(a, i, j) MOM6B_A2(a, i, j, D)
#define GM(f, i, j) (UNI ? U.f : MOM6B_A2(M.f, i, j, D))
#define F4U(c, i, j) (UNI ? U.f4u_row[((j) - 1) * 4 + (c) - 1] : MOM6B_F4(M.f_4_u, c, i, j, D))
#define F4V(c, i, j) (UNI ? U.f4v_row[((j) - 1) * 4 + (c) - 1] : MOM6B_F4(M.f_4_v, c, i, j, D))

    // averages of the owned points (x0 + txl + 32a, y0 + tyl + TY b), a, b in
    // {0, 1}, kept in registers; a tile beyond the box owns nothing
    double avu[kBtTileR], avv[kBtTileR];
#pragma unroll
    for (int r = 0; r < kBtTileR; ++r) avu[r] = avv[r] = 0.0;

    // init (:199-207): both buffers hold the whole input state
    for (int p = gtid; p < npts; p += gsz) {
        double e = eta_in[p], ub = ubt_in[p], vb = vbt_in[p];
        W.eta[p] = e; W.ubt[p] = ub; W.vbt[p] = vb;
        W.eta_pred[p] = e; W.ubt_prev[p] = ub; W.vbt_prev[p] = vb;
        if (TAVG) { W.uhbt[p] = 0.0; W.vhbt[p] = 0.0; }
    }
    if (tid == 0) W.tile_flag[blockIdx.x] = 0u;
    if (!grid_barrier(W, nblocks + (unsigned)P.stall_test, P.spin_budget)) return;

    // the (up to 8) tiles whose points lie in this tile's width-2 halo
    int nbr[8];
    int nnb = 0;
    for (int dyt = -1; dyt <= 1; ++dyt)
        for (int dxt = -1; dxt <= 1; ++dxt) {
            const int ax = tx + dxt, ay = ty + dyt;
            if ((dxt || dyt) && ax >= 0 && ax < T.nbx && ay >= 0 && ay < T.nby)
                nbr[nnb++] = ay * T.nbx + ax;
        }

    for (int n = 1; n <= P.nstep; ++n) {
        const bool v_first = ((n + P.first_direction) % 2) == 1;
        const double* ce = (n & 1) ? W.eta : W.eta_pred;
        const double* cu = (n & 1) ? W.ubt : W.ubt_prev;
        const double* cv = (n & 1) ? W.vbt : W.vbt_prev;
        double* ne = (n & 1) ? W.eta_pred : W.eta;
        double* nu = (n & 1) ? W.ubt_prev : W.ubt;
        double* nv = (n & 1) ? W.vbt_prev : W.vbt;
        // S1: previous state on the local window.  Owned points carry over in
        // shared memory (new eta in Sp, new ubt/vbt in Sun/Svn); the halo comes
        // from the neighbours' published buffers once they finished substep n-1.
        if (n > 1 && !wait_neighbours(W, nbr, nnb, (unsigned int)(n - 1), P.spin_budget)) return;
        if (n == 1) {
            for (int jl = tyl; jl < LH; jl += TY)
            for (int il = txl; il < LW; il += 32) {
                const int q = jl * LW + il, i = lx0 + il, j = ly0 + jl;
                double e = 0.0, ub = 0.0, vb = 0.0;
                if (i >= 1 && i <= D.n1 && j >= 1 && j <= D.n2) {
                    int p = (j - 1) * D.n1 + (i - 1);
                    e = __ldcg(ce + p); ub = __ldcg(cu + p); vb = __ldcg(cv + p);
                }
                Se[q] = e; Su[q] = ub; Sv[q] = vb; Sun[q] = ub; Svn[q] = vb;
            }
        } else {
            // owned points: each thread's own, already in shared memory
#pragma unroll
            for (int r = 0; r < kBtTileR; ++r) {
                const int i = x0 + txl + 32 * (r & 1), j = y0 + tyl + TY * (r >> 1);
                if (i > x1 || j > y1) continue;
                const int q = (j - ly0) * LW + (i - lx0);
                Se[q] = Sp[q]; Su[q] = Sun[q]; Sv[q] = Svn[q];
            }
            // the ring of the window around the owned rectangle, one flat index
            // per point, so a thread's loads are all in flight at once
            const int nb = y0 - ly0, na = (ly0 + LH - 1) - y1;
            const int nl = x0 - lx0, nr = (lx0 + LW - 1) - x1;
            const int mid = y1 - y0 + 1, side = nl + nr;
            const int nring = (nb + na) * LW + mid * side;
            for (int t = tid; t < nring; t += NT) {
                int i, j;
                if (t < nb * LW) {
                    j = ly0 + t / LW; i = lx0 + t % LW;
                } else if (t < (nb + na) * LW) {
                    const int t2 = t - nb * LW;
                    j = y1 + 1 + t2 / LW; i = lx0 + t2 % LW;
                } else {
                    const int t3 = t - (nb + na) * LW;
                    const int c = t3 % side;
                    j = y0 + t3 / side;
                    i = c < nl ? lx0 + c : x1 + 1 + (c - nl);
                }
                const int q = (j - ly0) * LW + (i - lx0);
                double e = 0.0, ub = 0.0, vb = 0.0;
                if (i >= 1 && i <= D.n1 && j >= 1 && j <= D.n2) {
                    int p = (j - 1) * D.n1 + (i - 1);
                    e = __ldcg(ce + p); ub = __ldcg(cu + p); vb = __ldcg(cv + p);
                }
                Se[q] = e; Su[q] = ub; Sv[q] = vb; Sun[q] = ub; Svn[q] = vb;
            }
        }
        __syncthreads();
        // S2: eta_pred on [x0-1, x1+1] x [y0-1, y1+1] within [is, ie] x [js, je]
        {
            int a0 = max(x0 - 1, is), a1 = min(x1 + 1, ie);
            int b0 = max(y0 - 1, js), b1 = min(y1 + 1, je);
            for (int j = b0 + tyl; j <= b1; j += TY)
            for (int i = a0 + txl; i <= a1; i += 32) {
                L(Sp, i, j) = L(Se, i, j) + (P.dtbt * GM(IareaT, i, j)) *
                                                (((GM(Datu, i - 1, j) * L(Su, i - 1, j)) -
                                                  (GM(Datu, i, j) * L(Su, i, j))) +
                                                 ((GM(Datv, i, j - 1) * L(Sv, i, j - 1)) -
                                                  (GM(Datv, i, j) * L(Sv, i, j))));
            }
        }
        __syncthreads();
        auto upd_u = [&](int i, int j, const double* Vsrc) {
            double PFu = ((L(Sp, i, j) * GM(gtot_E, i, j)) -
                          (L(Sp, i + 1, j) * GM(gtot_W, i + 1, j))) *
                         P.dgeo_de * GM(IdxCu, i, j);
            double Cor_u = (((F4U(4, i, j) * L(Vsrc, i + 1, j)) +
                             (F4U(1, i, j) * L(Vsrc, i, j - 1))) +
                            ((F4U(3, i, j) * L(Vsrc, i, j)) +
                             (F4U(2, i, j) * L(Vsrc, i + 1, j - 1))));
            L(Sun, i, j) = GM(bt_rem_u, i, j) * (L(Su, i, j) + P.dtbt * (Cor_u + PFu));
        };
        auto upd_v = [&](int i, int j, const double* Usrc) {
            double PFv = ((L(Sp, i, j) * GM(gtot_N, i, j)) -
                          (L(Sp, i, j + 1) * GM(gtot_S, i, j + 1))) *
                         P.dgeo_de * GM(IdyCv, i, j);
            double Cor_v = -1.0 * (((F4V(1, i, j) * L(Usrc, i - 1, j)) +
                                    (F4V(4, i, j) * L(Usrc, i, j + 1))) +
                                   ((F4V(2, i, j) * L(Usrc, i, j)) +
                                    (F4V(3, i, j) * L(Usrc, i - 1, j + 1))));
            L(Svn, i, j) = GM(bt_rem_v, i, j) * (L(Sv, i, j) + P.dtbt * (Cor_v + PFv));
        };
        // S3 / S4: the two velocity updates on the regions the tile needs
        if (v_first) {
            int a0 = max(x0 - 1, is), a1 = min(x1 + 1, ie);
            int b0 = max(y0 - 1, js), b1 = min(y1, je - 1);
            for (int j = b0 + tyl; j <= b1; j += TY)
            for (int i = a0 + txl; i <= a1; i += 32) upd_v(i, j, Su);
            __syncthreads();
            a0 = max(x0 - 1, is); a1 = min(x1, ie - 1);
            b0 = max(y0, js); b1 = min(y1, je);
            for (int j = b0 + tyl; j <= b1; j += TY)
            for (int i = a0 + txl; i <= a1; i += 32) upd_u(i, j, Svn);
        } else {
            int a0 = max(x0 - 1, is), a1 = min(x1, ie - 1);
            int b0 = max(y0 - 1, js), b1 = min(y1 + 1, je);
            for (int j = b0 + tyl; j <= b1; j += TY)
            for (int i = a0 + txl; i <= a1; i += 32) upd_u(i, j, Sv);
            __syncthreads();
            a0 = max(x0, is); a1 = min(x1, ie);
            b0 = max(y0 - 1, js); b1 = min(y1, je - 1);
            for (int j = b0 + tyl; j <= b1; j += TY)
            for (int i = a0 + txl; i <= a1; i += 32) upd_v(i, j, Sun);
        }
        __syncthreads();
        // S5: transports, eta update and averages on the owned points
        auto uhbt_at = [&](int i, int j) -> double {
            if (i < iu0 || i > iu1 || j < js || j > je) return 0.0;
            return GM(Datu, i, j) * (P.trans_wt1 * L(Sun, i, j) + P.trans_wt2 * L(Su, i, j));
        };
        auto vhbt_at = [&](int i, int j) -> double {
            if (j < jv0 || j > jv1 || i < is || i > ie) return 0.0;
            return GM(Datv, i, j) * (P.trans_wt1 * L(Svn, i, j) + P.trans_wt2 * L(Sv, i, j));
        };
#pragma unroll
        for (int r = 0; r < kBtTileR; ++r) {
            const int i = x0 + txl + 32 * (r & 1), j = y0 + tyl + TY * (r >> 1);
            if (i > x1 || j > y1) continue;
            int p = (j - 1) * D.n1 + (i - 1);
            double e = L(Se, i, j);
            if (i >= is && i <= ie && j >= js && j <= je) {
                e = L(Se, i, j) - P.dtbt * GM(IareaT, i, j) *
                                      ((uhbt_at(i, j) - uhbt_at(i - 1, j)) +
                                       (vhbt_at(i, j) - vhbt_at(i, j - 1)));
                ne[p] = e;
            }
            L(Sp, i, j) = e;   // eta_pred is dead: it carries the new eta
            if (i >= is && i <= ie - 1 && j >= js && j <= je) nu[p] = L(Sun, i, j);
            if (i >= is && i <= ie && j >= js && j <= je - 1) nv[p] = L(Svn, i, j);
            if (j >= js && j <= je && i >= iu0 && i <= iu1)
                avu[r] = avu[r] + L(Sun, i, j) * P.inv_nstep;
            if (j >= jv0 && j <= jv1 && i >= is && i <= ie)
                avv[r] = avv[r] + L(Svn, i, j) * P.inv_nstep;
            if (TAVG) {
                if (j >= js && j <= je && i >= iu0 && i <= iu1)
                    W.uhbt[p] = W.uhbt[p] + uhbt_at(i, j) * P.inv_nstep;
                if (j >= jv0 && j <= jv1 && i >= is && i <= ie)
                    W.vhbt[p] = W.vhbt[p] + vhbt_at(i, j) * P.inv_nstep;
            }
        }
        // publish substep n: every global write of this tile is done
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicExch(W.tile_flag + blockIdx.x, (unsigned int)n);
        }
    }
    if (!grid_barrier(W, nblocks, P.spin_budget)) return;
    // outputs (:296-302); they may alias the inputs
    const double* fe = (P.nstep & 1) ? W.eta_pred : W.eta;
    for (int p = gtid; p < npts; p += gsz) {
        eta_av[p] = fe[p];
        int i = p % D.n1 + 1, j = p / D.n1 + 1;
        if (i < is - 1 || i > ie || j < js - 1 || j > je) {  // not owned by a tile
            u_av[p] = 0.0;
            v_av[p] = 0.0;
        }
    }
#pragma unroll
    for (int r = 0; r < kBtTileR; ++r) {
        const int i = x0 + txl + 32 * (r & 1), j = y0 + tyl + TY * (r >> 1);
        if (i > x1 || j > y1) continue;
        int p = (j - 1) * D.n1 + (i - 1);
        u_av[p] = avu[r];
        v_av[p] = avv[r];
    }
#undef L
#undef G
#undef GM
#undef F4U
#undef F4V
}

// ---------------------------------------------------------------------------
// Slot variant of the tiled loop (1024 threads, tiles of at most 62 x 62):
// thread (txl, tyl) owns the four points (x0 - 1 + txl + 32 a, y0 - 1 + tyl +
// 32 b), a, b in {0, 1}, of the 64 x 64 window that covers the tile and its
// one-point rim, in every phase.  Each point's shared-memory offset and its
// membership of every phase's region are worked out once, so a phase is
// straight-line code over four slots.  A point's x neighbours belong to the
// same warp, so the barrier between eta_pred and a first update of u is a
// warp barrier.  The arithmetic of every point is k_btstep_tiled's.
// ---------------------------------------------------------------------------
enum : unsigned {
    SB_ETA = 1u << 0,   // eta_pred
    SB_V1 = 1u << 1,    // v update, v first
    SB_U2 = 1u << 2,    // u update, v first
    SB_U1 = 1u << 3,    // u update, u first
    SB_V2 = 1u << 4,    // v update, u first
    SB_OWN = 1u << 5,   // owned point of the tile
    SB_E = 1u << 6,     // eta update
    SB_NU = 1u << 7,    // ubt published
    SB_NV = 1u << 8,    // vbt published
    SB_AU = 1u << 9,    // uhbt(i, j) / ubt average range
    SB_AV = 1u << 10,   // vhbt(i, j) / vbt average range
    SB_UL = 1u << 11,   // uhbt(i - 1, j) range
    SB_VL = 1u << 12,   // vhbt(i, j - 1) range
};

template <bool UNI, bool TAVG>
__global__ void __launch_bounds__(1024, 1)
k_btstep_slots(Dims D, Metrics M, UniMetrics U, BTWork W, BTParams P, BTTiles T,
               const double* eta_in, const double* ubt_in, const double* vbt_in,
               double* u_av, double* v_av, double* eta_av)
{
    constexpr int NT = 1024, TY = 32;
    extern __shared__ double smem[];
    const unsigned int nblocks = gridDim.x;
    const int tid = (int)threadIdx.x;
    const int txl = tid & 31, tyl = tid >> 5;
    const int npts = D.n1 * D.n2;
    const int gtid = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int gsz = (int)(gridDim.x * blockDim.x);
    const int is = D.is, ie = D.ie, js = D.js, je = D.je;
    const int iu0 = P.extended ? is - 1 : is, iu1 = P.extended ? ie : ie - 1;
    const int jv0 = P.extended ? js - 1 : js, jv1 = P.extended ? je : je - 1;
    const int tx = (int)blockIdx.x % T.nbx, ty = (int)blockIdx.x / T.nbx;
    const int x0 = is - 1 + tx * T.tw, y0 = js - 1 + ty * T.th;
    const int x1 = min(x0 + T.tw - 1, ie), y1 = min(y0 + T.th - 1, je);
    const int lx0 = x0 - 2, ly0 = y0 - 2;
    const int LW = T.tw + 3, LH = T.th + 3;
    const int LN = LW * LH;
    double* Se = smem;
    double* Su = Se + LN;
    double* Sv = Su + LN;
    double* Sp = Sv + LN;
    double* Sun = Sp + LN;
    double* Svn = Sun + LN;
#define GM(f, i, j) (UNI ? U.f : MOM6B_A2(M.f, i, j, D))
#define F4U(c, i, j) (UNI ? U.f4u_row[((j) - 1) * 4 + (c) - 1] : MOM6B_F4(M.f_4_u, c, i, j, D))
#define F4V(c, i, j) (UNI ? U.f4v_row[((j) - 1) * 4 + (c) - 1] : MOM6B_F4(M.f_4_v, c, i, j, D))
#define SI(r) (x0 - 1 + txl + 32 * ((r) & 1))
#define SJ(r) (y0 - 1 + tyl + TY * ((r) >> 1))
#define SQ(r) (q0 + 32 * ((r) & 1) + TY * LW * ((r) >> 1))

    // shared offset of slot 0 and the phase regions of the four slots
    const int q0 = (tyl + 1) * LW + (txl + 1);
    unsigned mk[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int i = SI(r), j = SJ(r);
        auto in = [&](int a0, int a1, int b0, int b1) {
            return i >= a0 && i <= a1 && j >= b0 && j <= b1;
        };
        unsigned m = 0;
        if (in(max(x0 - 1, is), min(x1 + 1, ie), max(y0 - 1, js), min(y1 + 1, je))) m |= SB_ETA;
        if (in(max(x0 - 1, is), min(x1 + 1, ie), max(y0 - 1, js), min(y1, je - 1))) m |= SB_V1;
        if (in(max(x0 - 1, is), min(x1, ie - 1), max(y0, js), min(y1, je))) m |= SB_U2;
        if (in(max(x0 - 1, is), min(x1, ie - 1), max(y0 - 1, js), min(y1 + 1, je))) m |= SB_U1;
        if (in(max(x0, is), min(x1, ie), max(y0 - 1, js), min(y1, je - 1))) m |= SB_V2;
        if (in(x0, x1, y0, y1)) m |= SB_OWN;
        if (in(is, ie, js, je)) m |= SB_E;
        if (in(is, ie - 1, js, je)) m |= SB_NU;
        if (in(is, ie, js, je - 1)) m |= SB_NV;
        if (in(iu0, iu1, js, je)) m |= SB_AU;
        if (in(is, ie, jv0, jv1)) m |= SB_AV;
        if (i - 1 >= iu0 && i - 1 <= iu1 && j >= js && j <= je) m |= SB_UL;
        if (j - 1 >= jv0 && j - 1 <= jv1 && i >= is && i <= ie) m |= SB_VL;
        mk[r] = m;
    }

    double avu[4], avv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) avu[r] = avv[r] = 0.0;

    // init (:199-207): both buffers hold the whole input state
    for (int p = gtid; p < npts; p += gsz) {
        double e = eta_in[p], ub = ubt_in[p], vb = vbt_in[p];
        W.eta[p] = e; W.ubt[p] = ub; W.vbt[p] = vb;
        W.eta_pred[p] = e; W.ubt_prev[p] = ub; W.vbt_prev[p] = vb;
        if (TAVG) { W.uhbt[p] = 0.0; W.vhbt[p] = 0.0; }
    }
    if (tid == 0) W.tile_flag[blockIdx.x] = 0u;
    if (!grid_barrier(W, nblocks + (unsigned)P.stall_test, P.spin_budget)) return;

    int nbr[8];
    int nnb = 0;
    for (int dyt = -1; dyt <= 1; ++dyt)
        for (int dxt = -1; dxt <= 1; ++dxt) {
            const int ax = tx + dxt, ay = ty + dyt;
            if ((dxt || dyt) && ax >= 0 && ax < T.nbx && ay >= 0 && ay < T.nby)
                nbr[nnb++] = ay * T.nbx + ax;
        }

    for (int n = 1; n <= P.nstep; ++n) {
        const bool v_first = ((n + P.first_direction) % 2) == 1;
        const double* ce = (n & 1) ? W.eta : W.eta_pred;
        const double* cu = (n & 1) ? W.ubt : W.ubt_prev;
        const double* cv = (n & 1) ? W.vbt : W.vbt_prev;
        double* ne = (n & 1) ? W.eta_pred : W.eta;
        double* nu = (n & 1) ? W.ubt_prev : W.ubt;
        double* nv = (n & 1) ? W.vbt_prev : W.vbt;
        // S1: previous state on the window (as in k_btstep_tiled)
        if (n > 1 && !wait_neighbours(W, nbr, nnb, (unsigned int)(n - 1), P.spin_budget)) return;
        if (n == 1) {
            for (int jl = tyl; jl < LH; jl += TY)
            for (int il = txl; il < LW; il += 32) {
                const int q = jl * LW + il, i = lx0 + il, j = ly0 + jl;
                double e = 0.0, ub = 0.0, vb = 0.0;
                if (i >= 1 && i <= D.n1 && j >= 1 && j <= D.n2) {
                    int p = (j - 1) * D.n1 + (i - 1);
                    e = __ldcg(ce + p); ub = __ldcg(cu + p); vb = __ldcg(cv + p);
                }
                Se[q] = e; Su[q] = ub; Sv[q] = vb; Sun[q] = ub; Svn[q] = vb;
            }
        } else {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (!(mk[r] & SB_OWN)) continue;
                const int q = SQ(r);
                Se[q] = Sp[q]; Su[q] = Sun[q]; Sv[q] = Svn[q];
            }
            const int nb = y0 - ly0, na = (ly0 + LH - 1) - y1;
            const int nl = x0 - lx0, nr = (lx0 + LW - 1) - x1;
            const int mid = y1 - y0 + 1, side = nl + nr;
            const int nring = (nb + na) * LW + mid * side;
            for (int t = tid; t < nring; t += NT) {
                int i, j;
                if (t < nb * LW) {
                    j = ly0 + t / LW; i = lx0 + t % LW;
                } else if (t < (nb + na) * LW) {
                    const int t2 = t - nb * LW;
                    j = y1 + 1 + t2 / LW; i = lx0 + t2 % LW;
                } else {
                    const int t3 = t - (nb + na) * LW;
                    const int c = t3 % side;
                    j = y0 + t3 / side;
                    i = c < nl ? lx0 + c : x1 + 1 + (c - nl);
                }
                const int q = (j - ly0) * LW + (i - lx0);
                double e = 0.0, ub = 0.0, vb = 0.0;
                if (i >= 1 && i <= D.n1 && j >= 1 && j <= D.n2) {
                    int p = (j - 1) * D.n1 + (i - 1);
                    e = __ldcg(ce + p); ub = __ldcg(cu + p); vb = __ldcg(cv + p);
                }
                Se[q] = e; Su[q] = ub; Sv[q] = vb; Sun[q] = ub; Svn[q] = vb;
            }
        }
        __syncthreads();
        // S2: eta_pred
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (!(mk[r] & SB_ETA)) continue;
            const int i = SI(r), j = SJ(r), q = SQ(r);
            Sp[q] = Se[q] + (P.dtbt * GM(IareaT, i, j)) *
                                (((GM(Datu, i - 1, j) * Su[q - 1]) - (GM(Datu, i, j) * Su[q])) +
                                 ((GM(Datv, i, j - 1) * Sv[q - LW]) - (GM(Datv, i, j) * Sv[q])));
        }
        auto upd_u = [&](int r, const double* V) {
            const int i = SI(r), j = SJ(r), q = SQ(r);
            double PFu = ((Sp[q] * GM(gtot_E, i, j)) - (Sp[q + 1] * GM(gtot_W, i + 1, j))) *
                         P.dgeo_de * GM(IdxCu, i, j);
            double Cor_u = (((F4U(4, i, j) * V[q + 1]) + (F4U(1, i, j) * V[q - LW])) +
                            ((F4U(3, i, j) * V[q]) + (F4U(2, i, j) * V[q + 1 - LW])));
            Sun[q] = GM(bt_rem_u, i, j) * (Su[q] + P.dtbt * (Cor_u + PFu));
        };
        auto upd_v = [&](int r, const double* Uv) {
            const int i = SI(r), j = SJ(r), q = SQ(r);
            double PFv = ((Sp[q] * GM(gtot_N, i, j)) - (Sp[q + LW] * GM(gtot_S, i, j + 1))) *
                         P.dgeo_de * GM(IdyCv, i, j);
            double Cor_v = -1.0 * (((F4V(1, i, j) * Uv[q - 1]) + (F4V(4, i, j) * Uv[q + LW])) +
                                   ((F4V(2, i, j) * Uv[q]) + (F4V(3, i, j) * Uv[q - 1 + LW])));
            Svn[q] = GM(bt_rem_v, i, j) * (Sv[q] + P.dtbt * (Cor_v + PFv));
        };
        // S3 / S4: the two velocity updates
        if (v_first) {
            __syncthreads();   // eta_pred of the row above
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (mk[r] & SB_V1) upd_v(r, Su);
            __syncthreads();
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (mk[r] & SB_U2) upd_u(r, Svn);
        } else {
            __syncwarp();      // eta_pred of x + 1: same warp
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (mk[r] & SB_U1) upd_u(r, Sv);
            __syncthreads();
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (mk[r] & SB_V2) upd_v(r, Sun);
        }
        __syncthreads();
        // S5: transports, eta update and averages on the owned points
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const unsigned m = mk[r];
            if (!(m & SB_OWN)) continue;
            const int i = SI(r), j = SJ(r), q = SQ(r);
            const int p = (j - 1) * D.n1 + (i - 1);
            const double uh0 = (m & SB_AU)
                ? GM(Datu, i, j) * (P.trans_wt1 * Sun[q] + P.trans_wt2 * Su[q]) : 0.0;
            const double vh0 = (m & SB_AV)
                ? GM(Datv, i, j) * (P.trans_wt1 * Svn[q] + P.trans_wt2 * Sv[q]) : 0.0;
            double e = Se[q];
            if (m & SB_E) {
                const double uh1 = (m & SB_UL)
                    ? GM(Datu, i - 1, j) * (P.trans_wt1 * Sun[q - 1] + P.trans_wt2 * Su[q - 1])
                    : 0.0;
                const double vh1 = (m & SB_VL)
                    ? GM(Datv, i, j - 1) * (P.trans_wt1 * Svn[q - LW] + P.trans_wt2 * Sv[q - LW])
                    : 0.0;
                e = Se[q] - P.dtbt * GM(IareaT, i, j) * ((uh0 - uh1) + (vh0 - vh1));
                ne[p] = e;
            }
            Sp[q] = e;
            if (m & SB_NU) nu[p] = Sun[q];
            if (m & SB_NV) nv[p] = Svn[q];
            if (m & SB_AU) avu[r] = avu[r] + Sun[q] * P.inv_nstep;
            if (m & SB_AV) avv[r] = avv[r] + Svn[q] * P.inv_nstep;
            if (TAVG) {
                if (m & SB_AU) W.uhbt[p] = W.uhbt[p] + uh0 * P.inv_nstep;
                if (m & SB_AV) W.vhbt[p] = W.vhbt[p] + vh0 * P.inv_nstep;
            }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicExch(W.tile_flag + blockIdx.x, (unsigned int)n);
        }
    }
    if (!grid_barrier(W, nblocks, P.spin_budget)) return;
    const double* fe = (P.nstep & 1) ? W.eta_pred : W.eta;
    for (int p = gtid; p < npts; p += gsz) {
        eta_av[p] = fe[p];
        int i = p % D.n1 + 1, j = p / D.n1 + 1;
        if (i < is - 1 || i > ie || j < js - 1 || j > je) {
            u_av[p] = 0.0;
            v_av[p] = 0.0;
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        if (!(mk[r] & SB_OWN)) continue;
        const int i = SI(r), j = SJ(r);
        const int p = (j - 1) * D.n1 + (i - 1);
        u_av[p] = avu[r];
        v_av[p] = avv[r];
    }
#undef GM
#undef F4U
#undef F4V
#undef SI
#undef SJ
#undef SQ
}

// ---------------------------------------------------------------------------
// Ensemble variant: the barotropic loops of many domains in one cooperative
// launch.
// ---------------------------------------------------------------------------
// Every domain is split into tiles as above (EnsBtGeo, at most 64 x 64
// points); the tiles of all domains form one list and CTA c processes tiles
// c, c + gridDim.x, ... in that order at every substep.  A tile waits only for
// the tiles of its own domain that border it (flag >= n - 1), so the domains
// advance independently; a CTA that owns several tiles keeps nothing on chip
// between substeps: the owned points are re-read from the published buffers
// and the time averages accumulate in the domain's ubt_av / vbt_av work arrays.
// Waiting on substep n - 1 only cannot deadlock: the CTA at the lowest
// (substep, tile position) always finds every tile done with the previous
// substep.  The evaluation order of every point is the serial one.
// Largest d with tstart[d] <= t (the domain of global tile t).
__device__ __forceinline__ int ens_tile_domain(const int* __restrict__ tstart, int n, int t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(tstart + mid) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <int NT, bool UNI>
__global__ void __launch_bounds__(NT, 1)
k_btstep_ens(const EnsDomain* __restrict__ doms, const EnsBtGeo* __restrict__ geo,
             const int* __restrict__ tstart, int ndom, int ntiles, int max_tw, int max_th,
             int call, int max_nstep, BTWork C)
{
    extern __shared__ double smem[];
    __shared__ __align__(16) EnsDomain E;
    const unsigned int nblocks = gridDim.x;
    const int tid = (int)threadIdx.x;
    const int txl = tid & 31, tyl = tid >> 5;
    constexpr int TY = NT / 32;
    const int gtid = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int gsz = (int)(gridDim.x * blockDim.x);
    const int LWm = max_tw + 3, LHm = max_th + 3;
    const int LNm = LWm * LHm;
    double* Se = smem;
    double* Su = Se + LNm;
    double* Sv = Su + LNm;
    double* Sp = Sv + LNm;
    double* Sun = Sp + LNm;
    double* Svn = Sun + LNm;

    // init (:199-207) of every domain: both buffers hold the input state, the
    // averages start at zero
    for (int d = 0; d < ndom; ++d) {
        const EnsDomain& Q = doms[d];
        const double* ein = call ? Q.eta_av : Q.eta;
        const double* uin = call ? Q.ubt_av : Q.ubt;
        const double* vin = call ? Q.vbt_av : Q.vbt;
        const BTWork W = Q.W;
        const int npts = Q.D.n1 * Q.D.n2;
        for (int p = gtid; p < npts; p += gsz) {
            double e = ein[p], ub = uin[p], vb = vin[p];
            W.eta[p] = e; W.ubt[p] = ub; W.vbt[p] = vb;
            W.eta_pred[p] = e; W.ubt_prev[p] = ub; W.vbt_prev[p] = vb;
            W.ubt_av[p] = 0.0; W.vbt_av[p] = 0.0;
        }
    }
    for (int t = gtid; t < ntiles; t += gsz) C.tile_flag[t] = 0u;
    if (!grid_barrier(C, nblocks, 4000000000LL)) return;

    for (int n = 1; n <= max_nstep; ++n) {
        for (int t = (int)blockIdx.x; t < ntiles; t += (int)nblocks) {
            const int d = ens_tile_domain(tstart, ndom, t);
            __syncthreads();   // the previous tile's reads of E are done
            {
                const unsigned long long* src = (const unsigned long long*)(doms + d);
                unsigned long long* dst = (unsigned long long*)&E;
                for (int w = tid; w < (int)(sizeof(EnsDomain) / 8); w += NT) dst[w] = __ldg(src + w);
            }
            __syncthreads();
            const Dims& D = E.D;
            const Metrics& M = E.M;
            const UniMetrics& U = E.U;
            const BTParams& P = E.P;
            const BTWork& W = E.W;
            if (n > P.nstep) continue;
            const EnsBtGeo G = geo[d];
            const int lt = t - G.t0;
            const int tx = lt % G.nbx, ty = lt / G.nbx;
            const int is = D.is, ie = D.ie, js = D.js, je = D.je;
            const int iu0 = P.extended ? is - 1 : is, iu1 = P.extended ? ie : ie - 1;
            const int jv0 = P.extended ? js - 1 : js, jv1 = P.extended ? je : je - 1;
            const int x0 = is - 1 + tx * G.tw, y0 = js - 1 + ty * G.th;
            const int x1 = min(x0 + G.tw - 1, ie), y1 = min(y0 + G.th - 1, je);
            const int lx0 = x0 - 2, ly0 = y0 - 2;
            const int LW = G.tw + 3, LH = G.th + 3;
#define L(a, i, j) a[((j) - ly0) * LW + ((i) - lx0)]
#define GM(f, i, j) (UNI ? U.f : MOM6B_A2(M.f, i, j, D))
#define F4U(c, i, j) (UNI ? U.f4u_row[((j) - 1) * 4 + (c) - 1] : MOM6B_F4(M.f_4_u, c, i, j, D))
#define F4V(c, i, j) (UNI ? U.f4v_row[((j) - 1) * 4 + (c) - 1] : MOM6B_F4(M.f_4_v, c, i, j, D))
            const bool v_first = ((n + P.first_direction) % 2) == 1;
            const double* ce = (n & 1) ? W.eta : W.eta_pred;
            const double* cu = (n & 1) ? W.ubt : W.ubt_prev;
            const double* cv = (n & 1) ? W.vbt : W.vbt_prev;
            double* ne = (n & 1) ? W.eta_pred : W.eta;
            double* nu = (n & 1) ? W.ubt_prev : W.ubt;
            double* nv = (n & 1) ? W.vbt_prev : W.vbt;
            // neighbours of this tile in its own domain
            int nbr[8];
            int nnb = 0;
            for (int dyt = -1; dyt <= 1; ++dyt)
                for (int dxt = -1; dxt <= 1; ++dxt) {
                    const int ax = tx + dxt, ay = ty + dyt;
                    if ((dxt || dyt) && ax >= 0 && ax < G.nbx && ay >= 0 && ay < G.nby)
                        nbr[nnb++] = G.t0 + ay * G.nbx + ax;
                }
            if (n > 1 && !wait_neighbours(C, nbr, nnb, (unsigned int)(n - 1), P.spin_budget))
                return;
            // S1: the previous state on the window, owned points included
            for (int jl = tyl; jl < LH; jl += TY)
            for (int il = txl; il < LW; il += 32) {
                const int q = jl * LW + il, i = lx0 + il, j = ly0 + jl;
                double e = 0.0, ub = 0.0, vb = 0.0;
                if (i >= 1 && i <= D.n1 && j >= 1 && j <= D.n2) {
                    int p = (j - 1) * D.n1 + (i - 1);
                    e = __ldcg(ce + p); ub = __ldcg(cu + p); vb = __ldcg(cv + p);
                }
                Se[q] = e; Su[q] = ub; Sv[q] = vb; Sun[q] = ub; Svn[q] = vb;
            }
            __syncthreads();
            // S2: eta_pred on [x0-1, x1+1] x [y0-1, y1+1] within [is, ie] x [js, je]
            {
                int a0 = max(x0 - 1, is), a1 = min(x1 + 1, ie);
                int b0 = max(y0 - 1, js), b1 = min(y1 + 1, je);
                for (int j = b0 + tyl; j <= b1; j += TY)
                for (int i = a0 + txl; i <= a1; i += 32) {
                    L(Sp, i, j) = L(Se, i, j) + (P.dtbt * GM(IareaT, i, j)) *
                                                    (((GM(Datu, i - 1, j) * L(Su, i - 1, j)) -
                                                      (GM(Datu, i, j) * L(Su, i, j))) +
                                                     ((GM(Datv, i, j - 1) * L(Sv, i, j - 1)) -
                                                      (GM(Datv, i, j) * L(Sv, i, j))));
                }
            }
            __syncthreads();
            auto upd_u = [&](int i, int j, const double* Vsrc) {
                double PFu = ((L(Sp, i, j) * GM(gtot_E, i, j)) -
                              (L(Sp, i + 1, j) * GM(gtot_W, i + 1, j))) *
                             P.dgeo_de * GM(IdxCu, i, j);
                double Cor_u = (((F4U(4, i, j) * L(Vsrc, i + 1, j)) +
                                 (F4U(1, i, j) * L(Vsrc, i, j - 1))) +
                                ((F4U(3, i, j) * L(Vsrc, i, j)) +
                                 (F4U(2, i, j) * L(Vsrc, i + 1, j - 1))));
                L(Sun, i, j) = GM(bt_rem_u, i, j) * (L(Su, i, j) + P.dtbt * (Cor_u + PFu));
            };
            auto upd_v = [&](int i, int j, const double* Usrc) {
                double PFv = ((L(Sp, i, j) * GM(gtot_N, i, j)) -
                              (L(Sp, i, j + 1) * GM(gtot_S, i, j + 1))) *
                             P.dgeo_de * GM(IdyCv, i, j);
                double Cor_v = -1.0 * (((F4V(1, i, j) * L(Usrc, i - 1, j)) +
                                        (F4V(4, i, j) * L(Usrc, i, j + 1))) +
                                       ((F4V(2, i, j) * L(Usrc, i, j)) +
                                        (F4V(3, i, j) * L(Usrc, i - 1, j + 1))));
                L(Svn, i, j) = GM(bt_rem_v, i, j) * (L(Sv, i, j) + P.dtbt * (Cor_v + PFv));
            };
            // S3 / S4: the two velocity updates on the regions the tile needs
            if (v_first) {
                int a0 = max(x0 - 1, is), a1 = min(x1 + 1, ie);
                int b0 = max(y0 - 1, js), b1 = min(y1, je - 1);
                for (int j = b0 + tyl; j <= b1; j += TY)
                for (int i = a0 + txl; i <= a1; i += 32) upd_v(i, j, Su);
                __syncthreads();
                a0 = max(x0 - 1, is); a1 = min(x1, ie - 1);
                b0 = max(y0, js); b1 = min(y1, je);
                for (int j = b0 + tyl; j <= b1; j += TY)
                for (int i = a0 + txl; i <= a1; i += 32) upd_u(i, j, Svn);
            } else {
                int a0 = max(x0 - 1, is), a1 = min(x1, ie - 1);
                int b0 = max(y0 - 1, js), b1 = min(y1 + 1, je);
                for (int j = b0 + tyl; j <= b1; j += TY)
                for (int i = a0 + txl; i <= a1; i += 32) upd_u(i, j, Sv);
                __syncthreads();
                a0 = max(x0, is); a1 = min(x1, ie);
                b0 = max(y0 - 1, js); b1 = min(y1, je - 1);
                for (int j = b0 + tyl; j <= b1; j += TY)
                for (int i = a0 + txl; i <= a1; i += 32) upd_v(i, j, Sun);
            }
            __syncthreads();
            // S5: transports, eta update and averages on the owned points
            auto uhbt_at = [&](int i, int j) -> double {
                if (i < iu0 || i > iu1 || j < js || j > je) return 0.0;
                return GM(Datu, i, j) * (P.trans_wt1 * L(Sun, i, j) + P.trans_wt2 * L(Su, i, j));
            };
            auto vhbt_at = [&](int i, int j) -> double {
                if (j < jv0 || j > jv1 || i < is || i > ie) return 0.0;
                return GM(Datv, i, j) * (P.trans_wt1 * L(Svn, i, j) + P.trans_wt2 * L(Sv, i, j));
            };
#pragma unroll
            for (int r = 0; r < kBtTileR; ++r) {
                const int i = x0 + txl + 32 * (r & 1), j = y0 + tyl + TY * (r >> 1);
                if (i > x1 || j > y1) continue;
                int p = (j - 1) * D.n1 + (i - 1);
                if (i >= is && i <= ie && j >= js && j <= je)
                    ne[p] = L(Se, i, j) - P.dtbt * GM(IareaT, i, j) *
                                              ((uhbt_at(i, j) - uhbt_at(i - 1, j)) +
                                               (vhbt_at(i, j) - vhbt_at(i, j - 1)));
                if (i >= is && i <= ie - 1 && j >= js && j <= je) nu[p] = L(Sun, i, j);
                if (i >= is && i <= ie && j >= js && j <= je - 1) nv[p] = L(Svn, i, j);
                if (j >= js && j <= je && i >= iu0 && i <= iu1)
                    W.ubt_av[p] = W.ubt_av[p] + L(Sun, i, j) * P.inv_nstep;
                if (j >= jv0 && j <= jv1 && i >= is && i <= ie)
                    W.vbt_av[p] = W.vbt_av[p] + L(Svn, i, j) * P.inv_nstep;
            }
#undef L
#undef GM
#undef F4U
#undef F4V
            // publish substep n of tile t: every global write of it is done
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                atomicExch(C.tile_flag + t, (unsigned int)n);
            }
        }
    }
    if (!grid_barrier(C, nblocks, 4000000000LL)) return;
    // outputs (:296-302); they may alias the inputs.  The averages are zero
    // outside their ranges (the init of :204-205).
    for (int d = 0; d < ndom; ++d) {
        const EnsDomain& Q = doms[d];
        const BTWork W = Q.W;
        double* u_av = Q.ubt_av;
        double* v_av = Q.vbt_av;
        double* e_out = call ? Q.eta : Q.eta_av;
        const double* fe = (Q.P.nstep & 1) ? W.eta_pred : W.eta;
        const int npts = Q.D.n1 * Q.D.n2;
        for (int p = gtid; p < npts; p += gsz) {
            e_out[p] = fe[p];
            u_av[p] = W.ubt_av[p];
            v_av[p] = W.vbt_av[p];
        }
    }
}

// SM count of each device, looked up the first time a barotropic kernel is
// launched with that device current (one persistent CTA per SM).
static int g_bt_sms[64];

static cudaError_t bt_blocks(int* out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (g_bt_sms[dev] == 0) {
        int nsm = 0;
        e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        g_bt_sms[dev] = nsm;
    }
    *out = g_bt_sms[dev];
    return cudaSuccess;
}

// Tiles of the tiled kernel: nbx x nby tiles (at most one per SM) of at most
// 64 x 64 points covering the updated box [is-1, ie] x [js-1, je]; false when
// the box needs more (either side above 64 tiles' worth for the SM count).
static bool tiles_for(const Dims& D, int nsm, BTTiles& T)
{
    const int bw = D.ie - D.is + 2, bh = D.je - D.js + 2;
    T.nt = 1024;
    // the fewest tiles of at most 64 points per side, then as many as the SMs
    // allow while a tile keeps at least 8 points per side
    int nbx = (bw + 63) / 64, nby = (bh + 63) / 64;
    if ((long long)nbx * nby > nsm) return false;
    while ((long long)(nbx + 1) * (nby + 1) <= nsm && (bw + nbx) / (nbx + 1) >= 8 &&
           (bh + nby) / (nby + 1) >= 8) { ++nbx; ++nby; }
    while ((long long)(nbx + 1) * nby <= nsm && (bw + nbx) / (nbx + 1) >= 8) ++nbx;
    while ((long long)nbx * (nby + 1) <= nsm && (bh + nby) / (nby + 1) >= 8) ++nby;
    T.nbx = nbx; T.nby = nby;
    T.tw = (bw + nbx - 1) / nbx; T.th = (bh + nby - 1) / nby;
    const size_t smem = (size_t)6 * (T.tw + 3) * (T.th + 3) * sizeof(double);
    // each of the 32 x 32 threads owns the points (txl + 32a, tyl + 32b), a, b in {0, 1}
    return T.tw <= 64 && T.th <= 64 && smem <= 227 * 1024 && nbx * nby <= kBtMaxTiles;
}


static cudaError_t launch_btstep_tiled(const Dims& D, const Metrics& M, const UniMetrics& U,
                                       const BTWork& W, const BTParams& P, const BTTiles& T,
                                       const double* eta_in, const double* ubt_in,
                                       const double* vbt_in, double* u_av, double* v_av,
                                       double* eta_av, cudaStream_t s, bool tavg = false)
{
    const int NT = T.nt;
    size_t smem = (size_t)6 * (T.tw + 3) * (T.th + 3) * sizeof(double);
    // the slot kernel (four fixed points per thread) up to 62 x 62 tiles,
    // the general tiled kernel for 63 and 64
    const void* fn;
    if (T.tw <= 62 && T.th <= 62)
        fn = tavg ? (U.valid_bt ? (const void*)k_btstep_slots<true, true>
                                : (const void*)k_btstep_slots<false, true>)
                  : (U.valid_bt ? (const void*)k_btstep_slots<true, false>
                                : (const void*)k_btstep_slots<false, false>);
    else
        fn = tavg ? (U.valid_bt ? (const void*)k_btstep_tiled<1024, true, true>
                                : (const void*)k_btstep_tiled<1024, false, true>)
                  : (U.valid_bt ? (const void*)k_btstep_tiled<1024, true, false>
                                : (const void*)k_btstep_tiled<1024, false, false>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    Dims Dc = D; Metrics Mc = M; UniMetrics Uc = U; BTWork Wc = W; BTParams Pc = P;
    BTTiles Tc = T;
    void* args[] = {&Dc, &Mc, &Uc, &Wc, &Pc, &Tc, (void*)&eta_in, (void*)&ubt_in,
                    (void*)&vbt_in, (void*)&u_av, (void*)&v_av, (void*)&eta_av};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(T.nbx * T.nby, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

cudaError_t launch_btstep(const Dims& D, const Metrics& M, const UniMetrics& U,
                          const BTWork& W, const BTParams& P, const double* eta_in,
                          const double* ubt_in, const double* vbt_in,
                          double* u_av, double* v_av, double* eta_av,
                          cudaStream_t s)
{
    const size_t smem_fast = (size_t)PV_N * kBtMaxR * kBtThreads * sizeof(double);
    int nsm = 0;
    cudaError_t e0 = bt_blocks(&nsm);
    if (e0 != cudaSuccess) return e0;
    // tiled variant: the updated box split into at most one tile per SM
    BTTiles T;
    const bool cut = D.cw || D.ce || D.cs || D.cn;
    if (cut && P.substep == 0) return cudaErrorInvalidValue;   // one launch per substep
    if (!P.untiled && !cut && P.substep == 0 && tiles_for(D, nsm, T))
        return launch_btstep_tiled(D, M, U, W, P, T, eta_in, ubt_in, vbt_in, u_av, v_av,
                                   eta_av, s);
    {
        cudaError_t e = cudaFuncSetAttribute(k_btstep<true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem_fast);
        if (e != cudaSuccess) return e;
    }
    const long long nbox = (long long)(D.ie - D.is + 3 + 2 * (D.cw + D.ce)) *
                           (D.je - D.js + 3 + 2 * (D.cs + D.cn));
    int blocks = nsm;
    int need = (int)((nbox + kBtThreads - 1) / kBtThreads);
    if (blocks > need) blocks = need;
    // the shared-memory privates last one launch: a loop split over launches
    // keeps them in the global work arrays
    const bool fast = P.substep == 0 && (long long)blocks * kBtThreads * kBtMaxR >= nbox;
    Dims Dc = D; Metrics Mc = M; BTWork Wc = W; BTParams Pc = P;
    void* args[] = {&Dc, &Mc, &Wc, &Pc, (void*)&eta_in, (void*)&ubt_in, (void*)&vbt_in,
                    (void*)&u_av, (void*)&v_av, (void*)&eta_av};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks, 1, 1);
    cfg.blockDim = dim3(kBtThreads, 1, 1);
    cfg.dynamicSmemBytes = fast ? smem_fast : 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fast ? (const void*)k_btstep<true>
                                          : (const void*)k_btstep<false>, args);
}

EnsBtGeo ens_bt_geometry(const Dims& D, int max_edge)
{
    EnsBtGeo G;
    const int bw = D.ie - D.is + 2, bh = D.je - D.js + 2;
    G.nbx = (bw + max_edge - 1) / max_edge;
    G.nby = (bh + max_edge - 1) / max_edge;
    G.tw = (bw + G.nbx - 1) / G.nbx;
    G.th = (bh + G.nby - 1) / G.nby;
    G.t0 = 0;
    return G;
}

cudaError_t launch_ens_btstep(const EnsDomain* doms, const EnsBtGeo* geo, const int* tstart,
                              int n, int ntiles, int max_tw, int max_th, int call,
                              int max_nstep, const BTWork& ctl, bool uni, cudaStream_t s)
{
    if (ntiles <= 0) return cudaSuccess;
    if (max_tw > 64 || max_th > 64) return cudaErrorInvalidValue;
    int nsm = 0;
    cudaError_t e0 = bt_blocks(&nsm);
    if (e0 != cudaSuccess) return e0;
    const int NT = 1024;
    const size_t smem = (size_t)6 * (max_tw + 3) * (max_th + 3) * sizeof(double);
    const void* fn = uni ? (const void*)k_btstep_ens<NT, true> : (const void*)k_btstep_ens<NT, false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, NT, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int blocks = per_sm * nsm;
    if (blocks > ntiles) blocks = ntiles;
    BTWork C = ctl;
    void* args[] = {(void*)&doms, (void*)&geo, (void*)&tstart, (void*)&n, (void*)&ntiles,
                    (void*)&max_tw, (void*)&max_th, (void*)&call, (void*)&max_nstep, (void*)&C};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks, 1, 1);
    cfg.blockDim = dim3(NT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, fn, args);
}

cudaError_t launch_btstep_tavg(const Dims& D, const Metrics& M, const UniMetrics& U,
                               const BTWork& W, const BTParams& P, const double* eta_in,
                               const double* ubt_in, const double* vbt_in, double* u_av,
                               double* v_av, double* eta_av, cudaStream_t s)
{
    int nsm = 0;
    cudaError_t e0 = bt_blocks(&nsm);
    if (e0 != cudaSuccess) return e0;
    BTTiles T;
    if (!tiles_for(D, nsm, T)) return cudaErrorNotSupported;
    return launch_btstep_tiled(D, M, U, W, P, T, eta_in, ubt_in, vbt_in, u_av, v_av, eta_av, s,
                               true);
}

// ---------------------------------------------------------------------------
// Allocation-free barotropic entry point
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory at the point where they need
// the barotropic loop: a Fortran host whose device arrays are owned by an
// OpenMP-target or OpenACC runtime (map clauses; cudaMalloc from inside its
// data regions would fragment or bypass that runtime's pool).
// mom6b_btstep_noalloc therefore keeps every work array of the loop in the
// file-scope array below, sized for grids of at most kNoAllocMaxPoints
// points (n1 * n2), i.e. 6 x 589,824 doubles plus a 2.3 KB header, about
// 28.3 MB per GPU that loads this library, held until the process exits.
constexpr long long kNoAllocMaxPoints = 768LL * 768LL;
constexpr long long kNoAllocHeader = 288;  // doubles: barrier words, status, tile flags
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocHeader +
                                                          6 * kNoAllocMaxPoints];

// Device address of g_noalloc_scratch, looked up once per device with that
// device current.  In host code the symbol is only a host-side stand-in;
// kernels must be given the address returned by cudaGetSymbolAddress.
static double* g_noalloc_ptr[64];
// Wait limit of the loop's barriers (0: kBtDefaultWait) and the stall test
// aid (BTParams::stall_test), set by mom6b_btstep_noalloc_set_wait.
static long long g_noalloc_wait = 0;
static int g_noalloc_stall = 0;

static cudaError_t noalloc_scratch(double** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!g_noalloc_ptr[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// halo / boundary fill (halo_impl.cuh): one thread per halo point
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_halo_fill(Dims D, T* f, int nz, int kind)
{
    halo_fill_point<T>(D, f, nz, kind, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

template <typename T>
static cudaError_t launch_halo_fill_t(const Dims& D, T* f, int nz, int kind, cudaStream_t s)
{
    const int lo_x = (kind == 1) ? D.is - 2 : D.is - 1;
    const int lo_y = (kind == 2) ? D.js - 2 : D.js - 1;
    const int nxh = lo_x + (D.n1 - D.ie), nyh = lo_y + (D.n2 - D.je);
    long long per_layer = (long long)nyh * D.n1 + (long long)nxh * (D.n2 - nyh);
    long long total = per_layer * nz;
    int nb = 256;
    long long blocks = (total + nb - 1) / nb;
    k_halo_fill<T><<<(unsigned)blocks, nb, 0, s>>>(D, f, nz, kind);
    return cudaGetLastError();
}

// The fills of an h-point, a u-point and a v-point field (kinds 0, 1, 2) in one
// launch: grid row y fills the field of kind y.  The three fields are
// distinct arrays and each fill reads only its own field, so the result is
// that of the three separate fills.
template <typename T>
__global__ void k_halo_fill3(Dims D, T* fh, T* fu, T* fv, int nz)
{
    const int kind = (int)blockIdx.y;
    T* f = kind == 0 ? fh : (kind == 1 ? fu : fv);
    halo_fill_point<T>(D, f, nz, kind, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

template <typename T>
static cudaError_t launch_halo_fill3_t(const Dims& D, T* fh, T* fu, T* fv, int nz,
                                       cudaStream_t s)
{
    long long most = 0;
    for (int kind = 0; kind < 3; ++kind) {
        const long long t = halo_points_per_layer(D, kind) * nz;
        if (t > most) most = t;
    }
    const int nb = 256;
    const long long blocks = (most + nb - 1) / nb;
    k_halo_fill3<T><<<dim3((unsigned)blocks, 3, 1), nb, 0, s>>>(D, fh, fu, fv, nz);
    return cudaGetLastError();
}

cudaError_t launch_halo_fill3(const Dims& D, double* fh, double* fu, double* fv, int nz,
                              cudaStream_t s)
{
    return launch_halo_fill3_t<double>(D, fh, fu, fv, nz, s);
}

cudaError_t launch_halo_fill3_f(const Dims& D, float* fh, float* fu, float* fv, int nz,
                                cudaStream_t s)
{
    return launch_halo_fill3_t<float>(D, fh, fu, fv, nz, s);
}

cudaError_t launch_halo_fill(const Dims& D, double* f, int nz, int kind, cudaStream_t s)
{
    return launch_halo_fill_t<double>(D, f, nz, kind, s);
}

cudaError_t launch_halo_fill_f(const Dims& D, float* f, int nz, int kind, cudaStream_t s)
{
    return launch_halo_fill_t<float>(D, f, nz, kind, s);
}

// The barotropic loop on the static scratch (no allocation) with the
// caller's metric arrays and parameters: the allocation-free entry point and
// the deferred barotropic calls of the reference ABI.  P's wait limit and
// stall aid come from mom6b_btstep_noalloc_set_wait.  MOM6B_NOALLOC_* codes.
int btstep_static(const double* eta_in, const double* ubt_in, const double* vbt_in,
                  double* u_av, double* v_av, double* eta_av, const Metrics& M, const Dims& D,
                  BTParams P, cudaStream_t s)
{
    if ((long long)D.n1 * (long long)D.n2 > kNoAllocMaxPoints)
        return MOM6B_NOALLOC_ERR_TOO_LARGE;
    int nsm = 0;
    if (bt_blocks(&nsm) != cudaSuccess) return MOM6B_NOALLOC_ERR_CUDA;
    BTTiles T;
    if (!tiles_for(D, nsm, T)) return MOM6B_NOALLOC_ERR_TOO_LARGE;
    double* base = nullptr;
    if (noalloc_scratch(&base) != cudaSuccess) return MOM6B_NOALLOC_ERR_CUDA;
    // barrier words and status must start at zero; the field buffers are
    // fully written by the kernel's initial copy
    if (cudaMemsetAsync(base, 0, kNoAllocHeader * sizeof(double), s) != cudaSuccess)
        return MOM6B_NOALLOC_ERR_CUDA;
    const size_t np = (size_t)D.n1 * (size_t)D.n2;
    double* f = base + kNoAllocHeader;
    BTWork W{};
    W.eta = f; W.ubt = f + np; W.vbt = f + 2 * np;
    W.eta_pred = f + 3 * np; W.ubt_prev = f + 4 * np; W.vbt_prev = f + 5 * np;
    W.uhbt = nullptr; W.vhbt = nullptr; W.PFu = nullptr; W.PFv = nullptr;
    W.ubt_av = nullptr; W.vbt_av = nullptr;
    W.bar_count = (unsigned int*)base;
    W.bar_gen = (unsigned int*)base + 4;
    W.status = (int*)base + 8;
    W.tile_flag = (unsigned int*)base + 16;   // kBtMaxTiles words, inside the header
    static_assert(64 + kBtMaxTiles * 4 <= kNoAllocHeader * 8, "noalloc header too small");
    P.spin_budget = g_noalloc_wait > 0 ? g_noalloc_wait : kBtDefaultWait;
    P.stall_test = g_noalloc_stall;
    UniMetrics U{};
    if (launch_btstep_tiled(D, M, U, W, P, T, eta_in, ubt_in, vbt_in, u_av, v_av, eta_av, s) !=
        cudaSuccess)
        return MOM6B_NOALLOC_ERR_CUDA;
    return MOM6B_NOALLOC_OK;
}

} // namespace mom6b

// See mom6b.h.  Every call shares g_noalloc_scratch: calls that overlap on
// the GPU (two streams, or two host threads) race on it.  The first call on a
// device looks up the array's device address; make that first call before
// any stream capture begins.
extern "C" int mom6b_btstep_noalloc(
    const double* eta_in, const double* ubt_in, const double* vbt_in, double* u_av,
    double* v_av, double* eta_av, const double* Datu, const double* Datv,
    const double* gtot_E, const double* gtot_W, const double* gtot_N,
    const double* gtot_S, const double* f_4_u, const double* f_4_v,
    const double* bt_rem_u, const double* bt_rem_v, const double* IareaT,
    const double* IdxCu, const double* IdyCv, int n1, int n2, int is, int ie, int js,
    int je, int nstep, double dtbt, double bebt, double dgeo_de, int first_direction,
    int extended_ranges, void* stream)
{
    using namespace mom6b;
    if (!eta_in || !ubt_in || !vbt_in || !u_av || !v_av || !eta_av || !Datu || !Datv ||
        !gtot_E || !gtot_W || !gtot_N || !gtot_S || !f_4_u || !f_4_v || !bt_rem_u ||
        !bt_rem_v || !IareaT || !IdxCu || !IdyCv)
        return MOM6B_NOALLOC_ERR_ARG;
    if (n1 < 4 || n2 < 4 || nstep < 1 || is < 2 || js < 2 || ie > n1 - 1 || je > n2 - 1 ||
        ie - is < 2 || je - js < 2)
        return MOM6B_NOALLOC_ERR_ARG;
    Dims D{};
    D.n1 = n1; D.n2 = n2; D.nk = 1;
    D.is = is; D.ie = ie; D.js = js; D.je = je;
    D.isd = 1; D.ied = n1; D.jsd = 1; D.jed = n2;
    D.plane = (long long)n1 * (long long)n2;
    Metrics M{};
    M.Datu = Datu; M.Datv = Datv; M.gtot_E = gtot_E; M.gtot_W = gtot_W;
    M.gtot_N = gtot_N; M.gtot_S = gtot_S; M.f_4_u = f_4_u; M.f_4_v = f_4_v;
    M.bt_rem_u = bt_rem_u; M.bt_rem_v = bt_rem_v; M.IareaT = IareaT;
    M.IdxCu = IdxCu; M.IdyCv = IdyCv;
    BTParams P{};
    P.dtbt = dtbt; P.dgeo_de = dgeo_de;
    P.trans_wt1 = 1.0 + bebt; P.trans_wt2 = -bebt;
    P.inv_nstep = 1.0 / (double)nstep;
    P.nstep = nstep; P.first_direction = first_direction;
    P.extended = extended_ranges ? 1 : 0;
    return btstep_static(eta_in, ubt_in, vbt_in, u_av, v_av, eta_av, M, D, P,
                         (cudaStream_t)stream);
}

extern "C" int mom6b_btstep_noalloc_status(void* stream)
{
    using namespace mom6b;
    double* base = nullptr;
    if (noalloc_scratch(&base) != cudaSuccess) return MOM6B_NOALLOC_ERR_CUDA;
    if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) return MOM6B_NOALLOC_ERR_CUDA;
    int* status = (int*)base + 8;
    int st = 0;
    if (cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return MOM6B_NOALLOC_ERR_CUDA;
    if (st == kDevOk) return MOM6B_NOALLOC_OK;
    // clear the word and the barrier count the timed-out blocks left behind
    if (cudaMemset(base, 0, 16 * sizeof(double)) != cudaSuccess) return MOM6B_NOALLOC_ERR_CUDA;
    return MOM6B_NOALLOC_ERR_TIMEOUT;
}

extern "C" int mom6b_btstep_noalloc_set_wait(long long cycles, int stall_test)
{
    if (cycles < 0) return MOM6B_NOALLOC_ERR_ARG;
    mom6b::g_noalloc_wait = cycles;
    mom6b::g_noalloc_stall = stall_test ? 1 : 0;
    return MOM6B_NOALLOC_OK;
}
