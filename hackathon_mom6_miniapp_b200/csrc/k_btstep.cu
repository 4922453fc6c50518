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
#include "kernels.h"

namespace mom6b {

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
            while (*gen == g) {
                if (*st != kDevOk) { ok = 0; break; }
                if (clock64() - t0 > budget) {
                    atomicExch(W.status, kDevTimeout);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = ok && (*st == kDevOk);
    }
    __syncthreads();
    return s_ok != 0;
}

__global__ void __launch_bounds__(512)
k_btstep(Dims D, Metrics M, BTWork W, BTParams P, const double* eta_in,
         const double* ubt_in, const double* vbt_in, double* u_av, double* v_av,
         double* eta_av)
{
    const unsigned int nblocks = gridDim.x;
    const int npts = D.n1 * D.n2;
    const int gtid = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int gsz = (int)(gridDim.x * blockDim.x);
    const int is = D.is, ie = D.ie, js = D.js, je = D.je;
    // serial ranges vs. extended ranges for uhbt/vhbt and the averages
    const int iu0 = P.extended ? is - 1 : is, iu1 = P.extended ? ie : ie - 1;
    const int jv0 = P.extended ? js - 1 : js, jv1 = P.extended ? je : je - 1;
#define PT_LOOP for (int p = gtid; p < npts; p += gsz)
#define PT_IJ const int i = p % D.n1 + 1, j = p / D.n1 + 1
#define A(a, ii, jj) MOM6B_A2(a, ii, jj, D)

    // init (:199-207)
    PT_LOOP {
        W.eta[p] = eta_in[p];
        W.ubt[p] = ubt_in[p];
        W.vbt[p] = vbt_in[p];
        W.ubt_av[p] = 0.0;
        W.vbt_av[p] = 0.0;
    }
    if (!grid_barrier(W, nblocks, P.spin_budget)) return;

    auto phase_A = [&]() {
        PT_LOOP {
            PT_IJ;
            if (j >= js && j <= je && i >= is - 1 && i <= ie + 1) W.ubt_prev[p] = W.ubt[p];
            if (j >= js - 1 && j <= je + 1 && i >= is && i <= ie) W.vbt_prev[p] = W.vbt[p];
            if (i >= is && i <= ie && j >= js && j <= je)
                W.eta_pred[p] =
                    W.eta[p] + (P.dtbt * A(M.IareaT, i, j)) *
                                   (((A(M.Datu, i - 1, j) * A(W.ubt, i - 1, j)) -
                                     (A(M.Datu, i, j) * W.ubt[p])) +
                                    ((A(M.Datv, i, j - 1) * A(W.vbt, i, j - 1)) -
                                     (A(M.Datv, i, j) * W.vbt[p])));
        }
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

    phase_A();
    if (!grid_barrier(W, nblocks, P.spin_budget)) return;

    for (int n = 1; n <= P.nstep; ++n) {
        const bool v_first = ((n + P.first_direction) % 2) == 1;
        // phase B: pressure force (:234-247) and the first update
        PT_LOOP {
            PT_IJ;
            if (j >= js && j <= je && i >= is && i <= ie - 1)
                W.PFu[p] = ((W.eta_pred[p] * A(M.gtot_E, i, j)) -
                            (A(W.eta_pred, i + 1, j) * A(M.gtot_W, i + 1, j))) *
                           P.dgeo_de * A(M.IdxCu, i, j);
            if (j >= js && j <= je - 1 && i >= is && i <= ie)
                W.PFv[p] = ((W.eta_pred[p] * A(M.gtot_N, i, j)) -
                            (A(W.eta_pred, i, j + 1) * A(M.gtot_S, i, j + 1))) *
                           P.dgeo_de * A(M.IdyCv, i, j);
            if (v_first) {
                if (i >= is && i <= ie && j >= js && j <= je - 1) update_v(p, i, j, W.PFv[p]);
            } else {
                if (i >= is && i <= ie - 1 && j >= js && j <= je) update_u(p, i, j, W.PFu[p]);
            }
        }
        if (!grid_barrier(W, nblocks, P.spin_budget)) return;
        // phase C: second update, transports (:263-272), averages (:282-291)
        PT_LOOP {
            PT_IJ;
            if (v_first) {
                if (i >= is && i <= ie - 1 && j >= js && j <= je) update_u(p, i, j, W.PFu[p]);
            } else {
                if (i >= is && i <= ie && j >= js && j <= je - 1) update_v(p, i, j, W.PFv[p]);
            }
            if (j >= js && j <= je && i >= iu0 && i <= iu1) {
                W.uhbt[p] = A(M.Datu, i, j) * (P.trans_wt1 * W.ubt[p] + P.trans_wt2 * W.ubt_prev[p]);
                W.ubt_av[p] = W.ubt_av[p] + W.ubt[p] * P.inv_nstep;
            }
            if (j >= jv0 && j <= jv1 && i >= is && i <= ie) {
                W.vhbt[p] = A(M.Datv, i, j) * (P.trans_wt1 * W.vbt[p] + P.trans_wt2 * W.vbt_prev[p]);
                W.vbt_av[p] = W.vbt_av[p] + W.vbt[p] * P.inv_nstep;
            }
        }
        if (!grid_barrier(W, nblocks, P.spin_budget)) return;
        // phase D: eta update (:274-279), then phase A of the next substep
        PT_LOOP {
            PT_IJ;
            if (i >= is && i <= ie && j >= js && j <= je)
                W.eta[p] = W.eta[p] - P.dtbt * A(M.IareaT, i, j) *
                                          ((W.uhbt[p] - A(W.uhbt, i - 1, j)) +
                                           (W.vhbt[p] - A(W.vhbt, i, j - 1)));
        }
        if (n < P.nstep) {
            // eta_pred(i,j) needs only this thread's new eta(i,j); the velocity
            // neighbours were final before the last barrier
            phase_A();
        }
        if (!grid_barrier(W, nblocks, P.spin_budget)) return;
    }
    // copy output (:296-302); outputs may alias the inputs
    PT_LOOP {
        u_av[p] = W.ubt_av[p];
        v_av[p] = W.vbt_av[p];
        eta_av[p] = W.eta[p];
    }
#undef PT_LOOP
#undef PT_IJ
#undef A
}

static int g_bt_blocks = 0;

cudaError_t launch_btstep(const Dims& D, const Metrics& M, const BTWork& W,
                          const BTParams& P, const double* eta_in,
                          const double* ubt_in, const double* vbt_in,
                          double* u_av, double* v_av, double* eta_av,
                          cudaStream_t s)
{
    const int nb = 512;
    if (g_bt_blocks == 0) {
        int dev = 0, nsm = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_btstep, nb, 0);
        if (per_sm < 1) return cudaErrorLaunchOutOfResources;
        g_bt_blocks = nsm * (per_sm < 2 ? per_sm : 2);
    }
    int npts = D.n1 * D.n2;
    int blocks = g_bt_blocks;
    int need = (npts + nb - 1) / nb;
    if (blocks > need) blocks = need;
    Dims Dc = D; Metrics Mc = M; BTWork Wc = W; BTParams Pc = P;
    void* args[] = {&Dc, &Mc, &Wc, &Pc, (void*)&eta_in, (void*)&ubt_in, (void*)&vbt_in,
                    (void*)&u_av, (void*)&v_av, (void*)&eta_av};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks, 1, 1);
    cfg.blockDim = dim3(nb, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelExC(&cfg, (const void*)k_btstep, args);
}

// ---------------------------------------------------------------------------
// halo / boundary fill: periodic in i, solid walls in j
// ---------------------------------------------------------------------------
// kind 0: h point, 1: u point (faces is-1 and ie are the basin walls and keep
// their values), 2: v point (antisymmetric about the wall faces js-1, je).
// Every halo value is read from non-halo points only, so one pass suffices.
__global__ void k_halo_fill(Dims D, double* f, int nz, int kind)
{
    const int is = D.is, ie = D.ie, js = D.js, je = D.je;
    const int P = ie - is + 1;
    const int lo_x = (kind == 1) ? is - 2 : is - 1;   // x halo: i <= lo_x or i > ie
    const int lo_y = (kind == 2) ? js - 2 : js - 1;   // y halo: j <= lo_y or j > je
    const int nxh = lo_x + (D.n1 - ie);               // halo columns
    const int nyh = lo_y + (D.n2 - je);               // halo rows
    // enumerate: halo rows (all i) first, then halo columns of the other rows
    const long long per_layer = (long long)nyh * D.n1 + (long long)nxh * (D.n2 - nyh);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
    double val = MOM6B_A3(f, si, sj, k, D);
    MOM6B_A3(f, i, j, k, D) = (sgn < 0.0) ? -val : val;
}

cudaError_t launch_halo_fill(const Dims& D, double* f, int nz, int kind, cudaStream_t s)
{
    const int lo_x = (kind == 1) ? D.is - 2 : D.is - 1;
    const int lo_y = (kind == 2) ? D.js - 2 : D.js - 1;
    const int nxh = lo_x + (D.n1 - D.ie), nyh = lo_y + (D.n2 - D.je);
    long long per_layer = (long long)nyh * D.n1 + (long long)nxh * (D.n2 - nyh);
    long long total = per_layer * nz;
    int nb = 256;
    long long blocks = (total + nb - 1) / nb;
    k_halo_fill<<<(unsigned)blocks, nb, 0, s>>>(D, f, nz, kind);
    return cudaGetLastError();
}

} // namespace mom6b
