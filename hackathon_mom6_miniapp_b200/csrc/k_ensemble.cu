// k_ensemble.cu -- batched kernels of the ensemble: many independent domains
// of uneven size advanced in the mixed form, one launch per phase for all of
// them.
//
// Every batched kernel runs the same per-CTA device code as the single-domain
// mixed form (tendency_impl.cuh, vertvisc_impl.cuh, mixed_impl.cuh,
// halo_impl.cuh) and is built with the same FMA contraction, so a domain of an
// ensemble gets exactly the arithmetic it gets alone.  The grid is the
// concatenation of the domains' own grids: start[d] is domain d's first block
// (start[n] = total), a CTA finds its domain by binary search over start,
// copies that domain's descriptor (EnsDomain) to shared memory and derives
// its block coordinates inside the domain's grid from its offset.
#include "halo_impl.cuh"
#include "mixed_impl.cuh"
#include "tendency_impl.cuh"
#include "vertvisc_impl.cuh"

namespace mom6b {

static_assert(sizeof(EnsDomain) % 8 == 0, "EnsDomain is copied as 8-byte words");

// Largest d with start[d] <= b (start is non-decreasing, start[0] = 0).
__device__ __forceinline__ int ens_find(const int* __restrict__ start, int n, int b)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(start + mid) <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Copy doms[d] to shared memory with the whole CTA; ends with a barrier.
__device__ __forceinline__ void ens_load(EnsDomain& dst, const EnsDomain* __restrict__ doms,
                                         int d)
{
    const unsigned long long* src = (const unsigned long long*)(doms + d);
    unsigned long long* out = (unsigned long long*)&dst;
    const int nthreads = (int)(blockDim.x * blockDim.y);
    const int tid = (int)(threadIdx.y * blockDim.x + threadIdx.x);
    for (int w = tid; w < (int)(sizeof(EnsDomain) / 8); w += nthreads) out[w] = __ldg(src + w);
    __syncthreads();
}

// ---- host-side block counts ------------------------------------------------
static inline long long cdiv(long long a, long long b) { return (a + b - 1) / b; }

long long ens_blocks_tendency(const Dims& D, const EnsTuning& T)
{
    const int TX = kEnsTendTiles[T.tend][0], TY = kEnsTendTiles[T.tend][1];
    return cdiv(D.ie - D.is + 1, TX) * cdiv(D.je - D.js + 1, TY) * cdiv(D.nk, T.tend_kc);
}

long long ens_blocks_vertvisc(const Dims& D, const EnsTuning& T)
{
    const int ncol = D.ie - D.is + 2;
    const int nrows = (D.je - D.js + 1) + (D.je - D.js + 2);
    return cdiv(ncol, T.vv_nb) * nrows;
}

long long ens_blocks_ppm(const Dims& D, const EnsTuning& T)
{
    const int n = (D.ie + 1) - (D.is - 1) + 1;
    return cdiv(n, T.ppm_nb) * (long long)(D.je - D.js + 1) * D.nk;
}

static inline int faces_gx(const Dims& D, int nb)
{
    const int nfaces = D.ie - (D.is - 1) + 1, step = nb - 1;
    return (nfaces - 1 + step - 1) / step;
}

long long ens_blocks_faces(const Dims& D, const EnsTuning& T)
{
    return (long long)faces_gx(D, T.faces_nb) * (D.je - D.js + 1);
}

constexpr int kEnsHaloNB = 256;

__host__ __device__ inline int halo_fields(int which) { return which == 3 ? 1 : 3; }

long long ens_blocks_halo(const Dims& D, int which)
{
    // per field of the group: the largest of its kinds' halo sizes
    const int nz = which < 2 ? D.nk : 1;
    long long mx = 0;
    for (int kind = 0; kind < 3; ++kind) {
        long long p = halo_points_per_layer(D, kind) * nz;
        if (p > mx) mx = p;
    }
    return cdiv(mx, kEnsHaloNB);
}

size_t ens_ovl_floats(const Dims& D)
{
    return (size_t)faces_gx(D, 64) * (size_t)(D.je - D.js + 1) * (size_t)D.nk;
}

// ---- tendency ----------------------------------------------------------------
template <int TX, int TY, bool UNI>
__global__ void __launch_bounds__(TX * TY)
k_ens_tendency(const EnsDomain* __restrict__ doms, const int* __restrict__ start, int n,
               int half, int KC)
{
    __shared__ __align__(16) EnsDomain E;
    const int b = (int)blockIdx.x;
    const int d = ens_find(start, n, b);
    ens_load(E, doms, d);
    int local = b - __ldg(start + d);
    const int gx = (E.D.ie - E.D.is + 1 + TX - 1) / TX;
    const int gy = (E.D.je - E.D.js + 1 + TY - 1) / TY;
    const int bx = local % gx;
    local /= gx;
    const int by = local % gy, bz = local / gy;
    const bool corr = half != 0;
    const float coef = corr ? (float)(0.5 * E.dt) : (float)E.dt;
    tendency_tile<TX, TY, UNI, float>(E.D, E.M, E.U, corr ? E.up : E.u, corr ? E.vp : E.v,
                                      corr ? E.hB : E.h0, E.u, E.v, corr ? E.u : E.up,
                                      corr ? E.v : E.vp, coef, E.hv_neglect, 1, KC, bx, by,
                                      bz);
}

template <int TX, int TY>
static void ens_tend_launch(const EnsDomain* doms, const int* start, int n, int total,
                            int half, int kc, bool uni, cudaStream_t s)
{
    dim3 block(TX, TY, 1);
    if (uni)
        k_ens_tendency<TX, TY, true><<<total, block, 0, s>>>(doms, start, n, half, kc);
    else
        k_ens_tendency<TX, TY, false><<<total, block, 0, s>>>(doms, start, n, half, kc);
}

cudaError_t launch_ens_tendency(const EnsDomain* doms, const int* start, int n, int total,
                                int half, const EnsTuning& T, bool uni, cudaStream_t s)
{
    if (total <= 0) return cudaSuccess;
    switch (T.tend) {
    case 1: ens_tend_launch<32, 4>(doms, start, n, total, half, T.tend_kc, uni, s); break;
    case 2: ens_tend_launch<64, 4>(doms, start, n, total, half, T.tend_kc, uni, s); break;
    case 3: ens_tend_launch<32, 16>(doms, start, n, total, half, T.tend_kc, uni, s); break;
    default: ens_tend_launch<32, 8>(doms, start, n, total, half, T.tend_kc, uni, s); break;
    }
    return cudaGetLastError();
}

// ---- vertical viscosity ----------------------------------------------------------
// Register caps as threads per SM, the single-domain kernels' measured best:
// vertical viscosity 1024 (8 CTAs of 128), continuity faces 640 (5 of 128).
template <int KMAX, int CH, int NB>
__global__ void __launch_bounds__(NB, 1024 / NB)
k_ens_vertvisc(const EnsDomain* __restrict__ doms, const int* __restrict__ start, int n,
               int half)
{
    __shared__ __align__(16) EnsDomain E;
    const int b = (int)blockIdx.x;
    const int d = ens_find(start, n, b);
    ens_load(E, doms, d);
    const int local = b - __ldg(start + d);
    const int gx = (E.D.ie - E.D.is + 2 + NB - 1) / NB;
    const bool corr = half != 0;
    // the single-domain mixed kernel's columns: two sweeps where they apply
    __shared__ float stage[2 * CH * 3 * NB];
    float* u = corr ? E.u : E.up;
    float* v = corr ? E.v : E.vp;
    const float* h = corr ? E.hB : E.h0;
    const double dt = corr ? 0.5 * E.dt : E.dt;
    if (!vertvisc_column_up<KMAX, CH, float, double, NB>(E.D, E.M, u, v, h, dt, E.VV, E.taux_bot,
                                                         E.tauy_bot, local % gx, local / gx,
                                                         stage))
        vertvisc_column<KMAX, CH, float, double, false, false, true>(
            E.D, E.M, u, v, h, dt, E.VV, E.taux_bot, E.tauy_bot, local % gx, local / gx);
}

template <int KMAX>
static void ens_vv_launch(const EnsDomain* doms, const int* start, int n, int total, int half,
                          const EnsTuning& T, cudaStream_t s)
{
    const int nb = T.vv_nb, ch = T.vv_ch;
#define VV_CASE(NB, CH)                                                                   \
    if (nb == NB && ch == CH) {                                                           \
        k_ens_vertvisc<KMAX, CH, NB><<<total, NB, 0, s>>>(doms, start, n, half);          \
        return;                                                                           \
    }
    VV_CASE(64, 2) VV_CASE(64, 4) VV_CASE(256, 2) VV_CASE(256, 4) VV_CASE(128, 2)
#undef VV_CASE
    k_ens_vertvisc<KMAX, 4, 128><<<total, 128, 0, s>>>(doms, start, n, half);
}

cudaError_t launch_ens_vertvisc(const EnsDomain* doms, const int* start, int n, int total,
                                int half, int kmax, const EnsTuning& T, cudaStream_t s)
{
    if (total <= 0) return cudaSuccess;
    if (kmax <= 80) ens_vv_launch<80>(doms, start, n, total, half, T, s);
    else if (kmax <= 128) ens_vv_launch<128>(doms, start, n, total, half, T, s);
    else if (kmax <= 256) ens_vv_launch<256>(doms, start, n, total, half, T, s);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// ---- continuity ------------------------------------------------------------------
template <int NB>
__global__ void __launch_bounds__(NB)
k_ens_ppm(const EnsDomain* __restrict__ doms, const int* __restrict__ start, int n, int half)
{
    __shared__ __align__(16) EnsDomain E;
    const int b = (int)blockIdx.x;
    const int d = ens_find(start, n, b);
    ens_load(E, doms, d);
    int local = b - __ldg(start + d);
    const int gx = ((E.D.ie + 1) - (E.D.is - 1) + 1 + NB - 1) / NB;
    const int gy = E.D.je - E.D.js + 1;
    const int bx = local % gx;
    local /= gx;
    ppm_cell_f(E.D, E.M, half ? E.hB : E.h0, E.hW, E.hE, (float)E.h_min, bx, local % gy,
               local / gy);
}

cudaError_t launch_ens_ppm(const EnsDomain* doms, const int* start, int n, int total, int half,
                           const EnsTuning& T, cudaStream_t s)
{
    if (total <= 0) return cudaSuccess;
    if (T.ppm_nb == 256) k_ens_ppm<256><<<total, 256, 0, s>>>(doms, start, n, half);
    else k_ens_ppm<128><<<total, 128, 0, s>>>(doms, start, n, half);
    return cudaGetLastError();
}

template <int NB>
__global__ void __launch_bounds__(NB, 640 / NB)
k_ens_faces(const EnsDomain* __restrict__ doms, const int* __restrict__ start, int n, int half)
{
    __shared__ __align__(16) EnsDomain E;
    const int b = (int)blockIdx.x;
    const int d = ens_find(start, n, b);
    ens_load(E, doms, d);
    const int local = b - __ldg(start + d);
    const int nfaces = E.D.ie - (E.D.is - 1) + 1;
    const int gx = (nfaces - 1 + NB - 2) / (NB - 1);
    const bool corr = half != 0;
    ContOutF O{corr ? E.hA : E.hB, E.uh, E.h_u, E.O2.FA_u_W0, E.O2.FA_u_WW, E.O2.FA_u_E0,
               E.O2.FA_u_EE, E.O2.uBT_WW, E.O2.uBT_EE, E.O2.du_cor};
    cont_faces_f(E.D, E.M, corr ? E.u : E.up, corr ? E.hB : E.h0, E.hW, E.hE, E.uhbt0, O,
                 E.ovl, corr ? 0.5 * E.dt : E.dt, local % gx, local / gx, gx);
}

cudaError_t launch_ens_faces(const EnsDomain* doms, const int* start, int n, int total,
                             int half, const EnsTuning& T, cudaStream_t s)
{
    if (total <= 0) return cudaSuccess;
    if (T.faces_nb == 64) k_ens_faces<64><<<total, 64, 0, s>>>(doms, start, n, half);
    else if (T.faces_nb == 256) k_ens_faces<256><<<total, 256, 0, s>>>(doms, start, n, half);
    else k_ens_faces<128><<<total, 128, 0, s>>>(doms, start, n, half);
    return cudaGetLastError();
}

// ---- halo fill ---------------------------------------------------------------------
// Job q = domain q / F, field q % F of the group `which`; every field of a group
// gets the blocks of the group's largest field, threads past a field's own
// halo size return.
__global__ void __launch_bounds__(kEnsHaloNB)
k_ens_halo(const EnsDomain* __restrict__ doms, const int* __restrict__ start, int njobs,
           int which)
{
    __shared__ __align__(16) EnsDomain E;
    const int b = (int)blockIdx.x;
    const int q = ens_find(start, njobs, b);
    const int F = halo_fields(which);
    ens_load(E, doms, q / F);
    if (!E.bc_fill) return;
    const int f = q % F;
    const long long t = (long long)(b - __ldg(start + q)) * kEnsHaloNB + threadIdx.x;
    if (which == 0) {
        float* p = f == 0 ? E.hB : f == 1 ? E.up : E.vp;
        halo_fill_point<float>(E.D, p, E.D.nk, f, t);
    } else if (which == 1) {
        float* p = f == 0 ? E.hA : f == 1 ? E.u : E.v;
        halo_fill_point<float>(E.D, p, E.D.nk, f, t);
    } else if (which == 2) {
        double* p = f == 0 ? E.eta_av : f == 1 ? E.ubt_av : E.vbt_av;
        halo_fill_point<double>(E.D, p, 1, f, t);
    } else {
        halo_fill_point<double>(E.D, E.eta, 1, 0, t);
    }
}

cudaError_t launch_ens_halo(const EnsDomain* doms, const int* start, int njobs, int total,
                            int which, cudaStream_t s)
{
    if (total <= 0) return cudaSuccess;
    k_ens_halo<<<total, kEnsHaloNB, 0, s>>>(doms, start, njobs, which);
    return cudaGetLastError();
}

} // namespace mom6b
