// k_hor_visc.cu -- hor_visc with every scheme branch of the serial module
// (mom6_hor_visc_serial.F90:464-1109): Laplacian and biharmonic viscosity,
// Smagorinsky and Leith (optionally modified Leith) dynamic viscosities,
// free- or no-slip shear, and the thickness-aware stability bounds.  The
// driver's configuration (Laplacian, constant Kh, free slip, no bounds) stays
// in the fused tendency kernel; any other configuration runs this kernel
// first and the tendency reads its diffu, diffv.
//
// One CTA per 32 x 8 tile and kKC consecutive layers.  The biharmonic and Leith chains
// reach three points beyond the outputs (Ah <- Del2vort_q <- vort_xy_dx <-
// vort_xy), so the CTA stages u, v, h on a 40 x 16 region (4 points of halo)
// and evaluates each intermediate of the serial loop nest in shared memory,
// one barrier per stage, each stage over the part of the region the later
// stages read (the region less 1, 2 or 3 points).  On a uniform grid (UNI)
// the metrics and init's constants are scalars of the parameter bank.  Each intermediate keeps the
// serial's value outside the range the serial writes it on (0, or 1 for
// hrat_min), so the boundary stencils see what the serial's persistent work
// arrays hold there.  Only the points the velocity update reads are
// produced: diffu on I in [is, ie-1] x [js, je], diffv on [is, ie] x
// [js, je-1]; for those the shared CS%Kh / CS%Ah of the serial code are
// always the freshly computed values.  Built without FMA contraction so the
// accelerations equal the serial restatement bit for bit.
#include "hor_visc.h"

namespace mom6b {

namespace {

constexpr int kTX = 32, kTY = 8, kH = 4;
constexpr int kRX = kTX + 2 * kH, kRY = kTY + 2 * kH;   // staged region
constexpr int kRN = kRX * kRY;
constexpr int kNT = kTX * kTY;

// the shared arrays of one CTA (dynamic shared memory, kRN doubles each)
enum {
    S_U, S_V, S_H, S_SXX, S_SXY, S_VORT, S_D2U, S_D2V, S_VDX, S_VDY, S_D2VQ, S_HRAT,
    S_DIV, S_DDX, S_DDY, S_STRXX, S_STRXY, S_U1, S_V1, S_H1, S_COUNT
};
constexpr int kKC = 5;   // layers per CTA

// inv_PI3 = 1/3.14159265358979**3 and inv_PI6 = 1/3.14159265358979**6
// (mom6_hor_visc_serial.F90:154-155), the powers and quotients correctly
// rounded.
__device__ constexpr double kInvPI3 = 0x1.08345eb45d78dp-5;
__device__ constexpr double kInvPI6 = 0x1.10ac0e0a9d181p-10;

__device__ __forceinline__ double sq(double x) { return x * x; }

template <bool UNI>
__global__ void __launch_bounds__(kNT, 2)
k_hor_visc_gen(Dims D, Metrics M, UniMetrics U, HorViscGen P, const double* __restrict__ u,
               const double* __restrict__ v, const double* __restrict__ h,
               double* __restrict__ diffu, double* __restrict__ diffv)
{
    extern __shared__ double smem[];
    const int tid = (int)threadIdx.x;
    const int i0 = D.is + (int)blockIdx.x * kTX, j0 = D.js + (int)blockIdx.y * kTY;
    const int ri = i0 - kH, rj = j0 - kH;            // global index of region (0, 0)
    const int kb = 1 + (int)blockIdx.z * kKC;
    const int ke = kb + kKC - 1 < D.nk ? kb + kKC - 1 : D.nk;
    const int is = D.is, ie = D.ie, js = D.js, je = D.je;

// array a at offset (di, dj) from the current point, whose region index is q
#define SQ(a, di, dj) smem[(a) * kRN + q + (dj) * kRX + (di)]
#define G2(a, i, j) (UNI ? U.a : MOM6B_A2(M.a, i, j, D))
#define X2(a, i, j) (UNI ? P.s##a : MOM6B_A2(P.a, i, j, D))
    // region point p -> global (i, j); in(i, j, lo, hi) keeps neighbour reads in the region
    auto at = [&](int p, int& i, int& j) {
        const int b = p / kRX;
        i = ri + (p - b * kRX);
        j = rj + b;
    };
    // point p of the region less m points on every side -> global (i, j)
    auto at_in = [&](int p, int m, int& i, int& j) {
        const int w = kRX - 2 * m;
        const int b = p / w;
        i = ri + m + (p - b * w);
        j = rj + m + b;
    };
    auto count_in = [](int m) { return (kRX - 2 * m) * (kRY - 2 * m); };
    auto inreg = [&](int i, int j, int dl, int dr, int dd, int du) {
        return i - dl >= ri && i + dr < ri + kRX && j - dd >= rj && j + du < rj + kRY;
    };

    // ---- stage 0: u, v, h of layer k on the region into buffer b, with
    // cp.async: the next layer's copies run while the current one is computed
    auto stage = [&](int k, int b) {
        const size_t koff = (size_t)(k - 1) * (size_t)D.plane;
        for (int p = tid; p < kRN; p += kNT) {
            int i, j;
            at(p, i, j);
            const bool ok = i >= 1 && i <= D.n1 && j >= 1 && j <= D.n2;
            const size_t o = ok ? koff + (size_t)(j - 1) * D.n1 + (size_t)(i - 1) : 0;
            cp_async_elem(&smem[(b ? S_U1 : S_U) * kRN + p], u + o, ok);
            cp_async_elem(&smem[(b ? S_V1 : S_V) * kRN + p], v + o, ok);
            cp_async_elem(&smem[(b ? S_H1 : S_H) * kRN + p], h + o, ok);
        }
        cp_async_commit();
    };
    stage(kb, 0);
  for (int k = kb; k <= ke; ++k) {
    const int b = (k - kb) & 1;
    const int AU = b ? S_U1 : S_U, AV = b ? S_V1 : S_V, AH = b ? S_H1 : S_H;
    const size_t koff = (size_t)(k - 1) * (size_t)D.plane;
    cp_async_wait_all();
    // layer k is staged and visible; every thread is done with layer k-1,
    // whose buffer the next copies overwrite
    __syncthreads();
    if (k < ke) stage(k + 1, b ^ 1);

    // ---- stage 1: sh_xx (h), sh_xy and vort_xy (q), div_xx (h) (:496-535, :612-624, :661-665)
    for (int p = tid; p < count_in(1); p += kNT) {
        int i, j;
        at_in(p, 1, i, j);
        const int q = (j - rj) * kRX + (i - ri);
        double sxx = 0.0, sxy = 0.0, vort = 0.0, dv = 0.0;
        // every metric read below stays inside [is-2, ie+2] x [js-2, je+2]
        if (inreg(i, j, 1, 1, 1, 1)) {
            if (i >= is - 1 && i <= ie + 1 && j >= js - 1 && j <= je + 1) {
                const double dudx = G2(DY_dxT, i, j) * ((G2(IdyCu, i, j) * SQ(AU, 0, 0)) -
                                                        (G2(IdyCu, i - 1, j) * SQ(AU, -1, 0)));
                const double dvdy = G2(DX_dyT, i, j) * ((G2(IdxCv, i, j) * SQ(AV, 0, 0)) -
                                                        (G2(IdxCv, i, j - 1) * SQ(AV, 0, -1)));
                sxx = dudx - dvdy;
                if (P.mod_leith && i >= is && i <= ie && j >= js && j <= je) dv = dudx + dvdy;
            }
            if (i >= is - 1 && i <= ie && j >= js - 1 && j <= je) {
                const double dvdx = G2(DY_dxBu, i, j) * ((SQ(AV, 1, 0) * G2(IdyCv, i + 1, j)) -
                                                         (SQ(AV, 0, 0) * G2(IdyCv, i, j)));
                const double dudy = G2(DX_dyBu, i, j) * ((SQ(AU, 0, 1) * G2(IdxCu, i, j + 1)) -
                                                         (SQ(AU, 0, 0) * G2(IdxCu, i, j)));
                const double mB = G2(mask2dBu, i, j);
                const double f = P.no_slip ? (2.0 - mB) : mB;
                sxy = f * (dvdx + dudy);
                if (P.leith_kh) vort = f * (dvdx - dudy);
            }
        }
        SQ(S_SXX, 0, 0) = sxx;
        SQ(S_SXY, 0, 0) = sxy;
        SQ(S_VORT, 0, 0) = vort;
        SQ(S_DIV, 0, 0) = dv;
    }
    __syncthreads();

    // ---- stage 2: Del2u, Del2v (:587-608), vort_xy_dx/dy (:627-643),
    //      div_xx_dx/dy (:667-677), hrat_min (:732-739)
    for (int p = tid; p < count_in(2); p += kNT) {
        int i, j;
        at_in(p, 2, i, j);
        const int q = (j - rj) * kRX + (i - ri);
        double d2u = 0.0, d2v = 0.0, vdx = 0.0, vdy = 0.0, ddx = 0.0, ddy = 0.0, hr = 1.0;
        if (inreg(i, j, 1, 1, 1, 1)) {
            if (P.bih) {
                if (i >= is - 1 && i <= ie && j >= js && j <= je)
                    d2u = X2(Idx2dyCu, i, j) * ((G2(dx2q, i, j) * SQ(S_SXY, 0, 0)) -
                                                (G2(dx2q, i, j - 1) * SQ(S_SXY, 0, -1))) +
                          X2(Idxdy2u, i, j) * ((G2(dy2h, i + 1, j) * SQ(S_SXX, 1, 0)) -
                                               (G2(dy2h, i, j) * SQ(S_SXX, 0, 0)));
                if (i >= is && i <= ie && j >= js - 1 && j <= je)
                    d2v = X2(Idxdy2v, i, j) * ((G2(dy2q, i, j) * SQ(S_SXY, 0, 0)) -
                                               (G2(dy2q, i - 1, j) * SQ(S_SXY, -1, 0))) -
                          X2(Idx2dyCv, i, j) * ((G2(dx2h, i, j + 1) * SQ(S_SXX, 0, 1)) -
                                                (G2(dx2h, i, j) * SQ(S_SXX, 0, 0)));
            }
            if (P.leith_kh) {
                if (i >= is && i <= ie && j >= js && j <= je)
                    vdx = G2(DY_dxBu, i, j) * ((SQ(S_VORT, 0, 0) * G2(IdyCu, i, j)) -
                                               (SQ(S_VORT, -1, 0) * G2(IdyCu, i - 1, j)));
                if (i >= is - 1 && i <= ie && j >= js && j <= je)
                    vdy = G2(DX_dyBu, i, j) * ((SQ(S_VORT, 0, 0) * G2(IdxCv, i, j)) -
                                               (SQ(S_VORT, 0, -1) * G2(IdxCv, i, j - 1)));
                if (P.mod_leith) {
                    if (i >= is - 1 && i <= ie && j >= js && j <= je)
                        ddx = G2(IdxCu, i, j) * (SQ(S_DIV, 1, 0) - SQ(S_DIV, 0, 0));
                    if (i >= is && i <= ie && j >= js - 1 && j <= je)
                        ddy = G2(IdyCv, i, j) * (SQ(S_DIV, 0, 1) - SQ(S_DIV, 0, 0));
                }
            }
            if (P.bb && i >= is && i <= ie && j >= js && j <= je) {
                // CS%h_u(I, j), CS%h_v(i, J) with the land mask (:552-572)
                // di, dj: the face's offset from the point (0 or -1)
                auto hu = [&](int di) {
                    return 0.5 * (G2(mask2dT, i + di, j) * SQ(AH, di, 0) +
                                  G2(mask2dT, i + di + 1, j) * SQ(AH, di + 1, 0));
                };
                auto hv = [&](int dj) {
                    return 0.5 * (G2(mask2dT, i, j + dj) * SQ(AH, 0, dj) +
                                  G2(mask2dT, i, j + dj + 1) * SQ(AH, 0, dj + 1));
                };
                const double h_min = dmin(dmin(dmin(hu(0), hu(-1)), hv(0)), hv(-1));
                hr = dmin(1.0, h_min / (SQ(AH, 0, 0) + P.h_neglect));
            }
        }
        SQ(S_D2U, 0, 0) = d2u;
        SQ(S_D2V, 0, 0) = d2v;
        SQ(S_VDX, 0, 0) = vdx;
        SQ(S_VDY, 0, 0) = vdy;
        SQ(S_DDX, 0, 0) = ddx;
        SQ(S_DDY, 0, 0) = ddy;
        SQ(S_HRAT, 0, 0) = hr;
    }
    __syncthreads();

    // ---- stage 3: Del2vort_q (:647-658) ------------------------------------
    if (P.leith_ah) {
        for (int p = tid; p < count_in(3); p += kNT) {
            int I, J;
            at_in(p, 3, I, J);
            const int q = (J - rj) * kRX + (I - ri);
            double d = 0.0;
            if (inreg(I, J, 0, 1, 0, 1) && I >= is - 1 && I <= ie && J >= js - 1 && J <= je)
                d = G2(DY_dxBu, I, J) * ((SQ(S_VDX, 1, 0) * G2(IdyCv, I + 1, J)) -
                                         (SQ(S_VDX, 0, 0) * G2(IdyCv, I, J))) +
                    G2(DX_dyBu, I, J) * ((SQ(S_VDY, 0, 1) * G2(IdxCu, I, J + 1)) -
                                         (SQ(S_VDY, 0, 0) * G2(IdxCu, I, J)));
            SQ(S_D2VQ, 0, 0) = d;
        }
        __syncthreads();
    }

    // ---- stage 4: str_xx at h-points [is, ie] x [js, je] (:744-896 and
    //      :900-906) and str_xy at q-points [is-1, ie] x [js-1, je] (:900-1058)
    // h-points of the tile and one beyond on the east and north
    // ([i0, i0+TX] x [j0, j0+TY]); q-points of the tile and one beyond on the
    // west and south ([i0-1, i0+TX-1] x [j0-1, j0+TY-1])
    for (int p = tid; p < count_in(3); p += kNT) {
        int i, j;
        at_in(p, 3, i, j);
        const int q = (j - rj) * kRX + (i - ri);
        if (i >= i0 && j >= j0 && i >= is && i <= ie && j >= js && j <= je) {
            double shear = 0.0;
            if (P.smag_kh || P.smag_ah) {
                const double sh_xx_sq = sq(SQ(S_SXX, 0, 0));
                const double sh_xy_sq =
                    0.25 * ((sq(SQ(S_SXY, -1, -1)) + sq(SQ(S_SXY, 0, 0))) +
                            (sq(SQ(S_SXY, -1, 0)) + sq(SQ(S_SXY, 0, -1))));
                shear = sqrt(sh_xx_sq + sh_xy_sq);
            }
            const double hr = SQ(S_HRAT, 0, 0);
            double vbr = 1.0, str = 0.0;
            if (P.lap) {
                double K = P.Kh_bg;
                if (P.smag_kh) K = dmax(K, X2(L2c, i, j) * shear);
                if (P.leith_kh) {
                    const double gvm = sqrt(sq(0.5 * (SQ(S_VDX, 0, 0) + SQ(S_VDX, 0, -1))) +
                                            sq(0.5 * (SQ(S_VDY, 0, 0) + SQ(S_VDY, -1, 0))));
                    double gdm = 0.0;
                    if (P.mod_leith)
                        gdm = sqrt(sq(0.5 * (SQ(S_DDX, 0, 0) + SQ(S_DDX, -1, 0))) +
                                   sq(0.5 * (SQ(S_DDY, 0, 0) + SQ(S_DDY, 0, -1))));
                    K = dmax(K, X2(L3c, i, j) * (gvm + gdm) * kInvPI3);
                }
                K = dmax(K, P.Kh_bg_min);
                if (P.bb) {
                    // better_bound_Kh and better_bound_Ah: the remaining budget (:779-792)
                    const double Kh_max_here = hr * X2(Kh_Max, i, j);
                    if (K >= Kh_max_here) {
                        vbr = 0.0;
                        K = Kh_max_here;
                    } else if (K > 0.0) {
                        vbr = 1.0 - K / Kh_max_here;
                    }
                }
                str = -(K * SQ(S_SXX, 0, 0));
            }
            if (P.bih) {
                double A = P.Ah_bg;
                if (P.smag_ah) A = dmax(A, X2(Bc, i, j) * shear);
                if (P.leith_ah) {
                    const double d2vh = 0.25 * ((SQ(S_D2VQ, 0, 0) + SQ(S_D2VQ, -1, -1)) +
                                                (SQ(S_D2VQ, -1, 0) + SQ(S_D2VQ, 0, -1)));
                    A = dmax(A, X2(B6c, i, j) * fabs(d2vh) * kInvPI6);
                }
                if (P.bb) A = dmin(A, vbr * hr * X2(Ah_Max, i, j));
                const double d_del2u = (G2(IdyCu, i, j) * SQ(S_D2U, 0, 0)) -
                                       (G2(IdyCu, i - 1, j) * SQ(S_D2U, -1, 0));
                const double d_del2v = (G2(IdxCv, i, j) * SQ(S_D2V, 0, 0)) -
                                       (G2(IdxCv, i, j - 1) * SQ(S_D2V, 0, -1));
                const double d_str = A * ((G2(DY_dxT, i, j) * d_del2u) -
                                          (G2(DX_dyT, i, j) * d_del2v));
                str = str + d_str;
            }
            SQ(S_STRXX, 0, 0) = str * (SQ(AH, 0, 0) * G2(red_xx, i, j));
        }
        if (i <= i0 + kTX - 1 && j <= j0 + kTY - 1 && i >= is - 1 && i <= ie && j >= js - 1 &&
            j <= je) {
            const int I = i, J = j;
            double shear = 0.0;
            if (P.smag_kh || P.smag_ah) {
                const double sh_xx_sq =
                    0.25 * ((sq(SQ(S_SXX, 0, 0)) + sq(SQ(S_SXX, 1, 1))) +
                            (sq(SQ(S_SXX, 1, 0)) + sq(SQ(S_SXX, 0, 1))));
                const double sh_xy_sq = sq(SQ(S_SXY, 0, 0));
                shear = sqrt(sh_xx_sq + sh_xy_sq);
            }
            const double h_min = P.bb ? 0.25 * ((SQ(S_HRAT, 0, 0) + SQ(S_HRAT, 1, 1)) +
                                                (SQ(S_HRAT, 1, 0) + SQ(S_HRAT, 0, 1)))
                                      : 1.0;
            double str = 0.0;
            if (P.lap) {
                double K = P.Kh_bg;
                if (P.smag_kh) K = dmax(K, X2(L2c, I, J) * shear);
                if (P.leith_kh) {
                    const double gvm = sqrt(sq(0.5 * (SQ(S_VDX, 0, 0) + SQ(S_VDX, 1, 0))) +
                                            sq(0.5 * (SQ(S_VDY, 0, 0) + SQ(S_VDY, 0, 1))));
                    K = dmax(K, X2(L3c, I, J) * gvm * kInvPI3);
                }
                K = dmax(K, P.Kh_bg_min);
                if (P.bb) K = dmin(K, h_min * X2(Kh_Max, I, J));
                str = -(K * SQ(S_SXY, 0, 0));
            }
            if (P.bih) {
                double A = P.Ah_bg;
                if (P.smag_ah) A = dmax(A, X2(Bc, I, J) * shear);
                if (P.leith_ah) A = dmax(A, X2(B6c, I, J) * fabs(SQ(S_D2VQ, 0, 0)) * kInvPI6);
                if (P.bb) A = dmin(A, h_min * X2(Ah_Max, I, J));
                const double d_str =
                    A * ((G2(DY_dxBu, I, J) * ((SQ(S_D2V, 1, 0) * G2(IdyCv, I + 1, J)) -
                                               (SQ(S_D2V, 0, 0) * G2(IdyCv, I, J)))) +
                         (G2(DX_dyBu, I, J) * ((SQ(S_D2U, 0, 1) * G2(IdxCu, I, J + 1)) -
                                               (SQ(S_D2U, 0, 0) * G2(IdxCu, I, J)))));
                str = str + d_str;
            }
            const double hq = 0.25 * ((SQ(AH, 0, 0) + SQ(AH, 1, 1)) +
                                      (SQ(AH, 1, 0) + SQ(AH, 0, 1)));
            SQ(S_STRXY, 0, 0) = P.no_slip ? str * (hq * G2(red_xy, I, J))
                                         : str * (hq * G2(mask2dBu, I, J) * G2(red_xy, I, J));
        }
    }
    __syncthreads();

    // ---- stage 5: diffu, diffv of the tile's points (:1063-1080) ----------
    const int I = i0 + tid % kTX, j = j0 + tid / kTX;
    const int q = (j - rj) * kRX + (I - ri);
    const size_t oo = koff + (size_t)(j - 1) * D.n1 + (size_t)(I - 1);
    if (I <= ie - 1 && j <= je) {
        const double h_u = 0.5 * (G2(mask2dT, I, j) * SQ(AH, 0, 0) +
                                  G2(mask2dT, I + 1, j) * SQ(AH, 1, 0));
        diffu[oo] = ((G2(IdxCu, I, j) * ((G2(dx2q, I, j - 1) * SQ(S_STRXY, 0, -1)) -
                                         (G2(dx2q, I, j) * SQ(S_STRXY, 0, 0))) +
                      G2(IdyCu, I, j) * ((G2(dy2h, I, j) * SQ(S_STRXX, 0, 0)) -
                                         (G2(dy2h, I + 1, j) * SQ(S_STRXX, 1, 0)))) *
                     G2(IareaCu, I, j)) /
                    (h_u + P.h_neglect);
    }
    if (I <= ie && j <= je - 1) {
        const int i = I, J = j;
        const double h_v = 0.5 * (G2(mask2dT, i, J) * SQ(AH, 0, 0) +
                                  G2(mask2dT, i, J + 1) * SQ(AH, 0, 1));
        diffv[oo] = ((G2(IdyCv, i, J) * ((G2(dy2q, i - 1, J) * SQ(S_STRXY, -1, 0)) -
                                         (G2(dy2q, i, J) * SQ(S_STRXY, 0, 0))) -
                      G2(IdxCv, i, J) * ((G2(dx2h, i, J) * SQ(S_STRXX, 0, 0)) -
                                         (G2(dx2h, i, J + 1) * SQ(S_STRXX, 0, 1)))) *
                     G2(IareaCv, i, J)) /
                    (h_v + P.h_neglect);
    }
  }  // layer loop
#undef SQ
#undef G2
#undef X2
}

}  // namespace

cudaError_t launch_hor_visc_gen(const Dims& D, const Metrics& M, const UniMetrics& U,
                                const HorViscGen& P, const double* u, const double* v,
                                const double* h, double* diffu, double* diffv, cudaStream_t s)
{
    const size_t smem = (size_t)S_COUNT * kRN * sizeof(double);
    const bool uni = U.valid && P.uni;
    auto kern = uni ? k_hor_visc_gen<true> : k_hor_visc_gen<false>;
    cudaError_t e =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid((D.ie - D.is + 1 + kTX - 1) / kTX, (D.je - D.js + 1 + kTY - 1) / kTY,
              (D.nk + kKC - 1) / kKC);
    kern<<<grid, kNT, smem, s>>>(D, M, U, P, u, v, h, diffu, diffv);
    return cudaGetLastError();
}

}  // namespace mom6b
