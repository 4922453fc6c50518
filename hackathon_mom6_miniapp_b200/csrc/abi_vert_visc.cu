// abi_vert_visc.cu -- launch_vert_visc_cra_{u,v}_kernel.
//
// The CUDA C backend's fused vertical viscosity (mom6_vert_visc_kernels.cu:
// 19-290, launchers :301-345): per water column, hvel/z_i bottom-up, the
// viscosity profile a(K), a tridiagonal solve that yields both the remnant
// visc_rem and the new velocity, and the bottom stress.  Unlike the serial
// vert_visc_apply it has no Rayleigh drag and also returns visc_rem.
//
// One thread per column.  hvel(k) and z_i(k) live in a per-thread local array
// (the caller's hvel / z_i scratch is not touched), c1 overwrites z_i as in
// the reference, and the inputs of four layers are loaded per step.
#include "../../include/mom6_cuda_c.h"
#include "abi_common.cuh"

using namespace mom6b::abi;

namespace {

constexpr double kRho0Abi = 1035.0;   // RHO_0, mom6_vert_visc_kernels.cu:14
constexpr int kAbiVvMaxNz = 256;      // columns deeper than this use the generic path

struct VvArgs {
    double *vel, *visc_rem, *tbot;
    const double *h, *mask, *tau;
    double Kv, Kv_ml, Kv_extra_bbl, Hmix, dt, dt_Rho0, h_neglect, I_Hbbl;
    int n1, n2, nz;
    int i0, i1, j0, j1;   // column range
    int di, dj;           // neighbour offset: (1,0) u columns, (0,1) v columns
};

__device__ __forceinline__ double botfn_of(double z2)
{
    const double z2_6 = z2 * z2 * z2 * z2 * z2 * z2;
    return 1.0 / (1.0 + 0.09 * z2_6);
}

template <int NZMAX>
__global__ void __launch_bounds__(128) k_abi_vert_visc(VvArgs A)
{
    double hv[NZMAX + 2];   // hvel(k)
    double zi[NZMAX + 2];   // z_i(k), then c1(k)
    const int w = A.i1 - A.i0 + 1;
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= w * (A.j1 - A.j0 + 1)) return;
    const int i = A.i0 + t % w, j = A.j0 + t / w;
    const int n1 = A.n1, n2 = A.n2, nz = A.nz;
    const size_t p2 = at2(i, j, n1);
    const size_t plane = (size_t)n1 * (size_t)n2;
    double* vc = A.vel + p2;
    double* rc = A.visc_rem + p2;
    if (!(A.mask[p2] > 0.0)) {
        for (int k = 1; k <= nz; ++k) rc[(size_t)(k - 1) * plane] = 1.0;
        A.tbot[p2] = 0.0;
        return;
    }
    const double* hc = A.h + p2;
    const double* hn = A.h + at2(i + A.di, j + A.dj, n1);
    const double hneg = A.h_neglect;

    // coefficient phase, bottom-up (:43-63)
    zi[nz + 1] = 0.0;
    for (int kt = nz; kt >= 1; kt -= 4) {
        double a0[4], a1[4], uv[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int k = kt - c;
            if (k >= 1) {
                const size_t o = (size_t)(k - 1) * plane;
                a0[c] = hc[o]; a1[c] = hn[o]; uv[c] = vc[o];
            }
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int k = kt - c;
            if (k >= 1) {
                const double h_harm = 2.0 * a0[c] * a1[c] / (a0[c] + a1[c] + hneg);
                const double h_arith = 0.5 * (a1[c] + a0[c]);
                const double h_delta = a1[c] - a0[c];
                double hvk = h_harm;
                if (uv[c] * h_delta < 0.0) {
                    const double bf = botfn_of(zi[k + 1]);
                    hvk = (1.0 - bf) * h_harm + bf * h_arith;
                }
                hv[k] = hvk;
                zi[k] = zi[k + 1] + h_harm * A.I_Hbbl;
            }
        }
    }

    // a(K) on the fly (:73-95, :106-121)
    auto a_at = [&](int K, double z_top) -> double {
        double Kv_tot = A.Kv;
        if (z_top < A.Hmix) {
            const double topfn = 1.0 - z_top / A.Hmix;
            Kv_tot = Kv_tot + (A.Kv_ml - A.Kv) * topfn;
        }
        Kv_tot = Kv_tot + A.Kv_extra_bbl * botfn_of(zi[K]);
        const double h_shear = 0.5 * (hv[K] + hv[K - 1] + hneg);
        return Kv_tot / h_shear;
    };
    const double a_bottom_num = A.Kv + A.Kv_extra_bbl;
    const double sfc_stress = A.dt_Rho0 * A.tau[p2] * A.mask[p2];
    const double dt = A.dt;

    double a_k = 0.0, a_k1, z_top = 0.0;
    if (nz > 1) {
        z_top = hv[1];
        a_k1 = a_at(2, z_top);
    } else {
        a_k1 = a_bottom_num / (0.5 * hv[nz] + hneg);
    }
    double h_eff = hv[1] + hneg;
    double b_denom_1 = h_eff + dt * a_k;
    double b1 = 1.0 / (b_denom_1 + dt * a_k1);
    double d1 = b_denom_1 * b1;
    double vr_prev = b1 * h_eff;
    double u_prev = b1 * (h_eff * vc[0] + sfc_stress);
    rc[0] = vr_prev;
    vc[0] = u_prev;
    for (int kt = 2; kt <= nz; kt += 4) {
        double uv[4];
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if (kt + c <= nz) uv[c] = vc[(size_t)(kt + c - 1) * plane];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int k = kt + c;
            if (k <= nz) {
                zi[k] = dt * a_k1 * b1;   // c1(k); z_i(k) is dead from here on
                a_k = a_k1;
                if (k < nz) {
                    z_top = z_top + hv[k];
                    a_k1 = a_at(k + 1, z_top);
                } else {
                    a_k1 = a_bottom_num / (0.5 * hv[nz] + hneg);
                }
                h_eff = hv[k] + hneg;
                b_denom_1 = h_eff + dt * (a_k * d1);
                b1 = 1.0 / (b_denom_1 + dt * a_k1);
                d1 = b_denom_1 * b1;
                vr_prev = (h_eff + dt * a_k * vr_prev) * b1;
                u_prev = (h_eff * uv[c] + dt * a_k * u_prev) * b1;
                const size_t o = (size_t)(k - 1) * plane;
                rc[o] = vr_prev;
                vc[o] = u_prev;
            }
        }
    }
    // back substitution (:133-138)
    double vr_below = vr_prev, u_below = u_prev;
    for (int kt = nz - 1; kt >= 1; kt -= 4) {
        double pr[4], pu[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int k = kt - c;
            if (k >= 1) {
                const size_t o = (size_t)(k - 1) * plane;
                pr[c] = rc[o]; pu[c] = vc[o];
            }
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int k = kt - c;
            if (k >= 1) {
                const size_t o = (size_t)(k - 1) * plane;
                vr_below = pr[c] + zi[k + 1] * vr_below;
                u_below = pu[c] + zi[k + 1] * u_below;
                rc[o] = vr_below;
                vc[o] = u_below;
            }
        }
    }
    A.tbot[p2] = kRho0Abi * u_prev * a_k1;
}

void launch_abi_vv(const VvArgs& A, void* stream)
{
    const int ncol = (A.i1 - A.i0 + 1) * (A.j1 - A.j0 + 1);
    if (A.i1 < A.i0 || A.j1 < A.j0 || A.nz < 1) return;
    const int nb = 128;
    dim3 grid((ncol + nb - 1) / nb);
    cudaStream_t s = (cudaStream_t)stream;
    if (A.nz <= 80) k_abi_vert_visc<80><<<grid, nb, 0, s>>>(A);
    else if (A.nz <= kAbiVvMaxNz) k_abi_vert_visc<kAbiVvMaxNz><<<grid, nb, 0, s>>>(A);
    else k_abi_vert_visc<1024><<<grid, nb, 0, s>>>(A);
}

} // namespace

extern "C" void launch_vert_visc_cra_u_kernel(double* u, double* h, double* mask2dCu,
                                              double* visc_rem_u, double* taux_bot,
                                              double* taux, double Kv, double Kv_ml,
                                              double Kv_extra_bbl, double Hmix, double,
                                              double dt, double dt_Rho0, double h_neglect,
                                              double I_Hbbl, int n1, int n2, int nz, int is_l,
                                              int ie_l, int js_l, int je_l, double*, double*,
                                              int, int, int, int, void* stream)
{
    flush_deferred();
    if (nz > 1024) return;
    VvArgs A{u, visc_rem_u, taux_bot, h, mask2dCu, taux, Kv, Kv_ml, Kv_extra_bbl, Hmix,
             dt, dt_Rho0, h_neglect, I_Hbbl, n1, n2, nz,
             std::max(is_l - 1, 1), std::min(ie_l, n1), std::max(js_l, 1), std::min(je_l, n2),
             1, 0};
    launch_abi_vv(A, stream);
}

extern "C" void launch_vert_visc_cra_v_kernel(double* v, double* h, double* mask2dCv,
                                              double* visc_rem_v, double* tauy_bot,
                                              double* tauy, double Kv, double Kv_ml,
                                              double Kv_extra_bbl, double Hmix, double,
                                              double dt, double dt_Rho0, double h_neglect,
                                              double I_Hbbl, int n1, int n2, int nz, int is_l,
                                              int ie_l, int js_l, int je_l, double*, double*,
                                              int, int, int, int, void* stream)
{
    flush_deferred();
    if (nz > 1024) return;
    VvArgs A{v, visc_rem_v, tauy_bot, h, mask2dCv, tauy, Kv, Kv_ml, Kv_extra_bbl, Hmix,
             dt, dt_Rho0, h_neglect, I_Hbbl, n1, n2, nz,
             std::max(is_l, 1), std::min(ie_l, n1), std::max(js_l - 1, 1), std::min(je_l, n2),
             0, 1};
    launch_abi_vv(A, stream);
}
