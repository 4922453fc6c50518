// abi_coriolis.cu -- Coriolis and momentum advection entry points.
//
// The reference's CUDA C CorAdCalc is split into circulation/area/KE terms,
// vorticity and potential vorticity, optional Arakawa coefficients and the
// Sadourny or Arakawa acceleration (mom6_coriolis_kernels.cu:14-535,
// launchers :545-708).  Each entry point here covers the same index ranges
// with the same operation order.  phase1_kernel_smem and phase1_kernel
// compute identical values in the reference (the shared-memory tile only
// changes where the operands are read from), so both map to one kernel.
#include "../../include/mom6_cuda_c.h"
#include "abi_common.cuh"

using namespace mom6b::abi;

namespace {

constexpr double kC1_12 = 1.0 / 12.0;
constexpr double kC1_24 = 1.0 / 24.0;

// dvdx, dudy on [is-1, ie] x [js-1, je]; hArea_v on [is, ie+1] x [js-1, je];
// hArea_u on [is-1, ie] x [js, je+1]; KE on [is, ie] x [js, je] (:67-118)
struct Phase1 {
    double *dvdx, *dudy, *hArea_u, *hArea_v, *KE;
    const double *u, *v, *h, *dyCv, *dxCu, *dyCu, *dxCv, *areaT;
    int n1, n2, is, ie, js, je;
    bool circ, ke;

    __device__ void operator()(int i, int j, int k) const
    {
        const size_t p = at3(i, j, k, n1, n2), p2 = at2(i, j, n1);
        if (circ) {
            if (i >= is - 1 && i <= ie && j >= js - 1 && j <= je) {
                dvdx[p] = v[at3(i + 1, j, k, n1, n2)] * dyCv[at2(i + 1, j, n1)] - v[p] * dyCv[p2];
                dudy[p] = u[at3(i, j + 1, k, n1, n2)] * dxCu[at2(i, j + 1, n1)] - u[p] * dxCu[p2];
            }
            if (i >= is && i <= ie + 1 && j >= js - 1 && j <= je)
                hArea_v[p] = 0.5 * (areaT[p2] * h[p] +
                                    areaT[at2(i, j + 1, n1)] * h[at3(i, j + 1, k, n1, n2)]);
            if (i >= is - 1 && i <= ie && j >= js && j <= je + 1)
                hArea_u[p] = 0.5 * (areaT[p2] * h[p] +
                                    areaT[at2(i + 1, j, n1)] * h[at3(i + 1, j, k, n1, n2)]);
        }
        if (ke && i >= is && i <= ie && j >= js && j <= je) {
            const size_t pw = at3(i - 1, j, k, n1, n2), ps = at3(i, j - 1, k, n1, n2);
            const double xs = dyCu[p2] * u[p] * u[p] + dyCu[at2(i - 1, j, n1)] * u[pw] * u[pw];
            const double ys = dxCv[p2] * v[p] * v[p] + dxCv[at2(i, j - 1, n1)] * v[ps] * v[ps];
            KE[p] = 0.25 * (xs + ys) / areaT[p2];
        }
    }
};

void run_phase1(const Phase1& P, int n3, void* stream)
{
    const Box b = clip(Box{P.is - 1, P.ie + 1, P.js - 1, P.je + 1}, P.n1, P.n2);
    run_box(b, n3, stream, [=] __device__(int i, int j, int k) { P(i, j, k); });
}

// q at a vorticity point straight from u, v, h (:15-48)
__device__ __forceinline__ double pv_at(const double* u, const double* v, const double* h,
                                        const double* dyCv, const double* dxCu,
                                        const double* areaT, const double* IareaBu,
                                        const double* CoriolisBu, const double* mask2dBu,
                                        int n1, int n2, int i, int j, int k)
{
    const size_t p2 = at2(i, j, n1), pe2 = at2(i + 1, j, n1), pn2 = at2(i, j + 1, n1),
                 pne2 = at2(i + 1, j + 1, n1);
    const size_t p = at3(i, j, k, n1, n2), pe = at3(i + 1, j, k, n1, n2),
                 pn = at3(i, j + 1, k, n1, n2), pne = at3(i + 1, j + 1, k, n1, n2);
    const double dvdx = v[pe] * dyCv[pe2] - v[p] * dyCv[p2];
    const double dudy = u[pn] * dxCu[pn2] - u[p] * dxCu[p2];
    const double rel = mask2dBu[p2] * (dvdx - dudy) * IareaBu[p2];
    const double absv = CoriolisBu[p2] + rel;
    const double hau = 0.5 * (areaT[p2] * h[p] + areaT[pe2] * h[pe]);
    const double hau_n = 0.5 * (areaT[pn2] * h[pn] + areaT[pne2] * h[pne]);
    const double hav = 0.5 * (areaT[p2] * h[p] + areaT[pn2] * h[pn]);
    const double hav_e = 0.5 * (areaT[pe2] * h[pe] + areaT[pne2] * h[pne]);
    const double haq = hau + hau_n + hav + hav_e;
    const double aq = areaT[p2] + areaT[pne2] + areaT[pe2] + areaT[pn2];
    return absv * aq / (haq + 1.0e-20);
}

// KE at a tracer point (:51-64)
__device__ __forceinline__ double ke_at(const double* u, const double* v, const double* dyCu,
                                        const double* dxCv, const double* areaT, int n1, int n2,
                                        int i, int j, int k)
{
    const size_t p2 = at2(i, j, n1), p = at3(i, j, k, n1, n2);
    const size_t pw = at3(i - 1, j, k, n1, n2), ps = at3(i, j - 1, k, n1, n2);
    const double xs = dyCu[p2] * u[p] * u[p] + dyCu[at2(i - 1, j, n1)] * u[pw] * u[pw];
    const double ys = dxCv[p2] * v[p] * v[p] + dxCv[at2(i, j - 1, n1)] * v[ps] * v[ps];
    return 0.25 * (xs + ys) / areaT[p2];
}

} // namespace

extern "C" void launch_phase1_kernel(double* dvdx, double* dudy, double* hArea_u,
                                     double* hArea_v, double* KE, double* u, double* v,
                                     double* h, double* dyCv, double* dxCu, double* dyCu,
                                     double* dxCv, double* areaT, int n1, int n2, int n3,
                                     int is_l, int ie_l, int js_l, int je_l, int, int, int, int,
                                     int, int, void* stream)
{
    flush_deferred();
    run_phase1(Phase1{dvdx, dudy, hArea_u, hArea_v, KE, u, v, h, dyCv, dxCu, dyCu, dxCv, areaT,
                      n1, n2, is_l, ie_l, js_l, je_l, true, true},
               n3, stream);
}

extern "C" void launch_phase1_kernel_smem(double* dvdx, double* dudy, double* hArea_u,
                                          double* hArea_v, double* KE, double* u, double* v,
                                          double* h, double* dyCv, double* dxCu, double* dyCu,
                                          double* dxCv, double* areaT, int n1, int n2, int n3,
                                          int is_l, int ie_l, int js_l, int je_l, int, int, int,
                                          int, int, int, void* stream)
{
    flush_deferred();
    run_phase1(Phase1{dvdx, dudy, hArea_u, hArea_v, KE, u, v, h, dyCv, dxCu, dyCu, dxCv, areaT,
                      n1, n2, is_l, ie_l, js_l, je_l, true, true},
               n3, stream);
}

extern "C" void launch_phase1a_circ_kernel(double* dvdx, double* dudy, double* hArea_u,
                                           double* hArea_v, double* u, double* v, double* h,
                                           double* dyCv, double* dxCu, double* areaT, int n1,
                                           int n2, int n3, int is_l, int ie_l, int js_l,
                                           int je_l, int, int, int, int, int, int, void* stream)
{
    flush_deferred();
    run_phase1(Phase1{dvdx, dudy, hArea_u, hArea_v, nullptr, u, v, h, dyCv, dxCu, nullptr,
                      nullptr, areaT, n1, n2, is_l, ie_l, js_l, je_l, true, false},
               n3, stream);
}

extern "C" void launch_phase1b_ke_kernel(double* KE, double* u, double* v, double* dyCu,
                                         double* dxCv, double* areaT, int n1, int n2, int n3,
                                         int is_l, int ie_l, int js_l, int je_l, int, int, int,
                                         int, int, int, void* stream)
{
    flush_deferred();
    run_phase1(Phase1{nullptr, nullptr, nullptr, nullptr, KE, u, v, nullptr, nullptr, nullptr,
                      dyCu, dxCv, areaT, n1, n2, is_l, ie_l, js_l, je_l, false, true},
               n3, stream);
}

// relative/absolute vorticity, Ih_q and q on [is-1, ie] x [js-1, je] (:289-318)
extern "C" void launch_vorticity_pv_kernel(double* rel_vort, double* abs_vort, double* q,
                                           double* Ih_q, double* dvdx, double* dudy,
                                           double* hArea_u, double* hArea_v, double* Area_q,
                                           double* IareaBu, double* CoriolisBu,
                                           double* mask2dBu, int n1, int n2, int n3, int is_l,
                                           int ie_l, int js_l, int je_l, int, int, int, int,
                                           int, int, void* stream)
{
    flush_deferred();
    run_box(clip(Box{is_l - 1, ie_l, js_l - 1, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const size_t p = at3(i, j, k, n1, n2), p2 = at2(i, j, n1);
                const double rel = mask2dBu[p2] * (dvdx[p] - dudy[p]) * IareaBu[p2];
                const double absv = CoriolisBu[p2] + rel;
                const double ha = (hArea_u[p] + hArea_u[at3(i, j + 1, k, n1, n2)]) +
                                  (hArea_v[p] + hArea_v[at3(i + 1, j, k, n1, n2)]);
                const double ih = Area_q[p] / (ha + 1.0e-20);
                rel_vort[p] = rel;
                abs_vort[p] = absv;
                Ih_q[p] = ih;
                q[p] = absv * ih;
            });
}

// a, d on [is-1, ie] x [js, je]; b, c on [is, ie] x [js, je] (:323-352)
extern "C" void launch_arakawa_hsu90_coef_kernel(double* a, double* b, double* c, double* d,
                                                 double* q, int n1, int n2, int n3, int is_l,
                                                 int ie_l, int js_l, int je_l, int, int, int,
                                                 int, int, int, void* stream)
{
    flush_deferred();
    run_box(clip(Box{is_l - 1, ie_l, js_l, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const size_t p = at3(i, j, k, n1, n2);
                const double qs = q[at3(i, j - 1, k, n1, n2)];
                if (i >= is_l - 1) {
                    a[p] = (q[p] + (q[at3(i + 1, j, k, n1, n2)] + qs)) * kC1_12;
                    d[p] = ((q[p] + q[at3(i + 1, j - 1, k, n1, n2)]) + qs) * kC1_12;
                }
                if (i >= is_l) {
                    b[p] = (q[p] + (q[at3(i - 1, j, k, n1, n2)] + qs)) * kC1_12;
                    c[p] = ((q[p] + q[at3(i - 1, j - 1, k, n1, n2)]) + qs) * kC1_12;
                }
            });
}

// a(i-1), d(i-1), b(i), c(i) from the four q around (i-1/2, j-1/2) (:357-378)
extern "C" void launch_arakawa_lamb81_coef_kernel(double* a, double* b, double* c, double* d,
                                                  double* q, int n1, int n2, int n3, int is_l,
                                                  int ie_l, int js_l, int je_l, int, int, int,
                                                  int, int, int, void* stream)
{
    flush_deferred();
    run_box(clip(Box{is_l, ie_l, js_l, je_l}, n1, n2), n3, stream,
            [=] __device__(int i, int j, int k) {
                const double q00 = q[at3(i, j, k, n1, n2)];
                const double qmm = q[at3(i - 1, j - 1, k, n1, n2)];
                const double qm0 = q[at3(i - 1, j, k, n1, n2)];
                const double q0m = q[at3(i, j - 1, k, n1, n2)];
                const size_t pw = at3(i - 1, j, k, n1, n2), p = at3(i, j, k, n1, n2);
                a[pw] = (2.0 * (q00 + qmm) + (qm0 + q0m)) * kC1_24;
                d[pw] = ((q00 + qmm) + 2.0 * (qm0 + q0m)) * kC1_24;
                b[p] = ((q00 + qmm) + 2.0 * (qm0 + q0m)) * kC1_24;
                c[p] = (2.0 * (q00 + qmm) + (qm0 + q0m)) * kC1_24;
            });
}

// CAu on [is, ie-1] x [js, je], CAv on [is, ie] x [js, je-1] (:383-416)
extern "C" void launch_coriolis_sadourny_kernel(double* CAu, double* CAv, double* q, double* KE,
                                                double* uh, double* vh, double* IdxCu,
                                                double* IdyCv, int n1, int n2, int n3, int is_l,
                                                int ie_l, int js_l, int je_l, int, int, int, int,
                                                int, int, void* stream)
{
    flush_deferred();
    run_box(Box{is_l, ie_l, js_l, je_l}, n3, stream, [=] __device__(int i, int j, int k) {
        const size_t p = at3(i, j, k, n1, n2), p2 = at2(i, j, n1);
        if (i <= ie_l - 1) {
            const double KEx = (KE[at3(i + 1, j, k, n1, n2)] - KE[p]) * IdxCu[p2];
            const double n_ = q[p] * (vh[at3(i + 1, j, k, n1, n2)] + vh[p]);
            const double s_ = q[at3(i, j - 1, k, n1, n2)] *
                              (vh[at3(i, j - 1, k, n1, n2)] + vh[at3(i + 1, j - 1, k, n1, n2)]);
            CAu[p] = 0.25 * (n_ + s_) * IdxCu[p2] - KEx;
        }
        if (j <= je_l - 1) {
            const double KEy = (KE[at3(i, j + 1, k, n1, n2)] - KE[p]) * IdyCv[p2];
            const double w_ = q[at3(i - 1, j, k, n1, n2)] *
                              (uh[at3(i - 1, j, k, n1, n2)] + uh[at3(i - 1, j + 1, k, n1, n2)]);
            const double e_ = q[p] * (uh[p] + uh[at3(i, j + 1, k, n1, n2)]);
            CAv[p] = -0.25 * (w_ + e_) * IdyCv[p2] - KEy;
        }
    });
}

extern "C" void launch_coriolis_arakawa_kernel(double* CAu, double* CAv, double* a, double* b,
                                               double* c, double* d, double* KE, double* uh,
                                               double* vh, double* IdxCu, double* IdyCv, int n1,
                                               int n2, int n3, int is_l, int ie_l, int js_l,
                                               int je_l, int, int, int, int, int, int,
                                               void* stream)
{
    flush_deferred();
    run_box(Box{is_l, ie_l, js_l, je_l}, n3, stream, [=] __device__(int i, int j, int k) {
        const size_t p = at3(i, j, k, n1, n2), p2 = at2(i, j, n1);
        if (i <= ie_l - 1) {
            const double KEx = (KE[at3(i + 1, j, k, n1, n2)] - KE[p]) * IdxCu[p2];
            const double t1 = (a[p] * vh[at3(i + 1, j, k, n1, n2)]) +
                              (c[p] * vh[at3(i, j - 1, k, n1, n2)]);
            const double t2 = (b[p] * vh[p]) + (d[p] * vh[at3(i + 1, j - 1, k, n1, n2)]);
            CAu[p] = (t1 + t2) * IdxCu[p2] - KEx;
        }
        if (j <= je_l - 1) {
            const double KEy = (KE[at3(i, j + 1, k, n1, n2)] - KE[p]) * IdyCv[p2];
            const size_t pw = at3(i - 1, j, k, n1, n2), pn = at3(i, j + 1, k, n1, n2),
                         pwn = at3(i - 1, j + 1, k, n1, n2);
            const double t1 = (a[pw] * uh[pw]) + (c[pn] * uh[pn]);
            const double t2 = (b[p] * uh[p]) + (d[pwn] * uh[pwn]);
            CAv[p] = -(t1 + t2) * IdyCv[p2] - KEy;
        }
    });
}

// Sadourny acceleration with q and KE evaluated in place (:421-535)
extern "C" void launch_coriolis_fused_sadourny_kernel(
    double* CAu, double* CAv, double* u, double* v, double* h, double* uh, double* vh,
    double* dyCv, double* dxCu, double* dyCu, double* dxCv, double* areaT, double* IareaBu,
    double* CoriolisBu, double* mask2dBu, double* IdxCu, double* IdyCv, int n1, int n2, int n3,
    int is_l, int ie_l, int js_l, int je_l, int, int, int, int, int, int, void* stream)
{
    flush_deferred();
    run_box(Box{is_l, ie_l, js_l, je_l}, n3, stream, [=] __device__(int i, int j, int k) {
        const bool do_u = i <= ie_l - 1, do_v = j <= je_l - 1;
        if (!do_u && !do_v) return;
        const size_t p = at3(i, j, k, n1, n2), p2 = at2(i, j, n1);
        const double q0 = pv_at(u, v, h, dyCv, dxCu, areaT, IareaBu, CoriolisBu, mask2dBu, n1,
                                n2, i, j, k);
        const double ke0 = ke_at(u, v, dyCu, dxCv, areaT, n1, n2, i, j, k);
        if (do_u) {
            const double qs = pv_at(u, v, h, dyCv, dxCu, areaT, IareaBu, CoriolisBu, mask2dBu,
                                    n1, n2, i, j - 1, k);
            const double KEx = (ke_at(u, v, dyCu, dxCv, areaT, n1, n2, i + 1, j, k) - ke0) *
                               IdxCu[p2];
            const double n_ = q0 * (vh[at3(i + 1, j, k, n1, n2)] + vh[p]);
            const double s_ = qs * (vh[at3(i, j - 1, k, n1, n2)] + vh[at3(i + 1, j - 1, k, n1, n2)]);
            CAu[p] = 0.25 * (n_ + s_) * IdxCu[p2] - KEx;
        }
        if (do_v) {
            const double qw = pv_at(u, v, h, dyCv, dxCu, areaT, IareaBu, CoriolisBu, mask2dBu,
                                    n1, n2, i - 1, j, k);
            const double KEy = (ke_at(u, v, dyCu, dxCv, areaT, n1, n2, i, j + 1, k) - ke0) *
                               IdyCv[p2];
            const double w_ = qw * (uh[at3(i - 1, j, k, n1, n2)] + uh[at3(i - 1, j + 1, k, n1, n2)]);
            const double e_ = q0 * (uh[p] + uh[at3(i, j + 1, k, n1, n2)]);
            CAv[p] = -0.25 * (w_ + e_) * IdyCv[p2] - KEy;
        }
    });
}
