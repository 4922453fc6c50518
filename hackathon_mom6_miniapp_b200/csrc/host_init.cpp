// host_init.cpp -- grid metrics and initial state, built on the host.
//
// Grid: init_ocean_grid (mom6_types.F90:130-258) -- uniform spacing, 1-based
// data domain [1, ni+2] x [1, nj+2], compute domain [4, ni-1] x [4, nj-1].
// Derived metrics are those of hor_visc_init (mom6_hor_visc_serial.F90:209-268),
// coriolis_init (mom6_coriolis_serial.F90:74-80) and barotropic_init
// (mom6_barotropic_serial.F90:106-133), evaluated with the same expressions.
// Initial state: REF = initialize_state/initialize_forces_visc of
// rk2_serial_driver.F90:466-542; CFG = the seeded beta-plane construction
// (Philox4x32-10 normals, see philox_normal below).
#include "host_init.h"

#include <cmath>
#include <cstring>

namespace mom6b {

static constexpr double kOmega = 7.2921e-5;
static constexpr double kPiRef = 3.14159265358979323846;
static constexpr double kEarthRadius = 6.371e6;

// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, SC'11): 10 rounds of the
// published multiply-xor round function with Weyl key increments.
static void philox4x32_10(uint32_t c[4], uint32_t key0, uint32_t key1)
{
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ key0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ key1;
        uint32_t n3 = (uint32_t)p0;
        c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
        key0 += 0x9E3779B9u;
        key1 += 0xBB67AE85u;
    }
}

// Standard normal deviate for (seed, stream, index): two 53-bit uniforms from
// one Philox block, Box-Muller.
double philox_normal(uint64_t seed, uint32_t stream, uint64_t index)
{
    uint32_t c[4] = {(uint32_t)index, (uint32_t)(index >> 32), stream, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint64_t a = (((uint64_t)c[0] << 32) | c[1]) >> 11;
    uint64_t b = (((uint64_t)c[2] << 32) | c[3]) >> 11;
    double u1 = (double)a * 0x1.0p-53 + 0x1.0p-54;
    double u2 = (double)b * 0x1.0p-53;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

HostGrid::HostGrid(const mom6b_config& c) : cfg(c)
{
    ni = c.ni; nj = c.nj; nk = c.nk;
    gni = c.ni_global > 0 ? c.ni_global : c.ni;
    gnj = c.nj_global > 0 ? c.nj_global : c.nj;
    ioff = c.i_offset; joff = c.j_offset;
    isd = 1; ied = ni + 2; jsd = 1; jed = nj + 2;
    is = isd + 3; ie = ied - 3; js = jsd + 3; je = jed - 3;
    n1 = ied; n2 = jed;
    plane = (size_t)n1 * n2;
}

void HostGrid::build()
{
    const size_t n = plane;
    auto mk = [&](std::vector<double>& v) { v.assign(n, 0.0); };
    for (auto* v : {&IareaT, &areaT, &dxT, &dyT, &IdxT, &IdyT, &dxCu, &dyCu, &dy_Cu,
                    &IdxCu, &IdyCu, &dxCv, &dyCv, &IdxCv, &IdyCv, &IareaBu, &areaBu,
                    &CoriolisBu, &IareaCu, &IareaCv, &dxBu, &dyBu, &IdxBu, &IdyBu,
                    &mask2dT, &mask2dBu, &mask2dCu, &mask2dCv, &Area_q, &DX_dyT,
                    &DY_dxT, &DX_dyBu, &DY_dxBu, &dx2h, &dy2h, &dx2q, &dy2q, &red_xx,
                    &red_xy, &Kh_xx, &Kh_xy, &Datu, &Datv, &gtot_E, &gtot_W, &gtot_N,
                    &gtot_S, &bt_rem_u, &bt_rem_v, &taux, &tauy})
        mk(*v);
    f_4_u.assign(4 * n, 0.0);
    f_4_v.assign(4 * n, 0.0);

    const double dx_m = cfg.dx_km * 1000.0;
    dx = dx_m;
    const double f0 = 2.0 * kOmega * std::sin(cfg.lat_deg * kPiRef / 180.0);
    const double beta = 2.0 * kOmega * std::cos(cfg.lat_deg * kPiRef / 180.0) / kEarthRadius;
    const double Ly = (double)((gnj - 1) - js + 1) * dx_m;
    for (int j = jsd; j <= jed; ++j)
        for (int i = isd; i <= ied; ++i) {
            size_t p = at(i, j);
            areaT[p] = dx_m * dx_m;
            IareaT[p] = 1.0 / (dx_m * dx_m);
            dxT[p] = dx_m; dyT[p] = dx_m;
            IdxT[p] = 1.0 / dx_m; IdyT[p] = 1.0 / dx_m;
            dxCu[p] = dx_m; dyCu[p] = dx_m; dy_Cu[p] = dx_m;
            IdxCu[p] = 1.0 / dx_m; IdyCu[p] = 1.0 / dx_m;
            dxCv[p] = dx_m; dyCv[p] = dx_m;
            IdxCv[p] = 1.0 / dx_m; IdyCv[p] = 1.0 / dx_m;
            areaBu[p] = dx_m * dx_m;
            IareaBu[p] = 1.0 / (dx_m * dx_m);
            IareaCu[p] = 1.0 / (dx_m * dx_m);
            IareaCv[p] = 1.0 / (dx_m * dx_m);
            dxBu[p] = dx_m; dyBu[p] = dx_m;
            IdxBu[p] = 1.0 / dx_m; IdyBu[p] = 1.0 / dx_m;
            mask2dT[p] = 1.0; mask2dBu[p] = 1.0; mask2dCu[p] = 1.0; mask2dCv[p] = 1.0;
            if (cfg.init_mode == MOM6B_INIT_REF) {
                CoriolisBu[p] = f0 + beta * ((double)(j + joff - 1 - gnj / 2) - 0.5) * dx_m;
            } else {
                double yq = (double)(j + joff - js + 1) * dx_m;
                CoriolisBu[p] = 1.0e-4 + 2.0e-11 * (yq - 0.5 * Ly);
            }
        }
    // coriolis_init: Area_q on [isd, ied-1] x [jsd, jed-1]
    for (int j = jsd; j <= jed - 1; ++j)
        for (int i = isd; i <= ied - 1; ++i)
            Area_q[at(i, j)] = (areaT[at(i, j)] + areaT[at(i + 1, j + 1)]) +
                               (areaT[at(i + 1, j)] + areaT[at(i, j + 1)]);
    // hor_visc_init metric products; Kh = max(Kh_bg, Kh_bg_min = 0)
    for (int j = jsd; j <= jed; ++j)
        for (int i = isd; i <= ied; ++i) {
            size_t p = at(i, j);
            dx2h[p] = dxT[p] * dxT[p];
            dy2h[p] = dyT[p] * dyT[p];
            dx2q[p] = dxBu[p] * dxBu[p];
            dy2q[p] = dyBu[p] * dyBu[p];
            DX_dyT[p] = dxT[p] * IdyT[p];
            DY_dxT[p] = dyT[p] * IdxT[p];
            DX_dyBu[p] = dxBu[p] * IdyBu[p];
            DY_dxBu[p] = dyBu[p] * IdxBu[p];
            red_xx[p] = 1.0; red_xy[p] = 1.0;
            Kh_xx[p] = cfg.Kh > 0.0 ? cfg.Kh : 0.0;
            Kh_xy[p] = cfg.Kh > 0.0 ? cfg.Kh : 0.0;
        }
    // barotropic_init
    const double depth = 4000.0;
    for (int j = jsd; j <= jed; ++j)
        for (int i = isd; i <= ied; ++i) {
            size_t p = at(i, j);
            Datu[p] = depth * dyCu[p];
            Datv[p] = depth * dxCv[p];
            gtot_E[p] = kGEarthHost; gtot_W[p] = kGEarthHost;
            gtot_N[p] = kGEarthHost; gtot_S[p] = kGEarthHost;
            bt_rem_u[p] = 0.999; bt_rem_v[p] = 0.999;
            double fq = CoriolisBu[p];
            for (int cc = 0; cc < 4; ++cc) {
                f_4_u[4 * p + cc] = 0.25 * fq;
                f_4_v[4 * p + cc] = 0.25 * fq;
            }
        }
    // forcing: wind stress and bottom-layer Rayleigh drag
    for (int j = jsd; j <= jed; ++j)
        for (int i = isd; i <= ied; ++i) {
            taux[at(i, j)] = 0.1 * std::sin((double)(j + joff - 1) / (double)gnj * pi_init);
            tauy[at(i, j)] = 0.0;
        }
}

void HostGrid::initial_state(std::vector<double>& u, std::vector<double>& v,
                             std::vector<double>& h0, std::vector<double>& eta,
                             std::vector<double>& ubt, std::vector<double>& vbt) const
{
    const size_t n3 = plane * (size_t)nk;
    u.assign(n3, 0.0); v.assign(n3, 0.0); h0.assign(n3, 0.0);
    eta.assign(plane, 0.0); ubt.assign(plane, 0.0); vbt.assign(plane, 0.0);
    if (cfg.init_mode == MOM6B_INIT_REF) {
        const double total_depth = 4000.0;
        for (int k = 1; k <= nk; ++k)
            for (int j = jsd; j <= jed; ++j)
                for (int i = isd; i <= ied; ++i) {
                    size_t p = at(i, j, k);
                    h0[p] = total_depth / (double)nk +
                            10.0 * std::sin((double)(i + ioff - 1) / (double)gni * pi_init) *
                                std::cos((double)(j + joff - 1) / (double)gnj * pi_init) *
                                std::exp(-(double)k / 20.0);
                    u[p] = 0.1 * std::sin((double)(j + joff - 1) / (double)gnj * pi_init * 2.0) *
                           std::exp(-(double)k / 30.0);
                    v[p] = 0.1 * std::cos((double)(i + ioff - 1) / (double)gni * pi_init * 2.0) *
                           std::exp(-(double)k / 30.0);
                }
        for (int j = jsd; j <= jed; ++j)
            for (int i = isd; i <= ied; ++i) {
                size_t p = at(i, j);
                eta[p] = 0.5 * std::sin((double)(i + ioff - 1) / (double)gni * pi_init * 2.0) *
                         std::cos((double)(j + joff - 1) / (double)gnj * pi_init * 2.0);
                ubt[p] = 0.05 * std::sin((double)(j + joff - 1) / (double)gnj * pi_init);
                vbt[p] = 0.05 * std::cos((double)(i + ioff - 1) / (double)gni * pi_init);
            }
    } else {
        const double hbar = 4000.0 / (double)nk;
        for (int k = 1; k <= nk; ++k)
            for (int j = jsd; j <= jed; ++j)
                for (int i = isd; i <= ied; ++i) {
                    size_t p = at(i, j, k);
                    // the global point's Philox counter
                    uint64_t idx = ((uint64_t)(k - 1) * (uint64_t)(gnj + 2) +
                                    (uint64_t)(j + joff - 1)) * (uint64_t)(gni + 2) +
                                   (uint64_t)(i + ioff - 1);
                    double hv = hbar * (1.0 + 0.01 * philox_normal(cfg.seed, 1u, idx));
                    if (hv < 0.01 * hbar) hv = 0.01 * hbar;
                    h0[p] = hv;
                    u[p] = 0.05 * philox_normal(cfg.seed, 2u, idx);
                    v[p] = 0.05 * philox_normal(cfg.seed, 3u, idx);
                }
        const double Lx = (double)((gni - 1) - is + 1) * dx;
        const double Ly = (double)((gnj - 1) - js + 1) * dx;
        const double R = 200.0e3;
        for (int j = jsd; j <= jed; ++j)
            for (int i = isd; i <= ied; ++i) {
                double x = ((double)(i + ioff - is) + 0.5) * dx - 0.5 * Lx;
                double y = ((double)(j + joff - js) + 0.5) * dx - 0.5 * Ly;
                eta[at(i, j)] = 0.1 * std::exp(-(x * x + y * y) / (R * R));
            }
    }
}

void HostGrid::rayleigh(std::vector<double>& Ray_u, std::vector<double>& Ray_v) const
{
    const size_t n3 = plane * (size_t)nk;
    Ray_u.assign(n3, 0.0);
    Ray_v.assign(n3, 0.0);
    for (int j = jsd; j <= jed; ++j)
        for (int i = isd; i <= ied; ++i) {
            Ray_u[at(i, j, nk)] = 1.0e-4;
            Ray_v[at(i, j, nk)] = 1.0e-4;
        }
}

} // namespace mom6b
