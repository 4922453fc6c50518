// host_init.h -- host-side grid and initial-state construction.
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/mom6b.h"

namespace mom6b {

constexpr double kGEarthHost = 9.80;  // G_EARTH, mom6_types.F90:80

double philox_normal(uint64_t seed, uint32_t stream, uint64_t index);

struct HostGrid {
    mom6b_config cfg;
    int ni, nj, nk, n1, n2;
    // a subdomain's global ni, nj and compute-domain offsets (the whole
    // domain: ni, nj, 0, 0); positions are evaluated at the global indices
    int gni, gnj, ioff, joff;
    int isd, ied, jsd, jed, is, ie, js, je;
    size_t plane;
    double dx = 0.0;
    // pi in the analytic initial state and wind stress: 3.14159 in
    // rk2_serial_driver.F90:477-530, PI (mom6_types.F90:83) in rk2_cuda_c_driver
    double pi_init = 3.14159;

    std::vector<double> IareaT, areaT, dxT, dyT, IdxT, IdyT, dxCu, dyCu, dy_Cu,
        IdxCu, IdyCu, dxCv, dyCv, IdxCv, IdyCv, IareaBu, areaBu, CoriolisBu,
        IareaCu, IareaCv, dxBu, dyBu, IdxBu, IdyBu, mask2dT, mask2dBu, mask2dCu,
        mask2dCv;
    std::vector<double> Area_q, DX_dyT, DY_dxT, DX_dyBu, DY_dxBu, dx2h, dy2h,
        dx2q, dy2q, red_xx, red_xy, Kh_xx, Kh_xy;
    std::vector<double> Datu, Datv, gtot_E, gtot_W, gtot_N, gtot_S, f_4_u, f_4_v,
        bt_rem_u, bt_rem_v, taux, tauy;

    explicit HostGrid(const mom6b_config& c);
    void build();
    void initial_state(std::vector<double>& u, std::vector<double>& v,
                       std::vector<double>& h0, std::vector<double>& eta,
                       std::vector<double>& ubt, std::vector<double>& vbt) const;
    void rayleigh(std::vector<double>& Ray_u, std::vector<double>& Ray_v) const;

    size_t at(int i, int j) const { return (size_t)(j - 1) * n1 + (size_t)(i - 1); }
    size_t at(int i, int j, int k) const { return (size_t)(k - 1) * plane + at(i, j); }
};

} // namespace mom6b
