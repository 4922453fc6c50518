// diag.cu -- the diagnostics module (mom6_diag.F90) for device fields: the
// GPU product sums and driver diagnostics, the host-side control, the stats
// line and the raw binary dumps.  Built without FMA contraction: every sum
// runs in the serial loop's order, so the posted fields equal the serial
// driver's bit for bit.
#include "diag.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace mom6b {

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
// post_product_sum_u/v (mom6_diag.F90:274-334): one thread per point, the
// layers summed in order 1..nk from zero.
__global__ void k_diag_product_sum(Dims D, const double* __restrict__ a,
                                   const double* __restrict__ b, double* __restrict__ work,
                                   int ilo, int ihi, int jlo, int jhi)
{
    const int i = ilo + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = jlo + (int)blockIdx.y;
    if (i > ihi || j > jhi) return;
    const size_t p = (size_t)(j - 1) * D.n1 + (size_t)(i - 1);
    double w = 0.0;
    for (int k = 1; k <= D.nk; ++k) {
        const size_t o = (size_t)(k - 1) * (size_t)D.plane + p;
        w = w + a[o] * b[o];
    }
    work[p] = w;
}

// compute_and_post_KE (rk2_serial_driver.F90:664-693) on the computational
// domain: KE = 0.5 (0.5 (u(i)^2 + u(i-1)^2) + 0.5 (v(j)^2 + v(j-1)^2)).
__global__ void k_diag_KE(Dims D, const double* __restrict__ u, const double* __restrict__ v,
                          double* __restrict__ KE)
{
    const int i = D.is + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = D.js + (int)blockIdx.y;
    const int k = 1 + (int)blockIdx.z;
    if (i > D.ie || j > D.je) return;
    const size_t o = (size_t)(k - 1) * (size_t)D.plane + (size_t)(j - 1) * D.n1 + (size_t)(i - 1);
    const double u0 = u[o], u1 = u[o - 1], v0 = v[o], v1 = v[o - D.n1];
    KE[o] = 0.5 * (0.5 * (u0 * u0 + u1 * u1) + 0.5 * (v0 * v0 + v1 * v1));
}

// compute_and_post_mass (:695-728): the layer thicknesses summed in order.
__global__ void k_diag_mass(Dims D, const double* __restrict__ h, double* __restrict__ mass)
{
    const int i = D.is + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int j = D.js + (int)blockIdx.y;
    if (i > D.ie || j > D.je) return;
    const size_t p = (size_t)(j - 1) * D.n1 + (size_t)(i - 1);
    double w = 0.0;
    for (int k = 1; k <= D.nk; ++k) w = w + h[(size_t)(k - 1) * (size_t)D.plane + p];
    mass[p] = w;
}

cudaError_t launch_diag_product_sum(const Dims& D, const double* a, const double* b,
                                    double* work, int ilo, int ihi, int jlo, int jhi,
                                    cudaStream_t s)
{
    if (ihi < ilo || jhi < jlo) return cudaSuccess;
    dim3 grid((ihi - ilo + 1 + 127) / 128, jhi - jlo + 1, 1);
    k_diag_product_sum<<<grid, 128, 0, s>>>(D, a, b, work, ilo, ihi, jlo, jhi);
    return cudaGetLastError();
}

cudaError_t launch_diag_KE(const Dims& D, const double* u, const double* v, double* KE,
                           cudaStream_t s)
{
    dim3 grid((D.ie - D.is + 1 + 127) / 128, D.je - D.js + 1, D.nk);
    k_diag_KE<<<grid, 128, 0, s>>>(D, u, v, KE);
    return cudaGetLastError();
}

cudaError_t launch_diag_mass(const Dims& D, const double* h, double* mass, cudaStream_t s)
{
    dim3 grid((D.ie - D.is + 1 + 127) / 128, D.je - D.js + 1, 1);
    k_diag_mass<<<grid, 128, 0, s>>>(D, h, mass);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// format helpers
// ---------------------------------------------------------------------------
std::string fortran_es14_6(double x)
{
    char b[64];
    if (std::isnan(x)) {
        std::snprintf(b, sizeof(b), "%14s", "NaN");
        return b;
    }
    if (std::isinf(x)) {
        std::snprintf(b, sizeof(b), "%14s", x > 0 ? "Infinity" : "-Infinity");
        return b;
    }
    std::snprintf(b, sizeof(b), "%.6E", x);
    std::string t = b;
    // an exponent of three digits is written without its letter: 1.000000+100
    const size_t e = t.find('E');
    if (e != std::string::npos && t.size() - e - 2 >= 3) t.erase(e, 1);
    if (t.size() < 14) t.insert(0, 14 - t.size(), ' ');
    return t;
}

int diag_write_bin(const std::string& path, const double* values, int ni, int nj, int nk)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return -1;
    int32_t hdr[3] = {ni, nj, nk};
    const size_t nh = nk > 0 ? 3 : 2;
    const size_t n = (size_t)ni * nj * (nk > 0 ? nk : 1);
    bool ok = std::fwrite(hdr, sizeof(int32_t), nh, f) == nh &&
              std::fwrite(values, sizeof(double), n, f) == n;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? 0 : -1;
}

int diag_read_bin(const std::string& path, double* values, int ni, int nj, int nk)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return -1;
    int32_t hdr[3] = {0, 0, 0};
    const size_t nh = nk > 0 ? 3 : 2;
    if (std::fread(hdr, sizeof(int32_t), nh, f) != nh) { std::fclose(f); return -1; }
    if (hdr[0] != ni || hdr[1] != nj || (nk > 0 && hdr[2] != nk)) { std::fclose(f); return -2; }
    const size_t n = (size_t)ni * nj * (nk > 0 ? nk : 1);
    const bool ok = std::fread(values, sizeof(double), n, f) == n;
    std::fclose(f);
    return ok ? 0 : -1;
}

// ---------------------------------------------------------------------------
// DiagCtrl
// ---------------------------------------------------------------------------
DiagCtrl::~DiagCtrl()
{
    if (work_) cudaFree(work_);
}

int DiagCtrl::init(const Dims& D, const std::string& output_dir, int output_freq,
                   cudaStream_t s)
{
    if (init_) return 0;   // diag_init returns early when initialized
    if (output_freq < 1) return -2;   // mod(call_count, output_freq) needs a positive frequency
    D_ = D;
    dir_ = output_dir;
    freq_ = output_freq;
    call_count_ = total_calls_ = 0;
    fields_.clear();
    if (cudaMalloc(&work_, (size_t)D.plane * sizeof(double)) != cudaSuccess) return -1;
    if (cudaMemsetAsync(work_, 0, (size_t)D.plane * sizeof(double), s) != cudaSuccess) return -1;
    init_ = true;
    return 0;
}

int DiagCtrl::register_field(const std::string& name, const std::string& long_name,
                             const std::string& units, int ndims, const std::string& position,
                             int output_mode)
{
    if (output_mode == kDiagNone) return -1;
    if ((int)fields_.size() >= kDiagMax) {
        std::printf("WARNING: Maximum diagnostics reached: %4d\n", kDiagMax);
        std::fflush(stdout);
        return -1;
    }
    DiagField f;
    // character(len=32/64/16/4) components keep at most that many characters
    f.name = name.substr(0, 32);
    f.long_name = long_name.substr(0, 64);
    f.units = units.substr(0, 16);
    f.position = position.substr(0, 4);
    f.ndims = ndims;
    f.output_mode = output_mode;
    fields_.push_back(f);
    return (int)fields_.size();
}

const DiagField* DiagCtrl::field(int id) const
{
    if (id <= 0 || id > (int)fields_.size()) return nullptr;
    return &fields_[(size_t)id - 1];
}

int DiagCtrl::post_2d(int id, const double* field, cudaStream_t s) { return post(id, field, 2, s); }
int DiagCtrl::post_3d(int id, const double* field, cudaStream_t s) { return post(id, field, 3, s); }

int DiagCtrl::post_product_sum(int id, const double* a, const double* b, bool u_points,
                               cudaStream_t s)
{
    if (id <= 0 || !init_) return 0;
    const int ihi = u_points ? D_.ie - 1 : D_.ie;
    const int jhi = u_points ? D_.je : D_.je - 1;
    if (launch_diag_product_sum(D_, a, b, work_, D_.is, ihi, D_.js, jhi, s) != cudaSuccess)
        return -1;
    return post(id, work_, 2, s);
}

int DiagCtrl::post(int id, const double* field, int ndims, cudaStream_t s)
{
    if (id <= 0 || !init_) return 0;
    DiagField* F = id <= (int)fields_.size() ? &fields_[(size_t)id - 1] : nullptr;
    if (!F) return -1;
    ++total_calls_;
    ++call_count_;
    const int ni = D_.ie - D_.is + 1, nj = D_.je - D_.js + 1;
    const int nk = ndims == 3 ? D_.nk : 1;
    host_.resize((size_t)ni * nj * nk);
    // the computational domain, layer by layer, column-major
    for (int k = 0; k < nk; ++k) {
        const double* src = field + (size_t)k * (size_t)D_.plane +
                            (size_t)(D_.js - 1) * D_.n1 + (size_t)(D_.is - 1);
        if (cudaMemcpy2DAsync(host_.data() + (size_t)k * ni * nj, (size_t)ni * sizeof(double),
                              src, (size_t)D_.n1 * sizeof(double), (size_t)ni * sizeof(double),
                              (size_t)nj, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return -1;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    // statistics in the serial loop's order (k, then j, then i)
    double fmin = 1.7976931348623157e308, fmax = -1.7976931348623157e308;
    double fmean = 0.0, frms = 0.0;
    long long cnt = 0;
    for (size_t q = 0; q < host_.size(); ++q) {
        const double x = host_[q];
        fmin = x < fmin ? x : fmin;
        fmax = x > fmax ? x : fmax;
        fmean = fmean + x;
        frms = frms + x * x;
        ++cnt;
    }
    if (cnt > 0) {
        fmean = fmean / (double)cnt;
        frms = std::sqrt(frms / (double)cnt);
    }
    F->stats[0] = fmin; F->stats[1] = fmax; F->stats[2] = fmean; F->stats[3] = frms;
    F->posted = true;
    if (F->output_mode & kDiagStats) {
        std::string line = "  Diag: " + F->name + " min/max/mean/rms: " + fortran_es14_6(fmin) +
                           fortran_es14_6(fmax) + fortran_es14_6(fmean) + fortran_es14_6(frms);
        std::printf("%s\n", line.c_str());
        std::fflush(stdout);
    }
    if ((F->output_mode & kDiagFile) && (call_count_ % freq_) == 0) {
        char num[16];
        if (call_count_ <= 999999) std::snprintf(num, sizeof(num), "%06d", call_count_);
        else std::snprintf(num, sizeof(num), "******");
        last_file_ = dir_ + "/" + F->name + num + ".bin";
        if (diag_write_bin(last_file_, host_.data(), ni, nj, ndims == 3 ? D_.nk : 0) != 0) {
            std::printf("WARNING: Could not open file: %s\n", last_file_.c_str());
            std::fflush(stdout);
        }
    }
    return 0;
}

} // namespace mom6b
