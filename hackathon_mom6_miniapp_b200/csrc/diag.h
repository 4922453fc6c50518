// diag.h -- the diagnostics module of the mini-app (mom6_diag.F90) for
// device-resident fields, and its raw binary dump format.
//
// A DiagCtrl mirrors diag_ctrl: fields are registered with an output mode
// (none / stats / file / both) and return an id (> 0 when active); posting a
// 2-D or 3-D device field counts a call, prints min/max/mean/rms of its
// computational domain when the mode asks for stats (the reference's line,
// values in Fortran ES14.6) and, every output_freq-th call, writes the
// computational domain to <output_dir>/<name><call_count, 6 digits>.bin: the
// dimensions as 32-bit integers (ni, nj[, nk]) followed by the values as
// 64-bit floats in column-major order (mom6_diag.F90:362-431).  The vertical
// product sums of post_product_sum_u/v run on the GPU in the serial loop's
// per-column order into one persistent device work array, which keeps the
// values of the points a sum does not cover (as work_2d does).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "kernels.h"

namespace mom6b {

enum { kDiagNone = 0, kDiagStats = 1, kDiagFile = 2, kDiagBoth = 3 };
constexpr int kDiagMax = 100;   // MAX_DIAGS

struct DiagField {
    std::string name, long_name, units, position;
    int output_mode = kDiagNone;
    int ndims = 0;
    double stats[4] = {0.0, 0.0, 0.0, 0.0};   // of the last post
    bool posted = false;
};

class DiagCtrl {
public:
    ~DiagCtrl();
    // diag_init: D gives the data and computational domains; work_2d is
    // allocated on the current device and zeroed.
    int init(const Dims& D, const std::string& output_dir, int output_freq, cudaStream_t s);
    // register_diag_field: the id (1..kDiagMax), or -1 for kDiagNone or when
    // kDiagMax fields are registered already.
    int register_field(const std::string& name, const std::string& long_name,
                       const std::string& units, int ndims, const std::string& position,
                       int output_mode);
    // post_data_2d / post_data_3d of a device field ((n1, n2) or (n1, n2, nk));
    // id <= 0 is a no-op.  Synchronizes s.
    int post_2d(int id, const double* field, cudaStream_t s);
    int post_3d(int id, const double* field, cudaStream_t s);
    // post_product_sum_u / _v: work_2d = sum_k a b over the u (v) points of
    // the computational domain, then post_2d(work_2d).
    int post_product_sum(int id, const double* a, const double* b, bool u_points,
                         cudaStream_t s);
    const DiagField* field(int id) const;
    bool initialized() const { return init_; }
    int num_diags() const { return (int)fields_.size(); }
    int total_calls() const { return total_calls_; }
    int call_count() const { return call_count_; }
    const std::string& last_file() const { return last_file_; }

private:
    int post(int id, const double* field, int ndims, cudaStream_t s);
    bool init_ = false;
    Dims D_{};
    std::string dir_ = "./";
    int freq_ = 1;
    int call_count_ = 0, total_calls_ = 0;
    std::vector<DiagField> fields_;
    double* work_ = nullptr;          // device work_2d (n1, n2)
    std::vector<double> host_;        // computational domain of the posted field
    std::string last_file_;
};

// The reference's binary dump: dims as int32 then float64 values.  nk = 0
// writes a 2-D file.  0 on success.
int diag_write_bin(const std::string& path, const double* values, int ni, int nj, int nk);
// Reads a dump whose header must equal (ni, nj[, nk]); 0 on success, -1 when
// the file cannot be read, -2 on a header mismatch.
int diag_read_bin(const std::string& path, double* values, int ni, int nj, int nk);
// Fortran ES14.6 edit of one value (the stats line of post_data).
std::string fortran_es14_6(double x);

// Device helpers (diag.cu): the product sum over [ilo, ihi] x [jlo, jhi] into
// work, and the driver's KE (compute_and_post_KE) and mass
// (compute_and_post_mass) on the computational domain.
cudaError_t launch_diag_product_sum(const Dims& D, const double* a, const double* b,
                                    double* work, int ilo, int ihi, int jlo, int jhi,
                                    cudaStream_t s);
cudaError_t launch_diag_KE(const Dims& D, const double* u, const double* v, double* KE,
                           cudaStream_t s);
cudaError_t launch_diag_mass(const Dims& D, const double* h, double* mass, cudaStream_t s);

} // namespace mom6b
