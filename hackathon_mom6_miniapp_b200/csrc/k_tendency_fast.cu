// k_tendency_fast.cu -- the fast FP64 instantiation of the fused momentum
// tendency (tendency_impl.cuh with FAST), built with FMA contraction and with
// quotients by Newton-Raphson-refined reciprocals; within 1e-12 relative L2
// of the exact form (k_tendency.cu), tested.  Sadourny scheme without the
// diagnostic outputs (the other forms run the exact kernel).
#include "tendency_impl.cuh"

namespace mom6b {

cudaError_t launch_tendency_fast(const Dims& D, const Metrics& M, const UniMetrics& U,
                                 const double* uin, const double* vin, const double* h,
                                 const double* ubase, const double* vbase, double* uout,
                                 double* vout, double coef, double h_neglect, cudaStream_t s,
                                 int* status)
{
    return launch_tendency_t<double, true>(D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef,
                                           h_neglect, s, nullptr, nullptr, 1, false, status);
}

} // namespace mom6b
