// k_tendency.cu -- the FP64 instantiation of the fused momentum tendency
// (tendency_impl.cuh), compiled without FMA contraction so that it equals
// the serial Fortran bit for bit.
#include "tendency_impl.cuh"

namespace mom6b {

cudaError_t launch_tendency(const Dims& D, const Metrics& M, const UniMetrics& U,
                            const double* uin, const double* vin, const double* h,
                            const double* ubase, const double* vbase, double* uout,
                            double* vout, double coef, double h_neglect, cudaStream_t s,
                            double* diffu, double* diffv, int scheme, bool ext_visc,
                            int* status)
{
    return launch_tendency_t<double>(D, M, U, uin, vin, h, ubase, vbase, uout, vout, coef,
                                     h_neglect, s, diffu, diffv, scheme, ext_visc, status);
}

} // namespace mom6b
