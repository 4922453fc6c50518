// abi_helpers.cu -- the runtime helpers of the reference ABI.
//
// cuda_helpers.cu:8-48 of the reference: device selection, synchronisation,
// allocation and blocking copies that the Fortran wrappers use to own every
// device array (mom6_cuda_c_common.F90:74-128).  Return values are the CUDA
// error codes as int; cuda_malloc_c returns NULL on failure (the Fortran
// gpu_alloc stops on NULL).  The copies are blocking and ordered after all
// work on the legacy default stream, where the wrappers enqueue every
// launch_* call.  Each first replays an open barotropic record
// (abi_barotropic.cu), so whatever it observes follows the reference
// sequence.
#include <cuda_runtime.h>

#include "../../include/mom6_cuda_c.h"
#include "abi_common.cuh"

using mom6b::abi::flush_deferred;

extern "C" int cuda_set_device_c(int device)
{
    flush_deferred();
    return (int)cudaSetDevice(device);
}

extern "C" int cuda_device_synchronize_c(void)
{
    flush_deferred();
    return (int)cudaDeviceSynchronize();
}

extern "C" void* cuda_malloc_c(size_t bytes)
{
    flush_deferred();
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        (void)cudaGetLastError();  // do not leave the error sticky for the next call
        return nullptr;
    }
    return p;
}

extern "C" void cuda_free_c(void* ptr)
{
    flush_deferred();
    if (ptr) (void)cudaFree(ptr);
}

extern "C" int cuda_memcpy_h2d_c(void* dst, const void* src, size_t bytes)
{
    flush_deferred();
    return (int)cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
}

extern "C" int cuda_memcpy_d2h_c(void* dst, const void* src, size_t bytes)
{
    flush_deferred();
    return (int)cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
}

extern "C" int cuda_memcpy_d2d_c(void* dst, const void* src, size_t bytes)
{
    flush_deferred();
    return (int)cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToDevice);
}

extern "C" int cuda_memset_c(void* ptr, int value, size_t bytes)
{
    flush_deferred();
    return (int)cudaMemset(ptr, value, bytes);
}
