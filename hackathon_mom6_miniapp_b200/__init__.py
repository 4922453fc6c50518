"""B200-native split RK2 step of the MOM6 mini-app.

The computation lives in libmom6b.so (hand-written sm_100a CUDA kernels behind
a C ABI, see include/mom6b.h and include/mom6_cuda_c.h).  This package is the
thin Python host mirror used by tests and benchmarks: it loads the library
with ctypes and moves numpy arrays across the boundary.  There is no CPU
fallback: every entry point raises if the CUDA library cannot be loaded.
"""
from ._lib import (Model, Ensemble, Mlp, CudaCDriver, MixedNotBuilt, Mom6bError, FIELDS,
                   FIELDS_3D, INIT_CFG, INIT_REF, FP64, MIXED, TUNING_KEYS, library,
                   library_path, make_config, abi_set_deferral, HaloGroup, subdomain_config)

__all__ = ["Model", "Ensemble", "Mlp", "CudaCDriver", "Mom6bError", "MixedNotBuilt", "FIELDS",
           "FIELDS_3D", "INIT_CFG", "INIT_REF", "FP64", "MIXED", "TUNING_KEYS", "library",
           "library_path", "make_config", "abi_set_deferral", "HaloGroup", "subdomain_config"]
