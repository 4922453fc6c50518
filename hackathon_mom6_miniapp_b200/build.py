"""Build libmom6b.so in-tree with nvcc for sm_100a.

Every CUDA source is compiled with
    -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo --fmad=false
(no FMA contraction: the exact FP64 kernels reproduce the serial reference's
roundings) except FMA_SOURCES -- the mixed form, the ensemble, the network
and the fast FP64 kernels -- which contract multiply-adds; all are linked
into hackathon_mom6_miniapp_b200/libmom6b.so.  Host C++ is compiled with
-ffp-contract=off.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmom6b.so")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "--extended-lambda",
                   "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-O3"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-Wall"]

CU_SOURCES = ["k_tendency.cu", "k_vertvisc.cu", "k_continuity.cu", "k_btstep.cu",
              "mom6b_api.cu", "abi_helpers.cu", "abi_barotropic.cu", "abi_hor_visc.cu",
              "abi_vert_visc.cu", "abi_coriolis.cu", "abi_continuity.cu",
              "cudac_driver.cu", "k_mixed.cu", "k_ensemble.cu", "k_mlp.cu", "diag.cu", "k_hor_visc.cu",
              "k_cont_fast.cu", "k_vv_fast.cu", "k_tendency_fast.cu"]
# the mixed-precision form and the fast FP64 kernels contract FMAs; the exact
# FP64 files must not
FMA_SOURCES = {"k_mixed.cu", "k_ensemble.cu", "k_mlp.cu", "k_cont_fast.cu", "k_vv_fast.cu",
               "k_tendency_fast.cu"}
CXX_SOURCES = ["host_init.cpp"]
HEADERS = ["common.cuh", "kernels.h", "host_init.h", "abi_common.cuh", "tendency_impl.cuh",
           "vertvisc_impl.cuh", "mixed_impl.cuh", "halo_impl.cuh", "mlp.h", "mlp_gemm.cuh",
           "diag.h", "cont_impl.cuh", "tma.cuh"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("compile failed: " + os.path.basename(cmd[-1]))
    return r


def build(verbose=False, force=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(HERE, "..", "include", "mom6b.h"),
        os.path.join(HERE, "..", "include", "mom6_cuda_c.h")]
    objs, cmds = [], []
    for src in CU_SOURCES + CXX_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _newer(obj, [path] + hdrs):
            if src.endswith(".cu"):
                flags = CU_FLAGS
                if src in FMA_SOURCES:
                    flags = [f if f != "--fmad=false" else "--fmad=true" for f in CU_FLAGS]
                cmd = [NVCC] + flags + ["-I", CSRC, "-c", "-o", obj, path]
            else:
                cmd = ["g++"] + CXX_FLAGS + ["-I", CSRC, "-I", "/usr/local/cuda/include",
                                             "-c", "-o", obj, path]
            if verbose:
                print(" ".join(cmd))
            cmds.append(cmd)
    # the translation units compile independently: one compiler per core
    if cmds:
        from concurrent.futures import ThreadPoolExecutor
        n = jobs or max(1, min(len(cmds), os.cpu_count() or 1))
        with ThreadPoolExecutor(max_workers=n) as ex:
            for f in [ex.submit(_run, c) for c in cmds]:
                f.result()
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-ldl"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    print(LIB)
