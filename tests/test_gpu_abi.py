"""Per-kernel parity of the reference-compatible ABI on the GPU.

Each launch_* entry point of libmom6b.so is called on seeded inputs and
compared bit for bit with the same entry point of the reference's own CUDA C
kernels, compiled from their sources without FMA contraction
(oracle/_ref/libref_cuda_c_nofma.so, built by `make -C oracle ref`).  Every
kernel is run with the flags the reference wrappers pass and with each flag
flipped alone, on two grid shapes, so every branch of the reference's
kernels is exercised.
"""
import ctypes
import os

import numpy as np
import pytest

from tests.abi_cases import (SCRATCH, Grid, bind, declarations, flag_variants, make_case)

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                   "oracle", "_ref", "libref_cuda_c_nofma.so")
DECLS = declarations(os.path.join(os.path.dirname(REF), "..", "..", "include", "mom6_cuda_c.h"))
LAUNCH = sorted(n for n in DECLS if n.startswith("launch_"))
GRIDS = [Grid(38, 32, 8), Grid(71, 45, 5)]


def _libs():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref not built (make -C oracle ref)")
    from hackathon_mom6_miniapp_b200._lib import abi_set_deferral, library_path
    # one kernel at a time: the barotropic deferral off, so every launch_bt_*
    # call runs as it comes
    abi_set_deferral(False)
    ours = ctypes.CDLL(library_path())
    ref = ctypes.CDLL(REF)
    return ours, ref


def _run(lib, name, decl, arrays, values):
    import torch
    dev = {a: torch.from_numpy(np.ravel(x, order="F").copy()).cuda() for a, x in arrays.items()}
    args = []
    for kind, a in decl:
        if kind == "p":
            args.append(ctypes.c_void_p(dev[a].data_ptr()))
        elif kind == "v":
            args.append(None)
        else:
            args.append(values[a])
    bind(lib, name, decl)(*args)
    torch.cuda.synchronize()
    return {a: t.cpu().numpy() for a, t in dev.items()}


def _cases():
    out = []
    for name in LAUNCH:
        for gi, g in enumerate(GRIDS):
            for fi, fl in enumerate(flag_variants(DECLS[name])):
                out.append(pytest.param(name, gi, fl, id=f"{name[7:]}-g{gi}-f{fi}"))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name,gi,flags", _cases())
def test_launch_matches_reference_bitwise(name, gi, flags):
    ours, ref = _libs()
    decl = DECLS[name]
    arrays, values = make_case(name, decl, GRIDS[gi], seed=11 + gi, flags=flags)
    a = _run(ours, name, decl, arrays, values)
    b = _run(ref, name, decl, arrays, values)
    bad = []
    for arr in a:
        if arr in SCRATCH.get(name, ()):
            continue
        if not np.array_equal(a[arr].view(np.uint64), b[arr].view(np.uint64)):
            d = np.flatnonzero(a[arr].view(np.uint64) != b[arr].view(np.uint64))
            bad.append(f"{arr}: {d.size} differ, first flat index {d[0]}: "
                       f"{a[arr][d[0]]!r} vs {b[arr][d[0]]!r}")
    assert not bad, "\n".join(bad)


@pytest.mark.gpu
def test_runtime_helpers_roundtrip():
    ours, _ = _libs()
    d = declarations(os.path.join(os.path.dirname(REF), "..", "..", "include", "mom6_cuda_c.h"))
    f = {n: getattr(ours, n) for n in d if n.startswith("cuda_")}
    f["cuda_malloc_c"].restype = ctypes.c_void_p
    f["cuda_malloc_c"].argtypes = [ctypes.c_size_t]
    for n in ("cuda_memcpy_h2d_c", "cuda_memcpy_d2h_c", "cuda_memcpy_d2d_c"):
        f[n].argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    f["cuda_memset_c"].argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t]
    f["cuda_free_c"].argtypes = [ctypes.c_void_p]
    assert f["cuda_set_device_c"](0) == 0
    n = 1000
    x = np.arange(n, dtype=np.float64)
    a = f["cuda_malloc_c"](n * 8)
    b = f["cuda_malloc_c"](n * 8)
    assert a and b
    assert f["cuda_memcpy_h2d_c"](a, x.ctypes.data, n * 8) == 0
    assert f["cuda_memcpy_d2d_c"](b, a, n * 8) == 0
    y = np.empty(n)
    assert f["cuda_memcpy_d2h_c"](y.ctypes.data, b, n * 8) == 0
    assert np.array_equal(x, y)
    assert f["cuda_memset_c"](b, 0, n * 8) == 0
    assert f["cuda_device_synchronize_c"]() == 0
    assert f["cuda_memcpy_d2h_c"](y.ctypes.data, b, n * 8) == 0
    assert not y.any()
    f["cuda_free_c"](a)
    f["cuda_free_c"](b)
    f["cuda_free_c"](None)
    # an impossible allocation returns NULL and leaves no sticky error
    assert not f["cuda_malloc_c"](1 << 62)
    assert f["cuda_device_synchronize_c"]() == 0
