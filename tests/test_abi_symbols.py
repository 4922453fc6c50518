"""The C-ABI library loads and exports every function the headers declare.

Runs without a GPU: it only opens libmom6b.so and resolves symbols (no
compute call is made)."""
import ctypes

import pytest

from tests.abi_cases import declarations


def _lib():
    from hackathon_mom6_miniapp_b200._lib import library_path
    import os
    path = library_path()
    if not os.path.exists(path):
        pytest.skip("libmom6b.so not built")
    return ctypes.CDLL(path)


def test_every_declared_symbol_is_exported():
    lib = _lib()
    decls = declarations()
    missing = [n for n in decls if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_reference_abi_is_complete():
    # 35 launch_* kernels + 8 runtime helpers of the reference's src/cuda_c
    decls = declarations()
    launch = sorted(n for n in decls if n.startswith("launch_"))
    helpers = sorted(n for n in decls if n.startswith("cuda_") and n.endswith("_c"))
    assert len(launch) == 35, launch
    assert len(helpers) == 8, helpers


def test_reference_signatures_are_plain_c():
    # every argument of the reference ABI is a pointer, an int, a double or a size_t
    for name, args in declarations().items():
        if name.startswith(("launch_", "cuda_")):
            assert all(k in "pvidz" for k, _ in args), (name, args)
            if name.startswith("launch_"):
                assert args[-1] == ("v", "stream"), name
