"""Argument checks of the C-ABI entry points, on the host.

mom6b_create and mom6b_btstep_noalloc check their sizes, bounds and pointers
before any CUDA call, so an invalid call is rejected with MOM6B_ERR_ARG (and a
message from mom6b_last_error) or MOM6B_NOALLOC_ERR_ARG on a machine without a
GPU as well.  No call here reaches the device."""
import ctypes
import os

import pytest

ERR_ARG = 1            # MOM6B_ERR_ARG
NOALLOC_ERR_ARG = 1    # MOM6B_NOALLOC_ERR_ARG


def _lib():
    from hackathon_mom6_miniapp_b200._lib import library, library_path
    if not os.path.exists(library_path()):
        pytest.skip("libmom6b.so not built")
    return library()


@pytest.mark.parametrize("kw, msg", [
    (dict(ni=7), "sizes must satisfy"),
    (dict(nj=5), "sizes must satisfy"),
    (dict(nk=1), "sizes must satisfy"),
    (dict(bt_nsteps=0), "sizes must satisfy"),
    (dict(nk=1025), "nk > 1024"),
    (dict(ni=40000, nj=40000), "horizontal grid too large"),
    (dict(precision=7), "unknown precision"),
    # a 20x20 subdomain at i_offset 15 reaches global cell 31 of 26
    (dict(ni=20, nj=20, subdomain=(30, 30, 15, 0, 0)), "subdomain outside"),
    (dict(ni=20, nj=20, subdomain=(30, 30, 0, 0, 16)), "subdomain outside"),
    (dict(ni=20, nj=20, subdomain=(40, 20, 0, 0, 1), bc_fill=True), "cuts steps in FP64"),
    (dict(ni=20, nj=20, subdomain=(40, 20, 0, 0, 1), precision=1), "cuts steps in FP64"),
])
def test_model_rejects_invalid_configurations(kw, msg):
    from hackathon_mom6_miniapp_b200._lib import Model, Mom6bError
    _lib()
    with pytest.raises(Mom6bError) as e:
        Model(**kw)
    assert e.value.code == ERR_ARG
    assert msg in str(e.value)


def test_create_and_config_reject_null_pointers():
    L = _lib()
    vp = ctypes.c_void_p
    L.mom6b_create.argtypes = [vp, vp]
    L.mom6b_config_default.argtypes = [vp, ctypes.c_int]
    assert L.mom6b_create(None, None) == ERR_ARG
    assert "null" in L.mom6b_last_error().decode()
    assert L.mom6b_config_default(None, 0) == ERR_ARG


def _noalloc(L):
    vp = ctypes.c_void_p
    f = L.mom6b_btstep_noalloc
    f.argtypes = [vp] * 19 + [ctypes.c_int] * 7 + [ctypes.c_double] * 3 + [ctypes.c_int] * 2 + [vp]
    f.restype = ctypes.c_int
    return f


@pytest.mark.parametrize("null_at", [0, 5, 6, 18])
def test_noalloc_rejects_null_pointers(null_at):
    f = _noalloc(_lib())
    ptrs = [8] * 19          # never dereferenced: the checks come first
    ptrs[null_at] = None
    assert f(*ptrs, 64, 48, 4, 61, 4, 45, 10, 10.0, 0.2, 1.0, 0, 0, None) == NOALLOC_ERR_ARG


@pytest.mark.parametrize("dims", [
    (3, 48, 4, 61, 4, 45, 10),     # n1 < 4
    (64, 48, 4, 61, 4, 45, 0),     # nstep < 1
    (64, 48, 1, 61, 4, 45, 10),    # is < 2
    (64, 48, 4, 64, 4, 45, 10),    # ie > n1 - 1
    (64, 48, 4, 61, 4, 48, 10),    # je > n2 - 1
    (64, 48, 30, 31, 4, 45, 10),   # fewer than 3 columns
    (64, 48, 4, 61, 20, 21, 10),   # fewer than 3 rows
])
def test_noalloc_rejects_inconsistent_bounds(dims):
    f = _noalloc(_lib())
    n1, n2, is_, ie, js, je, nstep = dims
    assert f(*([8] * 19), n1, n2, is_, ie, js, je, nstep, 10.0, 0.2, 1.0, 0, 0,
             None) == NOALLOC_ERR_ARG
