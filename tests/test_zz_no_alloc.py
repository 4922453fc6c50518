"""The allocation-free barotropic entry point (mom6b_btstep_noalloc).

Callers that cannot allocate device memory where they run the barotropic
solver (a Fortran host whose device arrays belong to an OpenMP-target or
OpenACC runtime, which owns the device pool) get the whole
btstep loop from this entry point, with its work arrays in a static device
array of the library.  These tests call it through the C ABI twice in a row,
as the split RK2 step does (predictor, then corrector with aliased in/out),
and check the results bit for bit against the model's own barotropic kernel
(mom6b_step), which allocates its work arrays when the model is created.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

BT = 40


def _lib():
    from hackathon_mom6_miniapp_b200 import library
    L = library()
    vp = ctypes.c_void_p
    L.mom6b_btstep_noalloc.argtypes = ([vp] * 19 + [ctypes.c_int] * 7 +
                                       [ctypes.c_double] * 3 + [ctypes.c_int] * 2 + [vp])
    L.mom6b_btstep_noalloc.restype = ctypes.c_int
    L.mom6b_metric_device_ptr.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(vp)]
    return L


def _metric(L, model, name):
    p = ctypes.c_void_p()
    assert L.mom6b_metric_device_ptr(model._m, name.encode(), ctypes.byref(p)) == 0
    return p.value


def _call(L, model, mets, eta_in, ubt_in, vbt_in, u_av, v_av, eta_av, stream):
    dt = model.cfg.dt
    rc = L.mom6b_btstep_noalloc(
        eta_in, ubt_in, vbt_in, u_av, v_av, eta_av, *mets,
        model.n1, model.n2, model.is_, model.ie, model.js, model.je,
        BT, dt / BT, 0.2, 1.0, 0, 0, stream)
    return rc


@pytest.mark.gpu
def test_noalloc_matches_model_btstep_two_calls():
    import torch
    from hackathon_mom6_miniapp_b200 import INIT_REF, Model
    L = _lib()
    m = Model(64, 48, 6, BT, INIT_REF)  # no halo fill between the two btsteps
    names = ["Datu", "Datv", "gtot_E", "gtot_W", "gtot_N", "gtot_S", "f_4_u", "f_4_v",
             "bt_rem_u", "bt_rem_v", "IareaT", "IdxCu", "IdyCv"]
    mets = [_metric(L, m, n) for n in names]
    shape = (m.n2, m.n1)  # C-order (j, i) == Fortran (i, j)
    dev = torch.device("cuda:0")
    eta = torch.from_numpy(np.ascontiguousarray(m.get("eta").T)).to(dev)
    ubt = torch.from_numpy(np.ascontiguousarray(m.get("ubt").T)).to(dev)
    vbt = torch.from_numpy(np.ascontiguousarray(m.get("vbt").T)).to(dev)
    ua = torch.full(shape, np.nan, dtype=torch.float64, device=dev)
    va = torch.full(shape, np.nan, dtype=torch.float64, device=dev)
    ea = torch.full(shape, np.nan, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    # predictor: btstep(eta, ubt, vbt -> ubt_av, vbt_av, eta_av)
    assert _call(L, m, mets, eta.data_ptr(), ubt.data_ptr(), vbt.data_ptr(),
                 ua.data_ptr(), va.data_ptr(), ea.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    ea1 = ea.cpu().numpy().T.copy()
    # corrector: btstep(eta_av, ubt_av, vbt_av -> ubt_av, vbt_av, eta), aliased
    eta2 = torch.full(shape, np.nan, dtype=torch.float64, device=dev)
    assert _call(L, m, mets, ea.data_ptr(), ua.data_ptr(), va.data_ptr(),
                 ua.data_ptr(), va.data_ptr(), eta2.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    # the existing entry point: one model step runs the same two btsteps
    m.step(1)
    assert np.array_equal(ea1, m.get("eta_av"))
    assert np.array_equal(ua.cpu().numpy().T, m.get("ubt_av"))
    assert np.array_equal(va.cpu().numpy().T, m.get("vbt_av"))
    assert np.array_equal(eta2.cpu().numpy().T, m.get("eta"))


@pytest.mark.gpu
def test_noalloc_rejects_grids_beyond_capacity():
    L = _lib()
    fake = [1] * 19  # never dereferenced: the size check comes first
    rc = L.mom6b_btstep_noalloc(*fake[:6], *fake[6:], 800, 800, 4, 797, 4, 797,
                                10, 10.0, 0.2, 1.0, 0, 0, None)
    assert rc == 2  # MOM6B_NOALLOC_ERR_TOO_LARGE
