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
    L.mom6b_btstep_noalloc_status.argtypes = [vp]
    L.mom6b_btstep_noalloc_set_wait.argtypes = [ctypes.c_longlong, ctypes.c_int]
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
    m = Model(64, 48, 6, BT, INIT_REF, exact=True)  # no halo fill between the two btsteps
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


def _oracle_inputs(o):
    return [np.asfortranarray(o.get(n)) for n in ("eta", "ubt", "vbt")]


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(torch.device("cuda:0"))


def _noalloc_vs_oracle(ni, nj, extended, first_direction, nstep=12):
    """One call of the entry point against the oracle's btstep on the same
    inputs, with the model's metric arrays (both build init_ocean_grid's)."""
    import torch
    from hackathon_mom6_miniapp_b200 import INIT_REF, Model
    from oracle.pyoracle import INIT_REF as O_REF, Oracle
    L = _lib()
    m = Model(ni, nj, 2, nstep, INIT_REF, exact=True)
    o = Oracle(ni, nj, 2, nstep, O_REF)
    o.set_bt_extended(extended)
    o.set_bt_first_direction(first_direction)
    names = ["Datu", "Datv", "gtot_E", "gtot_W", "gtot_N", "gtot_S", "f_4_u", "f_4_v",
             "bt_rem_u", "bt_rem_v", "IareaT", "IdxCu", "IdyCv"]
    mets = [_metric(L, m, n) for n in names]
    eta, ubt, vbt = _oracle_inputs(o)
    rng = np.random.default_rng(3)
    ubt = np.asfortranarray(ubt + 0.01 * rng.standard_normal(ubt.shape))
    vbt = np.asfortranarray(vbt + 0.01 * rng.standard_normal(vbt.shape))
    want_u, want_v, want_e = o.btstep(eta, ubt, vbt)
    de, du, dv = _dev(eta), _dev(ubt), _dev(vbt)
    shape = (m.n2, m.n1)
    outs = [torch.full(shape, np.nan, dtype=torch.float64, device="cuda:0") for _ in range(3)]
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    rc = L.mom6b_btstep_noalloc(de.data_ptr(), du.data_ptr(), dv.data_ptr(),
                                *[t.data_ptr() for t in outs], *mets,
                                m.n1, m.n2, m.is_, m.ie, m.js, m.je, nstep,
                                m.cfg.dt / nstep, 0.2, 1.0, first_direction, int(extended),
                                stream)
    assert rc == 0
    assert L.mom6b_btstep_noalloc_status(stream) == 0
    got = [t.cpu().numpy().T for t in outs]
    return got, (want_u, want_v, want_e)


@pytest.mark.gpu
@pytest.mark.parametrize("extended", [0, 1])
@pytest.mark.parametrize("first_direction", [0, 1])
def test_noalloc_ranges_and_direction_match_oracle(extended, first_direction):
    """The extended uhbt/vhbt ranges of the CUDA C kernels and both update
    orders: the oracle's btstep with the same options, bit for bit."""
    got, want = _noalloc_vs_oracle(64, 48, extended, first_direction)
    for g, w, n in zip(got, want, ("ubt_av", "vbt_av", "eta")):
        assert np.array_equal(g, w), n


@pytest.mark.gpu
def test_noalloc_non_square_grid_within_capacity():
    """A 1022 x 574 grid (n1 * n2 = 589,824, the capacity) is elongated but
    splits into one tile per SM: it is accepted and matches the oracle."""
    got, want = _noalloc_vs_oracle(1022, 574, 0, 0, nstep=4)
    for g, w, n in zip(got, want, ("ubt_av", "vbt_av", "eta")):
        assert np.array_equal(g, w), n


@pytest.mark.gpu
def test_noalloc_rejects_boxes_without_a_tiling():
    # n1 * n2 at the capacity, but 4096 x 144 needs 64 x 3 tiles of 64 points
    L = _lib()
    fake = [1] * 19
    rc = L.mom6b_btstep_noalloc(*fake, 4096, 144, 4, 4093, 4, 141, 10, 10.0, 0.2, 1.0, 0, 0,
                                None)
    assert rc == 2  # MOM6B_NOALLOC_ERR_TOO_LARGE


@pytest.mark.gpu
def test_noalloc_reports_a_barrier_timeout():
    """With the stall testing aid the loop's first barrier waits for an
    arrival that never comes; every block gives up after the wait limit
    (2e6 cycles, about 1 ms) and the status query returns
    MOM6B_NOALLOC_ERR_TIMEOUT.  The next call, with the aid off, runs
    normally and its status is OK."""
    import torch
    from hackathon_mom6_miniapp_b200 import INIT_REF, Model
    L = _lib()
    m = Model(64, 48, 2, 12, INIT_REF, exact=True)
    names = ["Datu", "Datv", "gtot_E", "gtot_W", "gtot_N", "gtot_S", "f_4_u", "f_4_v",
             "bt_rem_u", "bt_rem_v", "IareaT", "IdxCu", "IdyCv"]
    mets = [_metric(L, m, n) for n in names]
    e, u, v = (_dev(m.get(n)) for n in ("eta", "ubt", "vbt"))
    outs = [torch.zeros_like(e) for _ in range(3)]
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    assert L.mom6b_btstep_noalloc_set_wait(2_000_000, 1) == 0
    try:
        rc = L.mom6b_btstep_noalloc(e.data_ptr(), u.data_ptr(), v.data_ptr(),
                                    *[t.data_ptr() for t in outs], *mets,
                                    m.n1, m.n2, m.is_, m.ie, m.js, m.je, 12, m.cfg.dt / 12,
                                    0.2, 1.0, 0, 0, stream)
        assert rc == 0
        assert L.mom6b_btstep_noalloc_status(stream) == 4   # MOM6B_NOALLOC_ERR_TIMEOUT
        assert L.mom6b_btstep_noalloc_status(stream) == 0   # cleared by the query
    finally:
        assert L.mom6b_btstep_noalloc_set_wait(0, 0) == 0
    got, want = _noalloc_vs_oracle(64, 48, 0, 0)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
