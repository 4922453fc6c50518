"""Meridional continuity on the GPU (k_ppm_edges_y + k_cont_faces_y): the
single pass against the oracle's meridional pass bit for bit; the single pass
against the GPU's own zonal pass on transposed inputs (square grid, symmetric
metrics) bit for bit; whole steps with zonal then meridional continuity
against the oracle bit for bit."""
import numpy as np
import pytest

from oracle.pyoracle import INIT_CFG, Oracle

DT = 600.0
BT_V = ["FA_v_S0", "FA_v_SS", "FA_v_N0", "FA_v_NN", "vBT_SS", "vBT_NN", "dv_cor"]
PAIRS = {"FA_u_W0": "FA_v_S0", "FA_u_WW": "FA_v_SS", "FA_u_E0": "FA_v_N0",
         "FA_u_EE": "FA_v_NN", "uBT_WW": "vBT_SS", "uBT_EE": "vBT_NN", "du_cor": "dv_cor"}


def _model(ni, nj, nk, seed):
    from hackathon_mom6_miniapp_b200 import Model
    m = Model(ni, nj, nk, 30, INIT_CFG, seed=seed, exact=True)
    m.set_continuity_merid(True)
    return m


def _inputs(shape, base_v, base_h, seed):
    rng = np.random.default_rng(seed)
    v = np.asfortranarray(base_v + rng.normal(0, 0.3, size=shape))
    h = np.asfortranarray(base_h * (1 + 0.5 * rng.random(shape)))
    return v, h


def _cells(m):
    return (slice(m.is_ - 1, m.ie), slice(m.js - 1, m.je))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(40, 28, 5), (33, 47, 6)])
def test_single_pass_matches_the_oracle(shape):
    m = _model(*shape, seed=4)
    o = Oracle(*shape, 30, INIT_CFG, seed=4)
    v, h0 = _inputs(m.get("v").shape, m.get("v"), m.get("h0"), seed=7)
    m.set("v", v)
    m.set("h0", h0)
    m.continuity_pass("y", DT)
    oh, ovh = o.continuity_merid(v, h0, DT)
    c = _cells(m)
    assert np.array_equal(m.get("h")[c], oh[c])
    assert np.array_equal(m.get("vh"), ovh)
    assert np.array_equal(m.get("hv_bt"), o.get("hv_bt"))
    for f in BT_V:
        assert np.array_equal(m.get(f), o.get(f)), f


@pytest.mark.gpu
def test_single_pass_is_the_transposed_zonal_pass():
    X = _model(38, 38, 5, seed=2)
    Y = _model(38, 38, 5, seed=2)
    u, h0 = _inputs(X.get("u").shape, X.get("u"), X.get("h0"), seed=3)
    X.set("u", u)
    X.set("h0", h0)
    X.continuity_pass("x", DT)
    Y.set("v", np.asfortranarray(u.transpose(1, 0, 2)))
    Y.set("h0", np.asfortranarray(h0.transpose(1, 0, 2)))
    Y.continuity_pass("y", DT)
    c = _cells(X)
    f = (slice(X.is_ - 2, X.ie), slice(X.js - 1, X.je))
    assert np.array_equal(X.get("h")[c], Y.get("h").transpose(1, 0, 2)[c])
    assert np.array_equal(X.get("uh")[f], Y.get("vh").transpose(1, 0, 2)[f])
    assert np.array_equal(X.get("hu_bt")[f], Y.get("hv_bt").transpose(1, 0, 2)[f])
    for zu, zv in PAIRS.items():
        assert np.array_equal(X.get(zu)[f], Y.get(zv).T[f]), zu


@pytest.mark.gpu
@pytest.mark.parametrize("bc_fill", [0, 1])
def test_steps_with_the_meridional_pass_match_the_oracle(bc_fill):
    from hackathon_mom6_miniapp_b200 import Model
    m = Model(40, 28, 5, 30, INIT_CFG, seed=6, bc_fill=bc_fill, exact=True)
    m.set_continuity_merid(True)
    o = Oracle(40, 28, 5, 30, INIT_CFG, seed=6, bc_fill=bc_fill)
    o.set_merid(True)
    m.step(3)
    o.step(3)
    for f in ["h", "u", "v", "eta", "ubt_av", "hv_bt"] + BT_V:
        assert np.array_equal(m.get(f), o.get(f)), f
    # the oracle's uh, vh also hold the transports of compute_transports
    # outside the faces continuity writes; the fused step keeps those on chip
    fu = (slice(m.is_ - 2, m.ie), slice(m.js - 1, m.je))
    fv = (slice(m.is_ - 1, m.ie), slice(m.js - 2, m.je))
    assert np.array_equal(m.get("uh")[fu], o.get("uh")[fu])
    assert np.array_equal(m.get("vh")[fv], o.get("vh")[fv])
