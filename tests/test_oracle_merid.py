"""The oracle's meridional continuity (the zonal restatement applied to the
transposed problem): on a square grid with symmetric metrics, the meridional
pass of transposed inputs is the transposed zonal pass, field by field.  The
GPU kernel is held to this oracle (tests/test_gpu_merid.py)."""
import numpy as np

from oracle.pyoracle import INIT_CFG, Oracle

PAIRS = {"FA_u_W0": "FA_v_S0", "FA_u_WW": "FA_v_SS", "FA_u_E0": "FA_v_N0",
         "FA_u_EE": "FA_v_NN", "uBT_WW": "vBT_SS", "uBT_EE": "vBT_NN", "du_cor": "dv_cor"}


def _inputs(o, seed):
    rng = np.random.default_rng(seed)
    u = np.asfortranarray(o.get("u") + rng.normal(0, 0.3, size=o.get("u").shape))
    h0 = np.asfortranarray(o.get("h0") * (1 + 0.5 * rng.random(o.get("h0").shape)))
    return u, h0


def test_meridional_pass_is_the_transposed_zonal_pass():
    o = Oracle(36, 36, 5, 30, INIT_CFG, seed=3)
    u, h0 = _inputs(o, 1)
    hz, uh = o.continuity(u, h0, 600.0)
    bt = {n: o.get(n).copy() for n in PAIRS}
    hu = o.get("hu_bt").copy()
    hm, vh = o.continuity_merid(np.asfortranarray(u.transpose(1, 0, 2)),
                                np.asfortranarray(h0.transpose(1, 0, 2)), 600.0)
    c = (slice(o.is_ - 1, o.ie), slice(o.js - 1, o.je))          # cells
    f = (slice(o.is_ - 2, o.ie), slice(o.js - 1, o.je))          # u faces
    assert np.array_equal(hz[c], hm.transpose(1, 0, 2)[c])
    assert np.array_equal(uh[f], vh.transpose(1, 0, 2)[f])
    assert np.array_equal(hu[f], o.get("hv_bt").transpose(1, 0, 2)[f])
    for zu, zv in PAIRS.items():
        assert np.array_equal(bt[zu][f], o.get(zv).T[f]), zu


def test_step_with_the_meridional_pass_writes_its_outputs():
    """A step with zonal then meridional continuity keeps h finite and
    non-negative and writes vh and the v fields of BT_cont."""
    o = Oracle(30, 24, 4, 30, INIT_CFG, seed=5)
    o.set_merid(True)
    o.step(2)
    h = o.get("h")
    assert np.all(np.isfinite(h)) and np.all(h >= 0)
    assert np.any(o.get("vh") != 0) and np.any(o.get("FA_v_S0") != 0)
