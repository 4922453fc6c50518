"""The fast FP64 form of the step (exact=False, the default) against the oracle.

The fast kernels may contract multiply-adds, form quotients by refined
reciprocals and sum columns in another order (the continuity kernel splits
each face column over 8 lanes and combines their partial sums by shuffles;
the vertical viscosity forms its bottom-boundary function top-down), so they
are held to the step's parity bound instead of bit equality: relative L2 <=
1e-12 per prognostic field after 10 steps, and the continuity and vertical
viscosity outputs of a step (transports, face thicknesses, BT_cont face
areas and velocities, bottom stresses) close to the exact form's.  Shapes
with odd n1 (= ni + 2) take the continuity kernel's cooperative tile copy,
even n1 its TMA tile loads; nk > 80 takes the 16-layers-per-lane
instantiation.
"""
import numpy as np
import pytest

from oracle.pyoracle import INIT_CFG, INIT_REF, Oracle
from tests.util import describe, rel_l2

TOL = 1e-12
STATE = ["h", "u", "v", "eta", "ubt", "vbt"]


def _models(ni, nj, nk, bt, mode, seed, **kw):
    from hackathon_mom6_miniapp_b200 import Model
    fast = Model(ni, nj, nk, bt, mode, seed=seed, exact=False, **kw)
    exact = Model(ni, nj, nk, bt, mode, seed=seed, exact=True, **kw)
    return fast, exact


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(13, 11, 5), (36, 30, 8), (70, 50, 12), (40, 30, 100)])
@pytest.mark.parametrize("mode", [INIT_CFG, INIT_REF])
def test_ten_steps_within_bound(shape, mode):
    ni, nj, nk = shape
    o = Oracle(ni, nj, nk, 40, mode, seed=7)
    fast, _ = _models(ni, nj, nk, 40, mode, 7)
    o.step(10)
    fast.step(10)
    bad = [f"{n}: {describe(fast.get(n), o.get(n))}" for n in STATE
           if not rel_l2(fast.get(n), o.get(n)) <= TOL]
    assert not bad, "\n".join(bad)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(37, 30, 8), (36, 30, 8), (40, 30, 100)])
def test_continuity_outputs_close_to_exact(shape):
    ni, nj, nk = shape
    fast, exact = _models(ni, nj, nk, 40, INIT_CFG, 2)
    fast.step(2)
    exact.step(2)
    sl = (slice(exact.is_ - 2, exact.ie), slice(exact.js - 1, exact.je))
    for n, tol in (("uh", 1e-12), ("hu_bt", 1e-12), ("h", 1e-13), ("du_cor", 1e-9),
                   ("FA_u_W0", 1e-12), ("FA_u_WW", 1e-12), ("FA_u_E0", 1e-12),
                   ("FA_u_EE", 1e-12), ("uBT_WW", 1e-8), ("uBT_EE", 1e-8), ("up", 1e-12),
                   ("vp", 1e-12)):
        a, b = fast.get(n)[sl], exact.get(n)[sl]
        assert np.isfinite(a).all(), n
        assert rel_l2(a, b) <= tol, f"{n}: {describe(a, b)}"
    for n in ("taux_bot", "tauy_bot"):
        a, b = fast.get(n), exact.get(n)
        assert rel_l2(a, b) <= 1e-11, f"{n}: {describe(a, b)}"


@pytest.mark.gpu
def test_fast_step_conserves_volume():
    from hackathon_mom6_miniapp_b200 import Model
    g = Model(64, 48, 10, 40, INIT_CFG, seed=1)
    g.step(5)
    assert g.verify()["rel_error"] < 1e-10


@pytest.mark.gpu
def test_fast_graph_replay_matches_eager():
    from hackathon_mom6_miniapp_b200 import Model
    a = Model(36, 30, 8, 40, INIT_CFG, seed=3, use_graph=False)
    b = Model(36, 30, 8, 40, INIT_CFG, seed=3, use_graph=True)
    a.step(4)
    b.step(4)
    for n in STATE + ["uh", "hu_bt"]:
        assert np.array_equal(a.get(n), b.get(n)), n



@pytest.mark.gpu
def test_vertvisc_two_sweep_and_fallback_columns():
    """The fast vertical viscosity eliminates bottom-up and back-substitutes
    top-down where the top four layers' harmonic thicknesses reach Hmix (50 m),
    and falls back to the three-sweep column elsewhere.  Half of this domain
    gets 5 m surface layers (20 m in total: fallback), the rest keeps its
    layers; the step's velocities, bottom stresses and thicknesses stay
    within the bound of the exact form's in both halves."""
    ni, nj, nk = 40, 30, 12
    fast, exact = _models(ni, nj, nk, 40, INIT_CFG, 9)
    h0 = exact.get("h0")
    h0[:, : h0.shape[1] // 2, :4] = 5.0
    for m in (fast, exact):
        m.set("h0", h0)
        m.set("h", h0)
    fast.step(2)
    exact.step(2)
    for n in ("u", "v", "h", "up", "vp"):
        a, b = fast.get(n), exact.get(n)
        assert rel_l2(a, b) <= 1e-12, f"{n}: {describe(a, b)}"
    for n in ("taux_bot", "tauy_bot"):
        a, b = fast.get(n), exact.get(n)
        assert rel_l2(a, b) <= 1e-11, f"{n}: {describe(a, b)}"
