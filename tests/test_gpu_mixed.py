"""The mixed-precision form (FP32 state and stencils; FP64 column sums,
Newton scalars, thickness update, vertical elimination and barotropic loop)
against the FP64 oracle: per-field relative L2 error after 10 steps at most
1e-5, the bound the mixed form is specified with.  The errors are printed."""
import numpy as np
import pytest

from oracle.pyoracle import INIT_CFG, INIT_REF, Oracle
from tests.util import rel_l2

FIELDS = ["h", "u", "v", "eta", "ubt_av", "vbt_av"]
BOUND = 1e-5


def _mixed(ni, nj, nk, bt, mode, seed=0, dt=None):
    from hackathon_mom6_miniapp_b200 import MIXED, Model
    return Model(ni, nj, nk, bt, mode, seed=seed, dt=dt, precision=MIXED, exact=True)


@pytest.mark.gpu
@pytest.mark.parametrize("case", [(70, 50, 12, 40, INIT_CFG, 600.0), (180, 180, 75, 30, INIT_REF, 300.0)])
def test_mixed_form_error_against_fp64_oracle(case):
    ni, nj, nk, bt, mode, dt = case
    o = Oracle(ni, nj, nk, bt, mode, seed=5, dt=dt)
    g = _mixed(ni, nj, nk, bt, mode, seed=5, dt=dt)
    o.step(10)
    g.step(10)
    errs = {f: rel_l2(g.get(f), o.get(f)) for f in FIELDS}
    print("mixed-form rel L2 after 10 steps", case[:3], {k: f"{v:.2e}" for k, v in errs.items()})
    assert all(np.isfinite(v) for v in errs.values())
    assert max(errs.values()) <= BOUND, errs


@pytest.mark.gpu
def test_mixed_form_conserves_mass():
    g = _mixed(70, 50, 12, 40, INIT_CFG, seed=2)
    g.step(10)
    # FP32 storage of h rounds every thickness (2**-24 relative) each step
    assert g.verify()["rel_error"] < 1e-6


@pytest.mark.gpu
def test_mixed_form_field_roundtrip():
    g = _mixed(36, 30, 8, 40, INIT_CFG, seed=1)
    h = g.get("h")
    h2 = h * 1.0009765625          # exactly representable scaling keeps FP32 values exact
    g.set("h0", h2)
    assert np.array_equal(g.get("h0"), h2.astype(np.float32).astype(np.float64))
    assert g.get("u").dtype == np.float64
