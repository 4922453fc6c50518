"""The Arakawa HSU90 and LAMB81 Coriolis schemes of CorAdCalc
(mom6_coriolis_serial.F90:171-193, :228-248), which the serial driver does
not exercise, in the fused FP64 step: bit for bit against the oracle (whose
schemes are pinned to the reference's CUDA C kernels in
test_gpu_oracle_pin.py), and different from the Sadourny step."""
import numpy as np
import pytest

from oracle.pyoracle import INIT_CFG, INIT_REF, Oracle

FIELDS = ["u", "v", "h", "up", "vp", "eta", "ubt_av"]


def _pair(scheme, mode, shape=(40, 30, 6), seed=2):
    from hackathon_mom6_miniapp_b200 import Model
    dt = 300.0 if mode == INIT_REF else None
    m = Model(*shape, 30, mode, seed=seed, dt=dt, exact=True)
    o = Oracle(*shape, 30, mode, seed=seed, dt=dt)
    m.set_coriolis_scheme(scheme)
    o.set_coriolis_scheme(scheme)
    return m, o


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [2, 3])
@pytest.mark.parametrize("mode", [INIT_CFG, INIT_REF])
def test_arakawa_steps_match_the_oracle(scheme, mode):
    m, o = _pair(scheme, mode)
    m.step(3)
    o.step(3)
    for f in FIELDS:
        assert np.array_equal(m.get(f), o.get(f)), f


@pytest.mark.gpu
def test_schemes_differ_and_switch_back():
    from hackathon_mom6_miniapp_b200 import Model
    a = Model(40, 30, 6, 30, INIT_CFG, seed=2, exact=True)
    b = Model(40, 30, 6, 30, INIT_CFG, seed=2, exact=True)
    c = Model(40, 30, 6, 30, INIT_CFG, seed=2, exact=True)
    b.set_coriolis_scheme(2)
    c.set_coriolis_scheme(3)
    c.set_coriolis_scheme(1)
    for m in (a, b, c):
        m.step(2)
    assert not np.array_equal(a.get("u"), b.get("u"))
    assert np.array_equal(a.get("u"), c.get("u"))
