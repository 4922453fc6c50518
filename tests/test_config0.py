"""Configuration 0 of the benchmark definition on the oracle (CPU).

Configuration 0 is 180x180x75 with the seeded beta-plane state, dt = 600 s
and bt_nsteps = 30.  The serial barotropic scheme is not stable there: its
substep dt/30 = 20 s puts gravity waves (sqrt(g H) ~ 198 m/s over 10 km
cells) past the forward-backward scheme's limit with the 1.2/-0.2 transport
weights, and the oracle -- the C restatement of rk2_serial_driver -- grows
eta by orders of magnitude within 10 steps.  31 substeps is the fewest that
stay bounded, so the parity tests and the ensemble run configuration 0's
construction at bt_nsteps = 31.
"""
import numpy as np
import pytest

from oracle.pyoracle import INIT_CFG, Oracle


def _max_eta_after(bt, nsteps, n=180, nk=75):
    o = Oracle(n, n, nk, bt, INIT_CFG, seed=0, dt=600.0, threads=0)
    o.step(nsteps)
    e = o.get("eta")
    o.close()
    return float(np.nanmax(np.abs(e))) if np.isfinite(e).any() else float("inf")


def test_bt30_diverges_in_the_oracle():
    # the initial bump is 0.1 m; after 10 steps at bt 30 eta is far beyond
    # any physical value (about 2e20 m here)
    assert not (_max_eta_after(30, 10) < 1.0e3)


@pytest.mark.parametrize("bt", [31, 35])
def test_bt31_and_above_stay_bounded(bt):
    assert _max_eta_after(bt, 10) < 0.1
