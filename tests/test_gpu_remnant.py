"""The vertical-viscosity remnant feeding continuity (Model.set_visc_remnant).

Every vertvisc of the step also solves vert_visc_remnant's tridiagonal system
(mom6_vert_visc_serial.F90:295-387) with the velocity's elimination
coefficients, and the continuity after it runs zonal_mass_flux's
use_visc_rem form (mom6_continuity_serial.F90:335-433, :581, :880,
:1001-1018, :730).  Whole steps are compared with the oracle bit for bit,
zonal only and zonal then meridional, with and without the halo fill; a
remnant of 1 reproduces the plain continuity bit for bit."""
import numpy as np
import pytest

from oracle.pyoracle import INIT_CFG, Oracle

BT_U = ["FA_u_W0", "FA_u_WW", "FA_u_E0", "FA_u_EE", "uBT_WW", "uBT_EE", "du_cor"]
BT_V = ["FA_v_S0", "FA_v_SS", "FA_v_N0", "FA_v_NN", "vBT_SS", "vBT_NN", "dv_cor"]
SHAPE = (40, 28, 6)


def _pair(merid, bc_fill=0, seed=5):
    from hackathon_mom6_miniapp_b200 import Model
    m = Model(*SHAPE, 30, INIT_CFG, seed=seed, bc_fill=bc_fill, exact=True)
    o = Oracle(*SHAPE, 30, INIT_CFG, seed=seed, bc_fill=bc_fill)
    m.set_visc_remnant(True)
    o.set_remnant(True)
    if merid:
        m.set_continuity_merid(True)
        o.set_merid(True)
    return m, o


@pytest.mark.gpu
@pytest.mark.parametrize("merid,bc_fill", [(False, 0), (False, 1), (True, 0), (True, 1)])
def test_steps_with_the_remnant_match_the_oracle(merid, bc_fill):
    m, o = _pair(merid, bc_fill)
    m.step(3)
    o.step(3)
    fields = ["h", "u", "v", "eta", "ubt_av", "vbt_av", "hu_bt", "visc_rem_u",
              "visc_rem_v"] + BT_U
    if merid:
        fields += ["hv_bt"] + BT_V
    for f in fields:
        assert np.array_equal(m.get(f), o.get(f)), f
    fu = (slice(m.is_ - 2, m.ie), slice(m.js - 1, m.je))
    assert np.array_equal(m.get("uh")[fu], o.get("uh")[fu])
    # the remnant is a fraction below 1 on the open faces and changes the step
    vr = m.get("visc_rem_u")[fu]
    assert (vr < 1.0).any() and (vr > 0.9).all() and (vr <= 1.0 + 1e-15).all()
    o2 = Oracle(*SHAPE, 30, INIT_CFG, seed=5, bc_fill=bc_fill)
    if merid:
        o2.set_merid(True)
    o2.step(3)
    assert not np.array_equal(m.get("h"), o2.get("h"))


@pytest.mark.gpu
@pytest.mark.parametrize("direction", ["x", "y"])
def test_unit_remnant_is_the_plain_continuity(direction):
    """With visc_rem = 1 every factor of the remnant form is exact, so the
    remnant kernels reproduce the plain ones bit for bit."""
    from hackathon_mom6_miniapp_b200 import Model
    out = []
    for rem in (False, True):
        m = Model(*SHAPE, 30, INIT_CFG, seed=8, exact=True)
        m.set_continuity_merid(True)
        if rem:
            m.set_visc_remnant(True)   # buffers start at 1; no vertvisc runs
            assert (m.get("visc_rem_u") == 1.0).all() and (m.get("visc_rem_v") == 1.0).all()
        rng = np.random.default_rng(3)
        f = "u" if direction == "x" else "v"
        m.set(f, np.asfortranarray(m.get(f) + rng.normal(0, 0.3, size=m.get(f).shape)))
        m.continuity_pass(direction, 600.0)
        names = ["h", "uh", "hu_bt"] + BT_U if direction == "x" else ["h", "vh", "hv_bt"] + BT_V
        out.append({n: m.get(n) for n in names})
    for n in out[0]:
        assert np.array_equal(out[0][n], out[1][n]), n


@pytest.mark.gpu
def test_remnant_is_refused_in_the_mixed_form():
    from hackathon_mom6_miniapp_b200 import MIXED, Model, Mom6bError
    m = Model(*SHAPE, 30, INIT_CFG, seed=1, precision=MIXED, exact=True)
    with pytest.raises(Mom6bError):
        m.set_visc_remnant(True)


@pytest.mark.gpu
def test_remnant_steps_at_180x180x75():
    """The remnant path at the configs' small size, bit for bit."""
    from hackathon_mom6_miniapp_b200 import Model
    m = Model(180, 180, 75, 30, INIT_CFG, seed=12, exact=True)
    o = Oracle(180, 180, 75, 30, INIT_CFG, seed=12, threads=0)
    m.set_visc_remnant(True)
    o.set_remnant(True)
    m.step(2)
    o.step(2)
    for f in ["h", "u", "v", "eta", "hu_bt", "visc_rem_u", "visc_rem_v"] + BT_U:
        assert np.array_equal(m.get(f), o.get(f)), f
