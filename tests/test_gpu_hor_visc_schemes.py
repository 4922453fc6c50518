"""hor_visc's scheme branches (mom6_hor_visc_serial.F90:464-1109) in the
fused FP64 step: the general hor_visc kernel followed by the tendency on its
accelerations, against the oracle's restatement of the serial module, bit for
bit over whole steps.  The options are hor_visc_init's (:160-193) plus
modified_Leith; the background viscosities are chosen so that the branch
under test sets the viscosity (Kh = 0 or Ah = 0 leaves Smagorinsky or Leith
in charge), and the bound cases run on a 100 m grid where the bounds bind.
The grid is all ocean (init_ocean_grid's masks are 1), where no-slip and
free-slip shear coincide; the no-slip case still runs the no-slip code."""
import numpy as np
import pytest

from oracle.pyoracle import INIT_CFG, Oracle

SHAPE = (40, 28, 5)
CASES = {
    "biharmonic": (dict(biharmonic=True), {}),
    "biharmonic_only": (dict(laplacian=False, biharmonic=True), {}),
    "smagorinsky": (dict(smagorinsky=True), dict(Kh=0.0)),
    "smagorinsky_biharmonic": (dict(biharmonic=True, smagorinsky=True, Ah=0.0), dict(Kh=0.0)),
    "leith": (dict(leith=True), dict(Kh=0.0)),
    "leith_biharmonic": (dict(biharmonic=True, leith=True, Ah=0.0), dict(Kh=0.0)),
    "modified_leith_no_slip": (dict(biharmonic=True, leith=True, modified_leith=True,
                                    no_slip=True, Ah=0.0), dict(Kh=0.0)),
    "no_slip": (dict(no_slip=True), {}),
    "inviscid": (dict(laplacian=False), {}),
    # 100 m grid: Kh_Max = 0.25 areaT = 2500 m2 s-1 and hrat_min spreads over
    # about [0.97, 1], so Kh = 2480 is bounded at some points and not at
    # others, and the biharmonic Ah is held to the budget Kh leaves
    "better_bound": (dict(biharmonic=True, smagorinsky=True, better_bound=True),
                     dict(Kh=2480.0, dx_km=0.1, dt=0.25)),
    "better_bound_laplacian": (dict(smagorinsky=True, leith=True, better_bound=True),
                               dict(Kh=2480.0, dx_km=0.1, dt=0.5)),
    "better_bound_biharmonic_only": (dict(laplacian=False, biharmonic=True, better_bound=True),
                                     dict(dx_km=0.1, dt=0.25)),
}
FIELDS = ["u", "v", "h", "eta", "ubt_av", "vbt_av", "up", "vp"]


def _pair(opts, cfg, seed=4, bc_fill=None, nsteps=3, general_metrics=False):
    from hackathon_mom6_miniapp_b200 import Model
    m = Model(*SHAPE, 30, INIT_CFG, seed=seed, bc_fill=bc_fill, **cfg, exact=True,
              general_metrics=general_metrics)
    o = Oracle(*SHAPE, 30, INIT_CFG, seed=seed, bc_fill=bc_fill, **cfg)
    m.set_hor_visc(**opts)
    o.set_hor_visc(**opts)
    m.step(nsteps)
    o.step(nsteps)
    return m, o


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_scheme_steps_match_the_oracle(case):
    opts, cfg = CASES[case]
    m, o = _pair(opts, cfg)
    for f in FIELDS:
        a, b = m.get(f), o.get(f)
        assert np.isfinite(a).all(), f
        assert np.array_equal(a, b), (f, float(np.abs(a - b).max()))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["modified_leith_no_slip", "better_bound"])
def test_scheme_steps_with_metric_arrays(case):
    """The kernel's 2-D metric form (the uniform grid read through its arrays)
    gives the same steps."""
    opts, cfg = CASES[case]
    m, o = _pair(opts, cfg, general_metrics=True)
    for f in FIELDS:
        assert np.array_equal(m.get(f), o.get(f)), f


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["biharmonic", "leith_biharmonic", "better_bound"])
def test_the_branch_changes_the_step(case):
    """The branch under test moves the solution away from the driver's
    Laplacian (the oracle without the option)."""
    opts, cfg = CASES[case]
    o = Oracle(*SHAPE, 30, INIT_CFG, seed=4, **cfg)
    o.step(3)
    m, _ = _pair(opts, cfg)
    assert not np.array_equal(m.get("u"), o.get("u"))


@pytest.mark.gpu
def test_background_dominated_smagorinsky_is_the_fused_laplacian():
    """With the CFG background Kh (1e3 m2 s-1) above every Smagorinsky value,
    the general kernel plus the external-viscosity tendency reproduce the
    fused Laplacian tendency bit for bit."""
    from hackathon_mom6_miniapp_b200 import Model
    a = Model(*SHAPE, 30, INIT_CFG, seed=9, exact=True)
    b = Model(*SHAPE, 30, INIT_CFG, seed=9, exact=True)
    b.set_hor_visc(smagorinsky=True)
    a.step(3)
    b.step(3)
    for f in FIELDS:
        assert np.array_equal(a.get(f), b.get(f)), f


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [2, 3])
def test_schemes_with_the_arakawa_coriolis(scheme):
    from hackathon_mom6_miniapp_b200 import Model
    opts = dict(biharmonic=True, smagorinsky=True, Ah=0.0)
    m = Model(*SHAPE, 30, INIT_CFG, seed=5, Kh=0.0, exact=True)
    o = Oracle(*SHAPE, 30, INIT_CFG, seed=5, Kh=0.0)
    for x in (m, o):
        x.set_hor_visc(**opts)
        x.set_coriolis_scheme(scheme)
        x.step(2)
    for f in FIELDS:
        assert np.array_equal(m.get(f), o.get(f)), f


@pytest.mark.gpu
def test_driver_diagnostics_with_a_scheme(tmp_path):
    """The predictor's diffu, diffv of the general kernel are what the
    driver's diffu_sum / diffv_sum posts sum."""
    from hackathon_mom6_miniapp_b200 import Model
    from hackathon_mom6_miniapp_b200.diag_format import dump_name, read_bin
    opts = dict(biharmonic=True, leith=True, Ah=0.0)
    m = Model(*SHAPE, 30, INIT_CFG, seed=2, Kh=0.0, exact=True)
    o = Oracle(*SHAPE, 30, INIT_CFG, seed=2, Kh=0.0)
    m.set_hor_visc(**opts)
    o.set_hor_visc(**opts)
    m.diag_init(tmp_path, 1)
    m.diag_driver(2)
    o.diag_enable()
    m.step(1)
    m.synchronize()
    o.step(1)
    c = (slice(o.is_ - 1, o.ie), slice(o.js - 1, o.je))
    for n, name in ((1, "diffu_sum"), (2, "diffv_sum")):
        assert np.array_equal(read_bin(dump_name(tmp_path, name, n)), o.diag_get(name)[c]), name


@pytest.mark.gpu
def test_schemes_are_refused_in_the_mixed_form():
    from hackathon_mom6_miniapp_b200 import MIXED, Model, Mom6bError
    m = Model(*SHAPE, 30, INIT_CFG, seed=1, precision=MIXED, exact=True)
    m.set_hor_visc()                       # the driver's options stay available
    with pytest.raises(Mom6bError):
        m.set_hor_visc(biharmonic=True)


@pytest.mark.gpu
def test_all_schemes_at_180x180x75():
    """Every branch at once at the configs' small size, bit for bit."""
    from hackathon_mom6_miniapp_b200 import Model
    opts = dict(biharmonic=True, smagorinsky=True, leith=True, modified_leith=True,
                better_bound=True, Ah=1.0e9)
    m = Model(180, 180, 75, 30, INIT_CFG, seed=11, Kh=0.0, exact=True)
    o = Oracle(180, 180, 75, 30, INIT_CFG, seed=11, Kh=0.0, threads=0)
    m.set_hor_visc(**opts)
    o.set_hor_visc(**opts)
    m.step(2)
    o.step(2)
    for f in FIELDS:
        assert np.array_equal(m.get(f), o.get(f)), f
