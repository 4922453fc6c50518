"""The oracle's hor_visc scheme branches on the CPU (test infrastructure):
the driver's options reproduce the driver's step, a background viscosity
above every dynamic value reproduces the plain Laplacian, and setting the
options resets the module's work arrays as hor_visc_init does."""
import numpy as np

from oracle.pyoracle import INIT_CFG, Oracle

SHAPE = (24, 20, 4)


def _run(opts=None, nsteps=2, **cfg):
    o = Oracle(*SHAPE, 20, INIT_CFG, seed=3, **cfg)
    if opts is not None:
        o.set_hor_visc(**opts)
    o.step(nsteps)
    return o


def test_driver_options_are_the_driver_step():
    a, b = _run(), _run(dict())
    for f in ("u", "v", "h", "eta"):
        assert np.array_equal(a.get(f), b.get(f)), f


def test_background_above_smagorinsky_and_leith_is_the_laplacian():
    a = _run()
    b = _run(dict(smagorinsky=True, leith=True, modified_leith=True))
    for f in ("u", "v", "h"):
        assert np.array_equal(a.get(f), b.get(f)), f


def test_dynamic_viscosity_acts_without_background():
    a = _run(Kh=0.0)
    b = _run(dict(smagorinsky=True), Kh=0.0)
    c = _run(dict(leith=True), Kh=0.0)
    assert not np.array_equal(a.get("u"), b.get("u"))
    assert not np.array_equal(a.get("u"), c.get("u"))
    assert not np.array_equal(b.get("u"), c.get("u"))


def test_reset_restores_the_driver_step():
    o = Oracle(*SHAPE, 20, INIT_CFG, seed=3)
    o.set_hor_visc(biharmonic=True, leith=True, better_bound=True)
    o.set_hor_visc()
    o.step(2)
    a = _run()
    for f in ("u", "v", "h"):
        assert np.array_equal(a.get(f), o.get(f)), f
