"""The learned barotropic surrogate.

The network's tensor-core kernels against the CPU oracle (oracle/mlp_oracle.py):
outputs, loss and the gradient of every parameter block; one Adam step;
prediction on ragged batch sizes.  Then the surrogate inside a model: training
lowers the loss, eta advanced from the predicted transports conserves volume,
the shadow run falls back to the plain btstep (whose results the model then
carries exactly), and what the trained network gains over the method without
it (the untrained network, and skipping the barotropic update)."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo
from tests.util import rel_l2

BLOCKS = {"W1": (mo.OFF_W1, mo.OFF_B1), "b1": (mo.OFF_B1, mo.OFF_W2),
          "W2": (mo.OFF_W2, mo.OFF_B2), "b2": (mo.OFF_B2, mo.OFF_W3),
          "W3": (mo.OFF_W3, mo.OFF_B3), "b3": (mo.OFF_B3, mo.NPARAMS)}


def _batch(B, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(B, mo.IN)).astype(np.float32)
    # a smooth target the network can learn
    Y = np.stack([np.tanh(X[:, :10].sum(1) / 3), 0.5 * X[:, 20] * X[:, 30]], 1).astype(np.float32)
    return X, Y


@pytest.mark.gpu
@pytest.mark.parametrize("B", [1024, 136])
def test_gradients_match_cpu_oracle(B):
    from hackathon_mom6_miniapp_b200 import Mlp
    net = Mlp(batch=1024, seed=3)
    p = net.params()
    X, Y = _batch(B, seed=B)
    g, loss, out = net.gradients(X, Y)
    lo, go, oo = mo.gradients(p, X, Y)
    assert rel_l2(out, oo) < 2e-3
    assert loss == pytest.approx(lo, rel=2e-3)
    for name, (a, b) in BLOCKS.items():
        assert rel_l2(g[a:b], go[a:b]) < 2e-2, (name, rel_l2(g[a:b], go[a:b]))
    # the padded input column of W1 gets no gradient
    assert np.all(g[mo.OFF_W1:mo.OFF_B1].reshape(mo.HID, mo.IN_PAD)[:, mo.IN] == 0)


@pytest.mark.gpu
def test_adam_step_matches_cpu_oracle():
    from hackathon_mom6_miniapp_b200 import Mlp
    net = Mlp(batch=512, seed=5)
    p = net.params()
    X, Y = _batch(512, seed=9)
    g, _, _ = net.gradients(X, Y)
    net.train(X, Y, lr=1e-3, nsteps=1)
    p1 = net.params()
    # the oracle's Adam step from the GPU's own gradient
    po, _, _ = mo.adam_step(p, g, np.zeros_like(p), np.zeros_like(p), 1, 1e-3)
    assert np.max(np.abs(p1 - po)) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 300, 2048])
def test_predict_matches_cpu_oracle(n):
    from hackathon_mom6_miniapp_b200 import Mlp
    net = Mlp(batch=256, seed=2)
    X, _ = _batch(n, seed=n)
    out = net.predict(X)
    oo, _ = mo.forward(net.params(), X)
    assert rel_l2(out, oo) < 2e-3


@pytest.mark.gpu
def test_training_on_a_fixed_batch_lowers_the_loss():
    from hackathon_mom6_miniapp_b200 import Mlp
    net = Mlp(batch=2048, seed=1)
    X, Y = _batch(2048, seed=4)
    losses = net.train(X, Y, lr=3e-3, nsteps=300)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.1 * losses[0], (losses[0], losses[-1])


def _model(**kw):
    from hackathon_mom6_miniapp_b200 import INIT_CFG, Model
    args = dict(ni=96, nj=80, nk=4, bt_nsteps=50, init_mode=INIT_CFG, seed=0, dt=600.0)
    args.update(kw)
    return Model(args.pop("ni"), args.pop("nj"), args.pop("nk"), args.pop("bt_nsteps"),
                 args.pop("init_mode"), **args, exact=True)


def _volume(m):
    eta = m.get("eta")
    return float(eta[m.is_ - 1:m.ie, m.js - 1:m.je].sum())


@pytest.fixture(scope="module")
def trained_params():
    m = _model()
    stats = m.surrogate_train(nstates=3, nsteps=150, batch=4096, lr=1e-3, seed=7)
    p = m.surrogate_params()
    st = m.surrogate_status()
    m.close()
    return p, stats, st


@pytest.mark.gpu
def test_surrogate_training_lowers_the_loss(trained_params):
    _, stats, st = trained_params
    assert stats["batches"] == 3 * 150 * 2
    assert np.isfinite(stats["loss_last"])
    assert stats["loss_last"] < 0.2 * stats["loss_first"], stats
    assert st["train_batches"] == stats["batches"]


@pytest.mark.gpu
def test_surrogate_conserves_volume(trained_params):
    p, _, _ = trained_params
    m = _model()
    m.set_surrogate_params(p)
    m.surrogate_enable(True, shadow_every=0)
    v0 = _volume(m)
    m.step(5)
    m.synchronize()
    v1 = _volume(m)
    eta = m.get("eta")
    assert np.all(np.isfinite(eta))
    assert abs(v1 - v0) <= 1e-12 * np.abs(eta).sum(), (v0, v1)
    st = m.surrogate_status()
    assert st["enabled"] == 1 and st["fallen_back"] == 0 and st["steps"] == 5


@pytest.mark.gpu
def test_shadow_run_falls_back_to_the_plain_btstep(trained_params):
    p, _, _ = trained_params
    plain = _model()
    plain.step(3)
    m = _model()
    m.set_surrogate_params(p)
    m.surrogate_enable(True, shadow_every=1, threshold=1e-14)
    m.step(3)
    st = m.surrogate_status()
    assert st["fallen_back"] == 1 and st["fallbacks"] == 1 and st["shadow_checks"] == 1
    assert st["last_shadow_error"] > 1e-14
    # the first step's plain results were kept and the plain btstep ran after
    for f in ("eta", "ubt_av", "vbt_av", "eta_av", "h", "u"):
        assert np.array_equal(m.get(f), plain.get(f)), f


@pytest.mark.gpu
def test_trained_network_gains_over_the_method_without_it(trained_params):
    """On a barotropic state the training never saw, the trained network's
    substep-averaged transports are closer to the plain btstep's than those
    of the same network untrained or of no transport at all (the barotropic
    update left out).  Its eta after a few steps is printed beside
    the same two, for the record: a 5 x 5 stencil sees +-2 cells while gravity
    waves cross about 12 cells in one barotropic call here, which is why the
    shadow run is the check of the multi-step error."""
    p, _, _ = trained_params
    errs, eta_errs = {}, {}
    nsteps = 4
    plain = _model()
    eta0 = plain.get("eta")
    plain.step(nsteps)
    want = plain.get("eta")
    for name, params in (("trained", p), ("untrained", None)):
        m = _model()
        if params is None:
            m.surrogate_train(nstates=1, nsteps=1, batch=128, lr=0.0, seed=7)  # untouched weights
        else:
            m.set_surrogate_params(params)
        ev = m.surrogate_eval(seed=7, state=50, nsteps=5)
        errs[name] = ev["rel_error"]
        errs["zero transport"] = ev["zero_prediction_error"]
        m.surrogate_enable(True, shadow_every=0)
        m.step(nsteps)
        eta_errs[name] = rel_l2(m.get("eta"), want)
        m.close()
    eta_errs["no barotropic update"] = rel_l2(eta0, want)
    print("held-out transport rel L2:", {k: f"{v:.3e}" for k, v in errs.items()})
    print("eta rel L2 after", nsteps, "steps:", {k: f"{v:.3e}" for k, v in eta_errs.items()})
    # a modest gain on this small basin after a short training (the 720 x 720
    # bench trains on the full set); the stencil's reach bounds how far it can go
    assert errs["trained"] < 0.8 * errs["untrained"], errs
    assert errs["trained"] < 0.97 * errs["zero transport"], errs
