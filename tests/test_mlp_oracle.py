"""The CPU restatement of the surrogate network checks itself before it
checks the GPU: its bf16 rounding equals torch's bfloat16 conversion, and its
backward pass equals finite differences of its forward pass (with the bf16
rounding switched off, in float64)."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(size=10000).astype(np.float32) * 10.0 ** rng.integers(-8, 8, 10000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 65504.0], np.float32)])
    want = torch.from_numpy(x.astype(np.float32)).to(torch.bfloat16).float().numpy()
    assert np.array_equal(mo.bf16(x), want)


def test_gelu_grad_is_the_derivative_of_gelu(monkeypatch):
    monkeypatch.setattr(mo, "FT", np.float64)
    z = np.linspace(-6, 6, 2001)
    h = 1e-6
    fd = (mo.gelu(z + h) - mo.gelu(z - h)) / (2 * h)
    assert np.max(np.abs(fd - mo.gelu_grad(z))) < 1e-7


def test_backward_matches_finite_differences(monkeypatch):
    # exact arithmetic version of the same network: no bf16 rounding, float64
    monkeypatch.setattr(mo, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    monkeypatch.setattr(mo, "FT", np.float64)
    rng = np.random.default_rng(1)
    B = 6
    X = rng.normal(size=(B, mo.IN))
    Y = rng.normal(size=(B, mo.OUT))
    p = rng.normal(size=mo.NPARAMS) * 0.05
    p[mo.OFF_W1:mo.OFF_B1].reshape(mo.HID, mo.IN_PAD)[:, mo.IN] = 0.0

    def f(pp):
        out, _ = mo.forward(pp, X)
        return float(np.sum((out - Y) ** 2) / (2 * B))

    loss, g, _ = mo.gradients(p, X, Y)
    assert loss == pytest.approx(f(p), rel=1e-5)
    idx = np.concatenate([rng.integers(mo.OFF_W1, mo.OFF_B1, 8), rng.integers(mo.OFF_B1, mo.OFF_W2, 4),
                          rng.integers(mo.OFF_W2, mo.OFF_B2, 8), rng.integers(mo.OFF_B2, mo.OFF_W3, 4),
                          rng.integers(mo.OFF_W3, mo.OFF_B3, 4), np.arange(mo.OFF_B3, mo.NPARAMS)])
    for k in idx:
        if mo.OFF_W1 <= k < mo.OFF_B1 and (k - mo.OFF_W1) % mo.IN_PAD == mo.IN:
            continue
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (f(p + e) - f(p - e)) / 2e-6
        assert abs(fd - g[k]) <= 1e-5 * max(abs(fd), 1e-3), (k, fd, g[k])


def test_adam_step_moves_against_the_gradient():
    p = np.zeros(4, np.float32)
    g = np.array([1.0, -2.0, 0.0, 3.0], np.float32)
    p1, m, v = mo.adam_step(p, g, np.zeros(4, np.float32), np.zeros(4, np.float32), 1, 1e-3)
    # first step: m_hat / sqrt(v_hat) = sign(g)
    assert np.allclose(p1, -1e-3 * np.sign(g), atol=1e-9)
