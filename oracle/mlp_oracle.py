"""CPU restatement of the barotropic surrogate network (test infrastructure).

This module is the oracle the GPU network is checked against: only tests/
may import it.  It restates, in numpy, the network of the library's
surrogate (hackathon_mom6_miniapp_b200/csrc/k_mlp.cu): a 175-256-256-2 MLP
with the tanh form of GELU, bf16 rounding (round to nearest even) at the
points where the GPU stores bf16 (inputs, weights W1 W2 W3, hidden
activations H1 H2, the backward dZ1 dZ2), fp32 sums elsewhere, the loss
sum (out - y)^2 / (2 B), and Adam with bias correction folded into the step
size.  The surrogate has no counterpart in the reference mini-app, so there
is nothing of the reference to pin it to: parity is with this restatement of
the published formulas (GELU: Hendrycks & Gimpel 2016; Adam: Kingma & Ba
2015).
"""
import numpy as np

IN, IN_PAD, HID, OUT = 175, 176, 256, 2
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * IN_PAD
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUT * HID
NPARAMS = OFF_B3 + OUT
C_GELU = 0.7978845608028654
# working type of every non-bf16 quantity (fp32 like the GPU; the self-checks
# switch it to float64 together with switching the bf16 rounding off)
FT = np.float32


def bf16(x):
    """Round fp32 values to the nearest bf16 (ties to even), kept as fp32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def gelu(z):
    z = np.asarray(z, dtype=FT)
    t = np.tanh(C_GELU * (z + 0.044715 * z * z * z))
    return 0.5 * z * (1.0 + t)


def gelu_grad(z):
    z = np.asarray(z, dtype=FT)
    z2 = z * z
    t = np.tanh(C_GELU * (z + 0.044715 * z2 * z))
    return 0.5 * (1 + t) + 0.5 * z * (1 - t * t) * C_GELU * (1 + 3 * 0.044715 * z2)


def unpack(p):
    p = np.asarray(p, dtype=FT)
    return dict(W1=p[OFF_W1:OFF_B1].reshape(HID, IN_PAD), b1=p[OFF_B1:OFF_W2],
                W2=p[OFF_W2:OFF_B2].reshape(HID, HID), b2=p[OFF_B2:OFF_W3],
                W3=p[OFF_W3:OFF_B3].reshape(OUT, HID), b3=p[OFF_B3:NPARAMS])


def _mm(a, b):
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(FT)


def forward(p, X):
    """Outputs [B][2] and the intermediates of a batch X [B][175]."""
    q = unpack(p)
    Xb = np.zeros((X.shape[0], IN_PAD), dtype=FT)
    Xb[:, :IN] = bf16(X)
    Z1 = _mm(Xb, bf16(q["W1"]).T) + q["b1"]
    H1 = bf16(gelu(Z1))
    Z2 = _mm(H1, bf16(q["W2"]).T) + q["b2"]
    H2 = bf16(gelu(Z2))
    W3r = bf16(q["W3"])
    out = _mm(H2, W3r.T) + q["b3"]
    return out, dict(Xb=Xb, Z1=Z1, H1=H1, Z2=Z2, H2=H2, W3r=W3r)


def gradients(p, X, Y):
    """(loss, gradient of every parameter in the flat layout, outputs)."""
    q = unpack(p)
    B = X.shape[0]
    out, c = forward(p, X)
    d = out - Y
    loss = float(np.sum(d.astype(np.float64) ** 2) / (2 * B))
    dOut = (d / B).astype(FT)
    dZ2 = bf16(_mm(dOut, c["W3r"]) * gelu_grad(c["Z2"]))
    g = np.zeros(NPARAMS, dtype=FT)
    g[OFF_W3:OFF_B3] = _mm(dOut.T, c["H2"]).ravel()
    g[OFF_B3:NPARAMS] = dOut.sum(axis=0, dtype=np.float64)
    g[OFF_B2:OFF_W3] = dZ2.sum(axis=0, dtype=np.float64)
    g[OFF_W2:OFF_B2] = _mm(dZ2.T, c["H1"]).ravel()
    dH1 = _mm(dZ2, bf16(q["W2"]))
    dZ1 = bf16(dH1 * gelu_grad(c["Z1"]))
    g[OFF_B1:OFF_W2] = dZ1.sum(axis=0, dtype=np.float64)
    g[OFF_W1:OFF_B1] = _mm(dZ1.T, c["Xb"]).ravel()
    return loss, g, out


def adam_step(p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (t counts from 1); returns new (p, m, v)."""
    m = np.float32(b1) * m + np.float32(1 - b1) * g
    v = np.float32(b2) * v + np.float32(1 - b2) * g * g
    lr_t = np.float32(lr * np.sqrt(1 - b2 ** t) / (1 - b1 ** t))
    return (p - lr_t * m / (np.sqrt(v) + np.float32(eps))).astype(np.float32), m, v
