"""Comparison helpers shared by the parity tests."""
import numpy as np


def rel_l2(a, b):
    """Relative L2 error of a against the reference b."""
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return d / n if n > 0 else d


def describe(a, b):
    d = np.abs(a - b)
    idx = np.unravel_index(np.argmax(d), d.shape)
    return (f"max|diff|={d.max():.3e} at {tuple(int(x) + 1 for x in idx)} "
            f"(1-based), rel_l2={rel_l2(a, b):.3e}, "
            f"n_diff={int(np.count_nonzero(a != b))}/{a.size}")


def face_range_u(m):
    """Slices of the continuity face range I in [is-1, ie], j in [js, je]."""
    return (slice(m.is_ - 2, m.ie), slice(m.js - 1, m.je))
