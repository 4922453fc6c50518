"""The mini-app's raw binary dump format (mom6_diag.F90:362-431) and the
number format of its statistics line, for files written by the library's
diagnostics (Model.diag_*) and checkpoints (Model.write_field_bin).

A file holds the dimensions of the computational domain as 32-bit integers
(ni, nj for a 2-D field, ni, nj, nk for a 3-D one) followed by the values as
64-bit floats in column-major order.  The file does not say whether it is
2-D or 3-D; its size does.
"""
import os

import numpy as np

__all__ = ["read_bin", "write_bin", "es14_6", "stats_line", "dump_name"]


def read_bin(path):
    """The field of a dump as a Fortran-ordered float64 array (ni, nj[, nk])."""
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        hdr2 = np.frombuffer(f.read(8), dtype="<i4")
        ni, nj = int(hdr2[0]), int(hdr2[1])
        if size == 8 + 8 * ni * nj:
            shape = (ni, nj)
        else:
            nk = int(np.frombuffer(f.read(4), dtype="<i4")[0])
            if size != 12 + 8 * ni * nj * nk:
                raise ValueError(f"{path}: size {size} does not match its header")
            shape = (ni, nj, nk)
        data = np.frombuffer(f.read(), dtype="<f8")
    return data.reshape(shape, order="F").copy(order="F")


def write_bin(path, a):
    """Write a 2-D or 3-D array (its values in column-major order)."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim not in (2, 3):
        raise ValueError("a 2-D or 3-D field")
    with open(path, "wb") as f:
        f.write(np.asarray(a.shape, dtype="<i4").tobytes())
        f.write(np.asfortranarray(a).tobytes(order="F"))


def es14_6(x):
    """Fortran ES14.6 edit of one value: d.ddddddE+ee right-justified in 14
    characters; a three-digit exponent is written without its letter."""
    x = float(x)
    if np.isnan(x):
        return "%14s" % "NaN"
    if np.isinf(x):
        return "%14s" % ("Infinity" if x > 0 else "-Infinity")
    t = "%.6E" % x
    mant, exp = t.split("E")
    if len(exp) - 1 >= 3:
        t = mant + exp
    return "%14s" % t


def stats_line(name, stats):
    """The line post_data prints for (min, max, mean, rms)."""
    return "  Diag: " + name + " min/max/mean/rms: " + "".join(es14_6(v) for v in stats)


def dump_name(output_dir, name, call_count):
    """The file a post writes: <output_dir>/<name><call count, 6 digits>.bin."""
    num = "%06d" % call_count if call_count <= 999999 else "******"
    return str(output_dir) + "/" + name + num + ".bin"
