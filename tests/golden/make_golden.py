"""Generate the small oracle fixtures committed in tests/golden.

The reference ships no golden vectors for this path (no tests at all), and
its serial Fortran cannot be compiled in this environment (no Fortran
compiler).  These fixtures therefore pin the oracle restatement against
regressions; they were produced by this script from oracle/liboracle.so:

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.pyoracle import INIT_CFG, INIT_REF, Oracle  # noqa: E402

CASES = {
    "ref_20x16x5": dict(mode=INIT_REF, ni=20, nj=16, nk=5, bt_nsteps=30, seed=0,
                        dt=300.0, nsteps=3),
    "cfg_20x16x5": dict(mode=INIT_CFG, ni=20, nj=16, nk=5, bt_nsteps=40, seed=11,
                        dt=600.0, nsteps=3),
    # odd small grids: every range edge close to every other
    "ref_13x11x5": dict(mode=INIT_REF, ni=13, nj=11, nk=5, bt_nsteps=30, seed=0,
                        dt=300.0, nsteps=3),
    "cfg_13x11x5": dict(mode=INIT_CFG, ni=13, nj=11, nk=5, bt_nsteps=31, seed=5,
                        dt=600.0, nsteps=3),
    "ref_36x30x8": dict(mode=INIT_REF, ni=36, nj=30, nk=8, bt_nsteps=30, seed=0,
                        dt=300.0, nsteps=3),
    "cfg_36x30x8": dict(mode=INIT_CFG, ni=36, nj=30, nk=8, bt_nsteps=31, seed=7,
                        dt=600.0, nsteps=3),
}
FIELDS = ("h", "u", "v", "eta", "ubt_av", "vbt_av")

# 180x180x75 is too large to commit as arrays: the SHA-256 of each field's
# bytes (float64, Fortran order, halos included) after nsteps steps
HASH_CASES = {
    "ref_180x180x75": dict(mode=INIT_REF, ni=180, nj=180, nk=75, bt_nsteps=30, seed=0,
                           dt=300.0, nsteps=3),
    "cfg_180x180x75": dict(mode=INIT_CFG, ni=180, nj=180, nk=75, bt_nsteps=31, seed=0,
                           dt=600.0, nsteps=3),
}


def field_hash(a):
    return hashlib.sha256(np.asfortranarray(a, dtype="<f8").tobytes(order="F")).hexdigest()

if __name__ == "__main__":
    for name, c in CASES.items():
        o = Oracle(c["ni"], c["nj"], c["nk"], c["bt_nsteps"], c["mode"], seed=c["seed"],
                   dt=c["dt"])
        o.step(c["nsteps"])
        out = {k: np.asarray(v) for k, v in c.items() if k != "mode"}
        for n in FIELDS:
            out[n] = o.get(n)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {k: float(np.abs(out[k]).max()) for k in ("h", "u", "v", "eta")})
    hashes = {}
    for name, c in HASH_CASES.items():
        o = Oracle(c["ni"], c["nj"], c["nk"], c["bt_nsteps"], c["mode"], seed=c["seed"],
                   dt=c["dt"], threads=0)
        o.step(c["nsteps"])
        hashes[name] = dict(c, fields={n: field_hash(o.get(n)) for n in FIELDS})
        print(name, hashes[name]["fields"]["h"][:16])
    with open(os.path.join(HERE, "hashes_180x180x75.json"), "w") as f:
        json.dump(hashes, f, indent=1, sort_keys=True)
