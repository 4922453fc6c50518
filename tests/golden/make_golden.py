"""Generate the small oracle fixtures committed in tests/golden.

The reference ships no golden vectors for this path (no tests at all), and
its serial Fortran cannot be compiled in this environment (no Fortran
compiler).  These fixtures therefore pin the oracle restatement against
regressions; they were produced by this script from oracle/liboracle.so:

    python tests/golden/make_golden.py
"""
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
}

for name, c in CASES.items():
    o = Oracle(c["ni"], c["nj"], c["nk"], c["bt_nsteps"], c["mode"], seed=c["seed"],
               dt=c["dt"])
    o.step(c["nsteps"])
    out = {k: np.asarray(v) for k, v in c.items() if k != "mode"}
    for n in ("h", "u", "v", "eta", "ubt_av", "vbt_av"):
        out[n] = o.get(n)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, {k: float(np.abs(out[k]).max()) for k in ("h", "u", "v", "eta")})
