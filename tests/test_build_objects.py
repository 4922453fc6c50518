"""The exact (no-FMA) and the FMA translation units define disjoint kernels.

The FP64 kernels exist in two builds of the same templates: the exact form,
compiled without FMA contraction (bit-identical to the serial driver), and
the fast form, compiled with it.  If an FMA object instantiated a kernel with
the same template arguments as an exact object, the linker would keep one
copy of the weak symbol for both and the exact form could silently run FMA
code.  This checks the built objects: no kernel is defined in both sets.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "hackathon_mom6_miniapp_b200", "_build")


def _kernels(obj):
    out = subprocess.run(["nm", "-C", "--defined-only", obj], capture_output=True, text=True,
                         check=True).stdout
    names = set()
    for line in out.splitlines():
        parts = line.split(None, 2)
        if len(parts) == 3 and parts[1] in "TtWw" and "mom6b::k_" in parts[2]:
            names.add(parts[2])
    return names


def test_no_kernel_in_both_exact_and_fma_objects():
    if shutil.which("nm") is None or not os.path.isdir(BUILD):
        pytest.skip("no built objects or no nm")
    from hackathon_mom6_miniapp_b200 import build as b
    objs = {s: os.path.join(BUILD, s + ".o") for s in b.CU_SOURCES}
    if not all(os.path.exists(p) for p in objs.values()):
        pytest.skip("objects not built")
    exact, fma = {}, {}
    for s, p in objs.items():
        (fma if s in b.FMA_SOURCES else exact)[s] = _kernels(p)
    for se, ke in exact.items():
        for sf, kf in fma.items():
            both = ke & kf
            assert not both, f"{se} and {sf} both define {sorted(both)[:3]}"
