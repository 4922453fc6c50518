"""The reference's CUDA C host side, driven through the launch_* ABI.

The C++ mirror of rk2_cuda_c_driver and the src/cuda_c Fortran wrappers
(mom6b_cudac_*) runs a whole split RK2 iteration through the 27 entry points
those wrappers call.  Driving this library's entry points and driving the
reference's own kernels (built from their sources without FMA contraction,
oracle/_ref/libref_cuda_c_nofma.so) through the same mirror must give the
same state bit for bit, step after step: the drop-in boundary reproduces the
reference CUDA C backend's answers.
"""
import json
import os
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_NOFMA = os.path.join(ROOT, "oracle", "_ref", "libref_cuda_c_nofma.so")
REF_FMA = os.path.join(ROOT, "oracle", "_ref", "libref_cuda_c.so")
FIELDS = ["u", "v", "h", "uh", "up", "vp", "eta", "ubt_av", "vbt_av", "eta_av", "hu_bt",
          "FA_u_W0", "FA_u_WW", "FA_u_E0", "FA_u_EE", "uBT_WW", "uBT_EE", "taux_bot"]


def _need(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.relpath(path, ROOT)} not built (make -C oracle ref)")


@pytest.mark.gpu
@pytest.mark.parametrize("defer", [True, False])
@pytest.mark.parametrize("shape", [(36, 30, 8, 20), (70, 50, 12, 30)])
def test_abi_step_matches_reference_kernels(shape, defer):
    """Whole steps through the mirror, bit for bit against the reference's
    kernels: with the barotropic deferral (each btstep_cuda_c as one
    persistent loop) and with every launch_bt_* call run as it comes."""
    _need(REF_NOFMA)
    from hackathon_mom6_miniapp_b200 import CudaCDriver, abi_set_deferral
    abi_set_deferral(defer)
    ni, nj, nk, bt = shape
    ours = CudaCDriver(ni, nj, nk, bt, dt=300.0)
    ref = CudaCDriver(ni, nj, nk, bt, dt=300.0, kernel_lib=REF_NOFMA)
    for step in range(3):
        ours.step(1)
        ref.step(1)
        bad = [f for f in FIELDS if not np.array_equal(ours.get(f), ref.get(f))]
        assert not bad, f"step {step + 1}: fields differ: {bad}"
    abi_set_deferral(True)


@pytest.mark.gpu
def test_abi_step_180x180x75_matches_reference_kernels():
    _need(REF_NOFMA)
    from hackathon_mom6_miniapp_b200 import CudaCDriver
    ours = CudaCDriver(180, 180, 75, 30, dt=300.0)
    ref = CudaCDriver(180, 180, 75, 30, dt=300.0, kernel_lib=REF_NOFMA)
    ours.step(2)
    ref.step(2)
    for f in ("u", "v", "h", "eta", "ubt_av", "vbt_av"):
        assert np.array_equal(ours.get(f), ref.get(f)), f


@pytest.mark.gpu
def test_abi_step_conserves_mass():
    from hackathon_mom6_miniapp_b200 import CudaCDriver
    d = CudaCDriver(36, 30, 8, 20, dt=300.0)
    h0 = d.get("h0")[3:-3, 3:-3].sum()
    d.step(3)
    h = d.get("h")[3:-3, 3:-3].sum()
    # continuity is zonal only: the interior gains/loses only through the
    # i-boundary faces, which carry O(1e-6) of the volume per step here
    assert abs(h - h0) / h0 < 1e-3
    assert np.isfinite(d.get("u")).all() and np.isfinite(d.get("eta")).all()


def _steps_per_s(step, sync, n):
    step(2)
    sync()
    t0 = time.perf_counter()
    step(n)
    sync()
    return n / (time.perf_counter() - t0)


@pytest.mark.gpu
def test_speed_against_reference_cuda_c_backend():
    """steps/s at 720x720x75, bt_nsteps = 50 on this GPU: the reference CUDA C
    backend (its kernels built with the reference's own flags, driven by the
    mirror of its host side), this library's drop-in ABI path (same mirror,
    this library's entry points) and the fused graph path.  Wall-clock over a
    few steps, each path synchronised at its end; written to the JSON file
    named by MOM6B_SPEED_OUT when that is set."""
    _need(REF_FMA)
    import torch
    from hackathon_mom6_miniapp_b200 import CudaCDriver, INIT_CFG, Model
    n = int(os.environ.get("MOM6B_SPEED_STEPS", "5"))
    sync = torch.cuda.synchronize
    res = {"workload": "720x720x75 bt50 FP64", "steps": n}
    ref = CudaCDriver(720, 720, 75, 50, dt=300.0, kernel_lib=REF_FMA)
    res["reference_cuda_c_steps_per_s"] = _steps_per_s(ref.step, sync, n)
    ref.close()
    abi = CudaCDriver(720, 720, 75, 50, dt=300.0)
    res["abi_dropin_steps_per_s"] = _steps_per_s(abi.step, sync, n)
    abi.close()
    m = Model(720, 720, 75, 50, INIT_CFG, use_graph=True)
    res["fused_graph_steps_per_s"] = _steps_per_s(m.step, m.synchronize, 4 * n)
    m.close()
    out = os.environ.get("MOM6B_SPEED_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(res, f, indent=1)
    print(json.dumps(res))
    assert res["fused_graph_steps_per_s"] >= res["reference_cuda_c_steps_per_s"]
