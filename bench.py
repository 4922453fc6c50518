"""Benchmark: RK2 steps/s of the split RK2 step at 720x720x75, bt_nsteps=50.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the seeded beta-plane state at 720x720x75 (CFG init,
Philox4x32-10 normals, dt = 600 s, Kh = 1e3, halo fill on), ni = nj = 720,
nk = 75, bt_nsteps = 50, plain FP64 in its fast form (FMA contraction,
column sums in another order; within 1e-12 relative L2 of the serial driver,
tested).  The "exact_fp64" object times the exact form (bit-identical to the
serial driver) on the same protocol.  One "step" is one split RK2 iteration
of rk2_serial_driver.F90:218-399 on the whole domain.  The state (~6 GB)
stays resident in HBM and is far larger than L2, so no L2 flush is needed
between steps.  Under torchrun each rank advances its own replica of the
domain (the path does not shard across GPUs: replicas only, weak scaling);
the timed region is bracketed by a barrier and device synchronisation and
the time is the maximum over ranks.

The line's "reference_cuda_c" object times the reference's own CUDA C
backend on the same GPU and workload: its src/cuda_c kernels built from their
sources with the reference's -O3 for sm_100a (oracle/_ref), driven by a C++
mirror of rk2_cuda_c_driver and the src/cuda_c Fortran wrappers (same launch
sequence, arguments and per-phase device synchronisation).  "abi_dropin"
times this library's launch_* entry points through the same mirror: the path
an unchanged Fortran build of rk2_cuda_c_driver takes when it links this
library.  Both report the median per-step time over K steps after W warm-up
steps (CUDA events).

The "mixed" object measures the mixed-precision form (FP32 state, fluxes,
stencils and vertical-viscosity coefficients; FP64 column sums, thickness
update, vertical tridiagonal elimination and barotropic loop) on the same
workload and protocol, with its speed-up over the FP64 form, the same pair
at the mixed-form configuration 1440x1080x75 bt50, and its per-field
relative L2 error against the exact FP64 form of the same seed after 10 steps
at 720x720x75 and after 100 steps at 1440x1080x75.

The "ensemble" object advances 64 independent domains of uneven size
(ni = nj in {90, ..., 360}, nk in {25, 50, 75}, bt_nsteps = 31, mixed form)
together, one launch per phase for all of them with launch shapes from the
autotuner, reports aggregate cell-layer updates/s over 50 steps and checks
every domain for finite fields and conserved volume afterwards.

The "surrogate" object trains the learned barotropic surrogate on the GPU
(8 seeded states x 2000 steps of the plain btstep, batch 65536), reports its
transport error on a held-out state, and times the step with the network in
place of btstep: with the plain btstep as shadow check every 10 steps
(threshold 1e-3 relative eta error, falling back when exceeded) and alone,
with the network-alone eta error after 100 steps against the FP64 form.

--impl reference times the reference's CPU implementation of the path on the
host cores: the C restatement of the serial Fortran driver (the Fortran
itself cannot be compiled here), built with OpenMP over rows and run on all
host threads, on W untimed and K timed whole steps of the workload, on rank
0 only.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NI, NJ, NK, BT = 720, 720, 75, 50
N3 = (NI + 2) * (NJ + 2) * NK * 8
N2 = (NI + 2) * (NJ + 2) * 8
# algorithmic bytes of one RK2 step: 78 3-D + 30 2-D array touches of the
# reference's 16 phases (compulsory reads + writes per phase)
STEP_BYTES = 78 * N3 + 30 * N2
METRIC = "RK2 steps/s @720x720x75 bt50: plain FP64 vs mixed/learned at stated error"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []          # (host time the line arrived, line)
        self.t_begin = self.t_end = None

    def start(self):
        """Start sampling every 50 ms and wait (at most 5 s) for the first
        sample, so that the sampler runs before the timed region begins."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def begin(self):
        self.t_begin = time.time()

    def end(self):
        self.t_end = time.time()

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = [ln for t, ln in self.lines]
        if self.t_begin is not None and self.t_end is not None:
            # the samples that arrived while the timed region ran (a sample
            # reaches the reader a little after it is taken)
            inside = [ln for t, ln in self.lines if self.t_begin <= t <= self.t_end + 0.06]
            if inside:
                lines = inside
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


_DIST_DEVICE = "cpu"


def dist_setup(args, backend="nccl"):
    """One process per GPU (torchrun env vars).  The replicas share nothing:
    the process group only carries the timing barrier and reductions, with a
    short timeout so that ranks waiting for a failed peer end with an error."""
    global _DIST_DEVICE
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as td
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
            _DIST_DEVICE = f"cuda:{local}"
        else:
            _DIST_DEVICE = "cpu"
        td.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        dist = td
    return world, rank, local, dist


def _reduce(x, dist, op):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=_DIST_DEVICE)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, dist, local):
    return x if dist is None else _reduce(x, dist, dist.ReduceOp.MAX)


def sum_over_ranks(x, dist, local):
    return x if dist is None else _reduce(x, dist, dist.ReduceOp.SUM)


def barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_whole_steps(ni, nj, bt, nsteps, threads, warmup=1):
    """Time the oracle restatement of the serial driver on whole RK2 steps of
    the seeded ni x nj x 75 domain (dt 600 s): `warmup` untimed steps, then
    nsteps timed ones.  threads=None is the single-threaded build (the
    reference serial backend has no threading); threads=0 the OpenMP build of
    the same source on all host threads (rows in parallel, results
    identical)."""
    from oracle.pyoracle import INIT_CFG, Oracle
    o = Oracle(ni, nj, NK, bt, INIT_CFG, seed=0, dt=600.0, threads=threads)
    cores = o.threads
    if warmup:
        o.step(warmup)
    t0 = time.perf_counter()
    o.step(nsteps)
    dt = time.perf_counter() - t0
    o.close()
    what = "OpenMP over rows" if threads is not None else "single thread"
    return nsteps / dt, (f"{nsteps} whole RK2 steps of {ni}x{nj}x{NK} bt{bt} after {warmup} "
                         f"untimed ({dt:.1f} s, {what}, {cores} thread(s))"), cores


def cpu_baseline_line():
    """cpu_baseline: the oracle on all host threads on whole steps of the
    bench workload, and the single-thread build on whole steps of the
    180x180x75 case (a whole 720x720 step single-threaded takes about a
    minute)."""
    rn, sn, cores = cpu_whole_steps(NI, NJ, BT, 2, 0)
    r1, s1, _ = cpu_whole_steps(180, 180, 31, 2, None)
    return {"value": rn, "unit": "steps/s", "cores": cores, "kind": "port", "sample": sn,
            "single_thread_180x180x75": {"value": r1, "unit": "steps/s", "cores": 1,
                                         "sample": s1}}


def run_reference(args, world, rank, local, dist):
    """The reference's CPU implementation of the path (the oracle's C
    restatement of rk2_serial_driver, OpenMP over rows on all host threads)
    on the bench workload: args.warmup untimed whole steps, then args.steps
    timed whole steps.  Rank 0 only."""
    if rank != 0:
        return
    value, sample, cores = cpu_whole_steps(NI, NJ, BT, args.steps, 0, warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 / value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "split RK2 step 720x720x75 bt50 (seeded beta plane)",
                       "ni": NI, "nj": NJ, "nk": NK, "bt_nsteps": BT, "dt": 600.0},
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_cudac(kernel_lib, steps, warmup, local):
    """steps/s of the reference's CUDA C host side (the C++ mirror of
    rk2_cuda_c_driver and the src/cuda_c wrappers, per-phase device
    synchronisation included) on the bench workload (CFG state, dt 600 s,
    720x720x75, bt 50): kernel_lib None drives this library's launch_* entry
    points (the drop-in path), a path drives that library's (the reference's
    own kernels).  Median of per-step CUDA-event times after warm-up."""
    import numpy as np
    import torch
    from hackathon_mom6_miniapp_b200 import INIT_CFG, CudaCDriver
    d = CudaCDriver(NI, NJ, NK, BT, dt=600.0, kernel_lib=kernel_lib, init_mode=INIT_CFG,
                    seed=0)
    d.step(warmup)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        d.step(1)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    finite = bool(np.isfinite(d.get("h")).all() and np.isfinite(d.get("eta")).all())
    d.close()
    times.sort()
    med = times[len(times) // 2]
    return {"value": 1000.0 / med, "unit": "steps/s", "ms_per_step_median": med,
            "ms_per_step_min": times[0], "steps": steps, "warmup": warmup, "finite": finite,
            "config": {"ni": NI, "nj": NJ, "nk": NK, "bt_nsteps": BT, "dt": 600.0,
                       "init": "seeded beta plane (CFG), no halo fill"}}


def measured_traffic():
    """DRAM bytes per launch of each phase at the bench size, from the committed
    ncu summary (profiles/traffic_720x720x75.txt); {} when absent."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles",
                        "traffic_720x720x75.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            parts = line.split()
            if len(parts) == 2 and not line.startswith("#"):
                out[parts[0]] = float(parts[1])
    return out


MIXED_FIELDS = ("h", "u", "v", "eta", "ubt_av", "vbt_av")


def _rel_l2(a, b):
    import numpy as np
    d = float(np.linalg.norm((a - b).ravel()))
    n = float(np.linalg.norm(b.ravel()))
    return d / n if n > 0 else d


def mixed_errors(ni, nj, nsteps, seed, local):
    """Per-field relative L2 error of the mixed form against the FP64 form
    (bit-identical to the serial driver) after nsteps from the same seed."""
    from hackathon_mom6_miniapp_b200 import FP64, INIT_CFG, MIXED, Model
    ref = Model(ni, nj, NK, BT, INIT_CFG, seed=seed, dt=600.0, device=local,
                precision=FP64, use_graph=True)
    ref.step(nsteps)
    want = {f: ref.get(f) for f in MIXED_FIELDS}
    ref.close()
    mx = Model(ni, nj, NK, BT, INIT_CFG, seed=seed, dt=600.0, device=local,
               precision=MIXED, use_graph=True)
    mx.step(nsteps)
    errs = {f: _rel_l2(mx.get(f), want[f]) for f in MIXED_FIELDS}
    mx.close()
    return errs


def _finite(x):
    """x with every non-finite float replaced by None (null in the JSON line:
    NaN and Infinity are not JSON)."""
    if isinstance(x, float):
        return x if math.isfinite(x) else None
    if isinstance(x, dict):
        return {k: _finite(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [_finite(v) for v in x]
    return x


def _time_model(m, args, local, dist):
    """Device time of args.steps steps of a model after args.warmup, max over
    ranks (ms)."""
    m.step(args.warmup)
    m.synchronize()
    barrier(dist)
    return max_over_ranks(_timed_steps(m, args.steps, local), dist, local)


def run_mixed(args, world, rank, local, dist, fp64_ms_per_step):
    """The mixed form (FP32 state, fluxes, stencils and vertical-viscosity
    coefficients; FP64 column sums, thickness update, vertical elimination and
    barotropic loop) on the headline workload and timing protocol, and at the
    mixed-form configuration (1440x1080x75 bt50) beside the FP64 form of the
    same size, with its per-field errors."""
    from hackathon_mom6_miniapp_b200 import FP64, INIT_CFG, MIXED, Model
    m = Model(NI, NJ, NK, BT, INIT_CFG, seed=rank, dt=600.0, device=local,
              precision=MIXED, use_graph=not args.no_graph)
    ms = _time_model(m, args, local, dist)
    m.kernel_timing(True)
    m.step(2)
    m.synchronize()
    kt = {k: m.kernel_time_ms(k) for k in ("tendency", "vertvisc", "continuity", "btstep",
                                           "halo_fill")}
    m.close()
    out = {"value": world * args.steps / (ms / 1000.0), "unit": "steps/s",
           "ms_per_step": ms / args.steps,
           "speedup_vs_fp64": fp64_ms_per_step / (ms / args.steps),
           "kernel_ms_per_step": {k: v[0] * v[1] / 2 for k, v in kt.items()},
           "dtype": "f32 state/stencils/vertvisc coefficients, f64 column sums/thickness "
                    "update/vertical elimination/btstep"}
    if not args.no_cfg2:
        c2 = {}
        for name, prec in (("mixed", MIXED), ("fp64", FP64)):
            mm = Model(1440, 1080, NK, BT, INIT_CFG, seed=rank, dt=600.0, device=local,
                       precision=prec, use_graph=not args.no_graph)
            t = _time_model(mm, args, local, dist)
            mm.close()
            c2[name + "_steps_per_s"] = world * args.steps / (t / 1000.0)
            c2[name + "_ms_per_step"] = t / args.steps
        c2["speedup_vs_fp64"] = c2["fp64_ms_per_step"] / c2["mixed_ms_per_step"]
        c2["config"] = {"ni": 1440, "nj": 1080, "nk": NK, "bt_nsteps": BT, "dt": 600.0}
        out["config2_1440x1080x75"] = c2
    if rank == 0:
        out["rel_l2_720x720x75_10_steps"] = mixed_errors(NI, NJ, 10, 0, local)
        if not args.no_cfg2:
            out["rel_l2_1440x1080x75_100_steps"] = mixed_errors(1440, 1080, 100, 0, local)
        out["error_reference"] = ("exact FP64 form of the same seed (bit-identical to the "
                                  "oracle); eta, ubt_av, vbt_av come from the FP64 "
                                  "barotropic loop in both forms")
    return out


ENS_BT = 31


def ensemble_domains(n=64, seed=0):
    """The batched-ensemble configuration: n domains, square ni = nj drawn
    uniformly from {90, 120, ..., 360} and nk from {25, 50, 75}, each built
    like the 180x180 case (seeded beta plane, dt 600 s) with its own seed, at
    31 barotropic substeps: 30, the configured count, is unstable at dt
    600 s in the serial scheme itself (eta grows past 1e170 m in 50 steps),
    and 31 is the fewest that stay bounded."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = rng.choice(np.arange(90, 361, 30), size=n)
    depths = rng.choice(np.array([25, 50, 75]), size=n)
    return [dict(ni=int(a), nj=int(a), nk=int(k), bt_nsteps=ENS_BT, seed=q)
            for q, (a, k) in enumerate(zip(sizes, depths))]


def _ensemble_health(e):
    """Every domain finite after the run, and the largest relative change of
    its total volume (sum of h over the compute domain against h0's: the
    step conserves it with the periodic / wall halo fill)."""
    import numpy as np
    finite, worst = True, 0.0
    for d in range(len(e)):
        h, h0 = e.get(d, "h"), e.get(d, "h0")
        for n in ("u", "v", "eta"):
            finite = finite and bool(np.isfinite(e.get(d, n)).all())
        finite = finite and bool(np.isfinite(h).all())
        sl = (slice(3, -3), slice(3, -3))
        m0, m1 = float(h0[sl].sum()), float(h[sl].sum())
        worst = max(worst, abs(m1 - m0) / m0)
    return finite, worst


def run_ensemble(args, world, rank, local, dist):
    """64 uneven domains advanced together (one launch per phase for all of
    them, launch shapes from the autotuner): aggregate cell-layer updates/s
    over 50 steps, with every domain checked for finiteness and volume."""
    import torch
    from hackathon_mom6_miniapp_b200 import Ensemble
    doms = ensemble_domains(64, seed=rank)
    e = Ensemble(doms, device=local)
    t_tune = time.perf_counter()
    best = e.autotune(reps=2)
    t_tune = time.perf_counter() - t_tune
    stream = torch.cuda.ExternalStream(e.stream(), device=f"cuda:{local}")
    e.step(3)
    e.synchronize()
    barrier(dist)
    steps = 50
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    n0 = e.launch_count()
    e0.record(stream)
    e.step(steps)
    e1.record(stream)
    e.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, local)
    launches = e.launch_count() - n0
    cells = e.cell_layers()
    finite, mass_err = _ensemble_health(e)
    out = {"value": world * cells * steps / (ms / 1000.0), "unit": "cell-layer updates/s",
           "domains": len(doms), "steps": steps, "bt_nsteps": ENS_BT, "ms_per_step": ms / steps,
           "cell_layers": cells, "launches_per_step": launches / steps,
           "finite": finite, "max_rel_volume_change": mass_err,
           "tuning": e.tuning(), "autotune_best_ms": best, "autotune_s": t_tune,
           "sizes": "ni=nj from {90..360 step 30}, nk from {25,50,75}, numpy "
                    "default_rng(rank) draws, seeds 0..63",
           "dtype": "mixed form (f32 state/stencils, f64 column sums/thickness "
                    "update/vertical elimination/btstep)"}
    e.close()
    return out


def _timed_steps(m, steps, local):
    import torch
    stream = torch.cuda.ExternalStream(m.stream(), device=f"cuda:{local}")
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    m.step(steps)
    e1.record(stream)
    m.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def run_surrogate(args, world, rank, local, dist, fp64_ms_per_step):
    """The learned barotropic surrogate at 720x720x75 bt50: the network is
    trained on the GPU (8 seeded barotropic states x args.sur_steps RK2 steps
    of the plain btstep, batch 65536, Adam lr 1e-3), checked on a held-out
    state, then run in place of btstep with the plain btstep as shadow check
    (every 10 steps, relative eta error threshold 1e-3), and on its own."""
    from hackathon_mom6_miniapp_b200 import FP64, INIT_CFG, Model
    t = Model(NI, NJ, 2, BT, INIT_CFG, seed=rank, dt=600.0, device=local)
    train = t.surrogate_train(nstates=8, nsteps=args.sur_steps, batch=65536, lr=1e-3, seed=1)
    held = t.surrogate_eval(seed=1, state=100, nsteps=10)
    params = t.surrogate_params()
    t.close()
    out = {"training": dict(train, states=8, steps_per_state=args.sur_steps, batch=65536,
                            lr=1e-3),
           "heldout_transport_rel_l2": held["rel_error"],
           "heldout_zero_transport_rel_l2": held["zero_prediction_error"]}
    # with the shadow check
    m = Model(NI, NJ, NK, BT, INIT_CFG, seed=rank, dt=600.0, device=local, use_graph=True)
    m.set_surrogate_params(params)
    m.surrogate_enable(True, shadow_every=10, threshold=1e-3)
    m.step(args.warmup)
    m.synchronize()
    barrier(dist)
    ms = max_over_ranks(_timed_steps(m, args.steps, local), dist, local)
    st = m.surrogate_status()
    m.close()
    out.update({"value": world * args.steps / (ms / 1000.0), "unit": "steps/s",
                "ms_per_step": ms / args.steps,
                "speedup_vs_fp64": fp64_ms_per_step / (ms / args.steps),
                "shadow_every": 10, "threshold": 1e-3,
                "fallen_back": bool(st["fallen_back"]),
                "shadow_checks": st["shadow_checks"],
                "max_shadow_rel_error": st["max_shadow_error"]})
    # the network alone: speed, and eta after 100 steps against the plain form
    m = Model(NI, NJ, NK, BT, INIT_CFG, seed=rank, dt=600.0, device=local, use_graph=True)
    m.set_surrogate_params(params)
    m.surrogate_enable(True, shadow_every=0)
    m.step(args.warmup)
    m.synchronize()
    barrier(dist)
    ms_n = max_over_ranks(_timed_steps(m, args.steps, local), dist, local)
    m.close()
    pure = {"value": world * args.steps / (ms_n / 1000.0), "unit": "steps/s",
            "ms_per_step": ms_n / args.steps,
            "speedup_vs_fp64": fp64_ms_per_step / (ms_n / args.steps)}
    if rank == 0:
        a = Model(NI, NJ, NK, BT, INIT_CFG, seed=0, dt=600.0, device=local, use_graph=True,
                  precision=FP64)
        a.step(100)
        want = a.get("eta")
        a.close()
        b = Model(NI, NJ, NK, BT, INIT_CFG, seed=0, dt=600.0, device=local, use_graph=True)
        b.set_surrogate_params(params)
        b.surrogate_enable(True, shadow_every=0)
        b.step(100)
        pure["eta_rel_l2_100_steps"] = _rel_l2(b.get("eta"), want)
        b.close()
    out["network_alone"] = pure
    return out


def run_ours(args, world, rank, local, dist):
    import numpy as np
    import torch
    from hackathon_mom6_miniapp_b200 import INIT_CFG, Model
    torch.cuda.set_device(local)
    m = Model(NI, NJ, NK, BT, INIT_CFG, seed=rank, dt=600.0, device=local,
              use_graph=not args.no_graph)
    stream = torch.cuda.ExternalStream(m.stream(), device=f"cuda:{local}")
    # warm-up
    m.step(args.warmup)
    m.synchronize()
    barrier(dist)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    m.reset_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks.begin()
    e0.record(stream)
    m.step(args.steps)
    e1.record(stream)
    m.synchronize()
    torch.cuda.synchronize()
    clocks.end()
    launches = m.launch_count()
    ck = clocks.stop()
    ms_local = e0.elapsed_time(e1)
    barrier(dist)
    ms = max_over_ranks(ms_local, dist, local)
    value = world * args.steps / (ms / 1000.0)

    # per-kernel timing pass (events around every launch) for the roofline
    m.kernel_timing(True)
    m.step(max(2, min(args.steps, 5)))
    m.synchronize()
    kt = {}
    for name in ("tendency", "vertvisc", "continuity", "btstep", "halo_fill"):
        avg, n = m.kernel_time_ms(name)
        kt[name] = (avg, n)
    m.kernel_timing(False)
    steps_t = max(2, min(args.steps, 5))
    per_step_ms = {k: v[0] * v[1] / steps_t for k, v in kt.items()}
    dom = max(per_step_ms, key=per_step_ms.get)
    # algorithmic bytes per launch: the reference phases each fused kernel
    # covers (per step 78 N3 + 30 N2 = STEP_BYTES, split evenly over the
    # predictor and corrector launches):
    #   tendency   = h reset (2, predictor only) + transports 5 + hor_visc 5
    #                + CorAdCalc 7 + velocity update 8 -> 26 N3 on average
    #   vertvisc   = 7 N3 + 2 N2
    #   continuity = 5 N3 + 7 N2 (+ the corrector's htmp copy 2 N3) -> 6 N3 + 7 N2
    #   btstep     = 6 N2
    kbytes = {"tendency": 26 * N3, "vertvisc": 7 * N3 + 2 * N2,
              "continuity": 6 * N3 + 7 * N2, "btstep": 6 * N2, "halo_fill": 0}
    assert 2 * sum(kbytes.values()) == STEP_BYTES
    peak, peak_kind = _peaks()
    dom_avg_ms = kt[dom][0]
    achieved = kbytes[dom] / (dom_avg_ms / 1000.0) / 1e9 if dom_avg_ms > 0 else 0.0

    # end to end through the public API with pinned host buffers
    shape3 = (NI + 2, NJ + 2, NK)
    u = torch.empty(shape3[::-1], dtype=torch.float64, pin_memory=True).numpy().T
    v = torch.empty(shape3[::-1], dtype=torch.float64, pin_memory=True).numpy().T
    h = torch.empty(shape3[::-1], dtype=torch.float64, pin_memory=True).numpy().T
    eta = torch.empty((NJ + 2, NI + 2), dtype=torch.float64, pin_memory=True).numpy().T
    for name, a in (("u", u), ("v", v), ("h", h), ("eta", eta)):
        a[...] = m.get(name)
    # every step: upload the state the step reads (u, v, eta; h restarts from
    # h0 at every step) from pinned host memory, one RK2 step, read u, v, h,
    # eta back (the host-buffer C-ABI call mom6b_step_host_io)
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        m.step_host_io(1, u, v, eta, u, v, h, eta)
    t1 = time.perf_counter()
    e2e_s = max_over_ranks(t1 - t0, dist, local)
    e2e = world * args.steps / e2e_s
    bytes_h2d = 2 * N3 + N2
    bytes_d2h = 3 * N3 + N2
    # state resident on the device: one upload, K steps, one read-back
    barrier(dist)
    t0 = time.perf_counter()
    m.step_host_io(args.steps, u, v, eta, u, v, h, eta)
    t1 = time.perf_counter()
    e2e_res = world * args.steps / max_over_ranks(t1 - t0, dist, local)

    # the reference CUDA C backend on this GPU (its kernels built from their
    # sources with the reference's -O3) and this library's drop-in launch_*
    # path, both driven by the mirror of the reference host side
    ref_cudac = abi_dropin = None
    if not args.no_cudac:
        ref_so = os.path.join(ROOT, "oracle", "_ref", "libref_cuda_c.so")
        if os.path.exists(ref_so):
            ref_cudac = run_cudac(ref_so, args.steps, args.warmup, local)
            ref_cudac["kernels"] = "reference src/cuda_c/*.cu, nvcc -O3 sm_100a (oracle/_ref)"
        else:
            ref_cudac = {"unavailable": "oracle/_ref/libref_cuda_c.so not built "
                                        "(make -C oracle ref needs the reference sources)"}
        abi_dropin = run_cudac(None, args.steps, args.warmup, local)
        abi_dropin["kernels"] = "this library's launch_* entry points"
        if "value" in ref_cudac:
            abi_dropin["speedup_vs_reference_cuda_c"] = abi_dropin["value"] / ref_cudac["value"]
            ref_cudac["fused_speedup"] = value / world / ref_cudac["value"]

    # the exact form (bit-identical to the serial driver) on the same protocol
    exact_line = None
    if not args.no_exact:
        mx = Model(NI, NJ, NK, BT, INIT_CFG, seed=rank, dt=600.0, device=local,
                   use_graph=not args.no_graph, exact=True)
        t_ex = _time_model(mx, args, local, dist)
        mx.close()
        exact_line = {"value": world * args.steps / (t_ex / 1000.0), "unit": "steps/s",
                      "ms_per_step": t_ex / args.steps,
                      "what": "exact FP64 kernels (no FMA, serial column sums): bit-identical "
                              "to the serial driver"}

    mixed = None if args.no_mixed else run_mixed(args, world, rank, local, dist,
                                                   ms / args.steps)
    ensemble = None if args.no_ensemble else run_ensemble(args, world, rank, local, dist)
    surrogate = None if args.no_surrogate else run_surrogate(args, world, rank, local, dist,
                                                             ms / args.steps)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline_line()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": "split RK2 step 720x720x75 bt50, plain FP64, "
                                       "seeded beta plane (Philox), replicas per GPU",
                           "ni": NI, "nj": NJ, "nk": NK, "bt_nsteps": BT, "dt": 600.0,
                           "l2": "state 6 GB >> 126 MB L2, no flush needed",
                           "parallelism": f"replicas x{world}"},
                "step_bytes_algorithmic": STEP_BYTES,
                "step_roofline": {"achieved_GBs": STEP_BYTES / (ms / args.steps / 1000.0) / 1e9,
                                  "peak_GBs": peak, "frac": STEP_BYTES / (ms / args.steps / 1000.0) / 1e9 / peak},
                "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved,
                             "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                             "peak_kind": peak_kind,
                             "traffic": measured_traffic().get(dom),
                             "traffic_source": "ncu 360x360x75 capture scaled by units "
                                               "processed (profiles/traffic_720x720x75.txt)",
                             "bytes_per_launch": kbytes[dom], "avg_launch_ms": dom_avg_ms},
                "kernel_ms_per_step": per_step_ms,
                "cpu_baseline": cpu,
                "e2e": {"value": e2e, "unit": "steps/s", "h2d_bytes_per_step": bytes_h2d,
                        "d2h_bytes_per_step": bytes_d2h,
                        "what": "mom6b_step_host_io per step: u, v, eta uploaded from "
                                "pinned host memory (h restarts from h0 every step), one "
                                "step, u, v, h, eta read back"},
                "e2e_resident": {"value": e2e_res, "unit": "steps/s",
                                 "h2d_bytes_per_step": bytes_h2d / args.steps,
                                 "d2h_bytes_per_step": bytes_d2h / args.steps},
                "exact_fp64": exact_line,
                "reference_cuda_c": ref_cudac,
                "abi_dropin": abi_dropin,
                "mixed": mixed,
                "ensemble": ensemble,
                "surrogate": surrogate,
                "gpu_launches": launches,
                "clocks": ck}
        print(json.dumps(_finite(line)), flush=True)
    m.close()


def run_profile_case(args):
    """A small case of the same kernels for ncu: ni = nj = args.profile_case,
    nk = 75, bt 50, args.warmup + args.steps steps, nothing else."""
    from hackathon_mom6_miniapp_b200 import FP64, INIT_CFG, MIXED, Model
    n = args.profile_case
    m = Model(n, n, NK, BT, INIT_CFG, seed=0, dt=600.0,
              precision=MIXED if args.profile_mixed else FP64, exact=args.profile_exact)
    if args.profile_options:
        # the optional physics: hor_visc's scheme branches and the remnant
        m.set_hor_visc(biharmonic=True, smagorinsky=True, leith=True, better_bound=True)
        m.set_visc_remnant(True)
    m.step(args.warmup + args.steps)
    m.synchronize()
    print(json.dumps({"profile_case": n, "steps": args.warmup + args.steps,
                      "launches": m.launch_count()}))
    m.close()


def run_profile_abi(args):
    """A small case of the drop-in path for ncu: the mirror of the reference
    host side driving this library's launch_* entry points (kernel_lib None)
    or the reference's kernels (--profile-abi-ref), ni = nj =
    args.profile_abi, nk = 75, bt 50, CFG state, args.warmup + args.steps
    steps."""
    from hackathon_mom6_miniapp_b200 import INIT_CFG, CudaCDriver
    n = args.profile_abi
    lib = os.path.join(ROOT, "oracle", "_ref", "libref_cuda_c.so") if args.profile_abi_ref else None
    d = CudaCDriver(n, n, NK, BT, dt=600.0, kernel_lib=lib, init_mode=INIT_CFG, seed=0)
    d.step(args.warmup + args.steps)
    print(json.dumps({"profile_abi": n, "steps": args.warmup + args.steps,
                      "kernels": "reference" if lib else "libmom6b launch_*"}))
    d.close()


def run_profile_mlp(args):
    """The surrogate network's tensor-core kernels for ncu: forward and
    backward of a 65536-row batch (args.warmup + args.steps gradient calls)
    and one 716 x 716-column inference."""
    import numpy as np
    from hackathon_mom6_miniapp_b200 import Mlp
    B = 65536
    net = Mlp(batch=B, seed=1)
    rng = np.random.default_rng(0)
    X = rng.normal(size=(B, 175)).astype(np.float32)
    Y = rng.normal(size=(B, 2)).astype(np.float32)
    for _ in range(args.warmup + args.steps):
        net.gradients(X, Y)
    net.predict(X)
    print(json.dumps({"profile_mlp": B, "gradient_calls": args.warmup + args.steps}))
    net.close()


def run_decomp(args):
    """The decomposed step on one GPU: the 720x720x75 bt50 domain (FP64, no
    halo fill, seeded state) split PX x PY ways, one subdomain model per host
    thread, halos exchanged through the library's in-process halo group (peer
    copies, two host barriers per exchange, one launch per barotropic
    substep), against the same domain undecomposed (graph replay off in both,
    so the comparison is of the decomposition alone).  Wall time over
    args.steps steps after args.warmup, each subdomain synchronised.  Prints
    its own JSON line."""
    import threading
    import time
    from hackathon_mom6_miniapp_b200 import HaloGroup, INIT_CFG, Model, subdomain_config
    px, py = (int(x) for x in args.decomp.lower().split("x"))
    NI = NJ = 720

    def wall(models):
        errs = []

        def run(m, n):
            try:
                m.step(n)
                m.synchronize()
            except Exception as e:
                errs.append(e)

        for n in (args.warmup, args.steps):
            ts = [threading.Thread(target=run, args=(m, n)) for m in models]
            t0 = time.perf_counter()
            for t in ts:
                t.start()
            for t in ts:
                t.join()
            dt = time.perf_counter() - t0
        if errs:
            raise errs[0]
        return 1000.0 * dt / args.steps

    glob = Model(NI, NJ, NK, BT, INIT_CFG, seed=0, bc_fill=False, dt=600.0)
    single_ms = wall([glob])
    glob.close()
    group = HaloGroup(px, py, timeout_s=300.0)
    models = []
    for r in range(px * py):
        ni, nj, sub = subdomain_config(NI, NJ, px, py, r)
        m = Model(ni, nj, NK, BT, INIT_CFG, seed=0, bc_fill=False, dt=600.0, subdomain=sub)
        group.join(m, r)
        models.append(m)
    dec_ms = wall(models)
    print(json.dumps({"decomp": f"{px}x{py}", "workload": "720x720x75 bt50 FP64 fast form",
                      "single_domain_ms_per_step": single_ms,
                      "decomposed_ms_per_step": dec_ms,
                      "exchanges_per_step": 6 + 3 * 2 * BT,
                      "note": "one GPU; every subdomain on the same device"}))
    for m in models:
        m.close()
    group.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the mixed-precision form's line items")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="skip the learned-surrogate line item")
    ap.add_argument("--sur-steps", type=int, default=2000,
                    help="RK2 steps per training state of the surrogate (8 states)")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the 64-domain ensemble line item")
    ap.add_argument("--no-cfg2", action="store_true",
                    help="skip the mixed form's error at 1440x1080x75 after 100 steps")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--no-exact", action="store_true",
                    help="skip the exact FP64 form's timing")
    ap.add_argument("--no-cudac", action="store_true",
                    help="skip the reference CUDA C backend and drop-in ABI timings")
    ap.add_argument("--profile-mixed", action="store_true",
                    help="with --profile-case: the mixed-precision form's kernels")
    ap.add_argument("--profile-options", action="store_true",
                    help="with --profile-case: hor_visc schemes and the viscous remnant on")
    ap.add_argument("--profile-case", type=int, default=0,
                    help="run N steps of a ni=nj=N domain only (for ncu captures)")
    ap.add_argument("--profile-exact", action="store_true",
                    help="with --profile-case: the exact FP64 kernels")
    ap.add_argument("--profile-abi", type=int, default=0,
                    help="run the drop-in launch_* path on a ni=nj=N domain (for ncu)")
    ap.add_argument("--profile-abi-ref", action="store_true",
                    help="with --profile-abi: drive the reference's kernels instead")
    ap.add_argument("--profile-mlp", action="store_true",
                    help="run the surrogate network's GEMM kernels only (for ncu)")
    ap.add_argument("--decomp", default="",
                    help="PXxPY: time the decomposed step on one GPU against the single "
                         "domain (its own JSON line)")
    args = ap.parse_args()
    world, rank, local, dist = dist_setup(args)
    try:
        if args.profile_case:
            run_profile_case(args)
        elif args.profile_abi:
            run_profile_abi(args)
        elif args.profile_mlp:
            run_profile_mlp(args)
        elif args.decomp:
            run_decomp(args)
        elif args.impl == "reference":
            run_reference(args, world, rank, local, dist)
        else:
            run_ours(args, world, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
