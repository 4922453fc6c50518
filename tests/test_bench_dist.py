"""The multi-rank plumbing of bench.py with world size 2 on CPU (gloo).

bench.py runs one replica per GPU under torchrun; ranks share nothing but the
barrier around the timed region and the max / sum of their timings.  These
run here with the gloo backend and two spawned processes."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank)})
    import bench
    w, r, local, dist = bench.dist_setup(None, backend="gloo")
    try:
        bench.barrier(dist)
        mx = bench.max_over_ranks(1.5 * (r + 1), dist, local)
        sm = bench.sum_over_ranks(float(r + 1), dist, local)
        # value = units of all ranks / max time, as run_ours computes it
        steps, ms_local = 10, 100.0 * (r + 1)
        ms = bench.max_over_ranks(ms_local, dist, local)
        value = w * steps / (ms / 1000.0)
        q.put((r, w, mx, sm, value))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_and_barrier():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for r, w, mx, sm, value in out:
        assert w == 2 and mx == 3.0 and sm == 3.0
        assert value == pytest.approx(2 * 10 / 0.2)   # slowest rank sets the time
