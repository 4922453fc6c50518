"""A decomposed split RK2 step equals the undecomposed one bit for bit.

gloo ranks on the CPU each run the oracle on one subdomain of a 2-D
Cartesian layout (mpi_domain_init, mom6_mpi_domain.F90:57-137; non-periodic),
exchanging halos with the 8-direction exchange of `decomp.HaloExchange`
(halo_exchange_3d / _2d, mom6_mpi_halo_omp.F90:106-427) at the points of the
decomposed driver (rk2_mpi_cuda_c_driver.F90:305-412): up, vp before the
predictor continuity, h after it, u, v before the corrector continuity, and
the barotropic eta, ubt, vbt before every substep.  Each subdomain's initial
state and grid are those of its global points, and at a cut the ranges that
stop short of a wall reach the cut (the face on it is interior).  Every rank
compares its compute domain after the steps with the single-domain oracle's.
"""
import os
import socket

import numpy as np
import pytest

# fields compared on each rank's compute domain
_FIELDS = ("u", "v", "h", "eta", "up", "vp", "uh", "vh", "ubt_av", "vbt_av", "eta_av",
           "CAu", "CAv", "diffu", "diffv", "taux_bot", "tauy_bot", "du_cor", "hu_bt")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, px, py, NI, NJ, nk, nbt, mode, nsteps, first_dir, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch
    import torch.distributed as dist
    from hackathon_mom6_miniapp_b200.decomp import Decomposition, HaloExchange
    from oracle.pyoracle import CUT_E, CUT_N, CUT_S, CUT_W, Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # the mini-app's ni counts the compute width + 4 (n1 = ni + 2, is = 4)
        d = Decomposition(NI - 4, NJ - 4, px, py, rank)
        cuts = sum(bit for side, bit in (("W", CUT_W), ("E", CUT_E), ("S", CUT_S),
                                         ("N", CUT_N)) if d.neighbour(side) is not None)
        loc = Oracle(d.ni_local + 4, d.nj_local + 4, nk, nbt, init_mode=mode, bc_fill=False,
                     subdomain=(NI, NJ, d.i_offset, d.j_offset, cuts))
        assert (loc.n1, loc.n2) == (d.n1, d.n2)
        x = HaloExchange(d)

        def exchange(a, kind):
            x.exchange(torch.from_numpy(a.T))   # (nz, n2, n1) view of the Fortran array

        loc.set_exchange(exchange)
        loc.set_bt_first_direction(first_dir)
        glob = Oracle(NI, NJ, nk, nbt, init_mode=mode, bc_fill=False)
        glob.set_bt_first_direction(first_dir)
        # the initial state of each subdomain is the global one, halos included
        bad0 = 0
        for name in ("u", "v", "h", "eta", "ubt", "vbt", "taux"):
            a, g = loc.get(name), glob.get(name)
            sl = (slice(d.i_offset, d.i_offset + d.n1), slice(d.j_offset, d.j_offset + d.n2))
            bad0 += int(np.count_nonzero(a != g[sl]))
        loc.step(nsteps)
        glob.step(nsteps)
        res = {}
        i0, i1, j0, j1 = loc.is_ - 1, loc.ie, loc.js - 1, loc.je
        for name in _FIELDS:
            a, g = loc.get(name), glob.get(name)
            gi0, gj0 = i0 + d.i_offset, j0 + d.j_offset
            gs = g[gi0:gi0 + (i1 - i0), gj0:gj0 + (j1 - j0)]
            res[name] = int(np.count_nonzero(a[i0:i1, j0:j1] != gs))
        res["initial"] = bad0
        res["finite"] = bool(np.isfinite(loc.get("h")).all())
        loc.set_exchange(None)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def _run(px, py, NI, NJ, nk, nbt, mode, nsteps, first_dir=0):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = px * py
    procs = [ctx.Process(target=_worker,
                         args=(r, world, px, py, NI, NJ, nk, nbt, mode, nsteps, first_dir,
                               port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    return sorted(q.get(timeout=10) for _ in range(world))


@pytest.mark.parametrize("px,py,NI,NJ,mode", [
    (2, 1, 28, 22, 1),     # world size 2, an east-west cut, seeded state
    (1, 2, 26, 27, 0),     # world size 2, a north-south cut, analytic state
    (2, 2, 29, 25, 1),     # world size 4, both cuts and the corner, uneven split
    (2, 2, 28, 28, 0),
])
def test_decomposed_step_is_bit_identical(px, py, NI, NJ, mode):
    out = _run(px, py, NI, NJ, nk=5, nbt=8, mode=mode, nsteps=2)
    for rank, res in out:
        assert res["finite"], rank
        bad = {k: v for k, v in res.items() if k != "finite" and v}
        assert not bad, (rank, bad)


def test_decomposed_step_other_first_direction():
    """The barotropic u/v update order alternates from the other side."""
    out = _run(2, 2, 27, 26, nk=4, nbt=7, mode=1, nsteps=1, first_dir=1)
    for rank, res in out:
        bad = {k: v for k, v in res.items() if k != "finite" and v}
        assert not bad, (rank, bad)


def test_decomposed_step_in_threads_with_the_local_exchange():
    """The same decomposition with the subdomains held by threads of one
    process, exchanging through decomp.LocalHaloExchange (the in-process form
    of the exchange that Model.set_exchange takes): bit-identical as well."""
    import threading

    import torch
    from hackathon_mom6_miniapp_b200.decomp import Decomposition, LocalBoard, LocalHaloExchange
    from oracle.pyoracle import CUT_E, CUT_N, CUT_S, CUT_W, Oracle
    px, py, NI, NJ, nk, nbt, nsteps = 2, 2, 27, 30, 4, 6, 2
    board = LocalBoard(px * py, timeout=120.0)
    locs, errs = [], []
    for r in range(px * py):
        d = Decomposition(NI - 4, NJ - 4, px, py, r)
        cuts = sum(bit for side, bit in (("W", CUT_W), ("E", CUT_E), ("S", CUT_S),
                                         ("N", CUT_N)) if d.neighbour(side) is not None)
        o = Oracle(d.ni_local + 4, d.nj_local + 4, nk, nbt, init_mode=1, bc_fill=False,
                   subdomain=(NI, NJ, d.i_offset, d.j_offset, cuts))
        x = LocalHaloExchange(d, board)
        o.set_exchange(lambda a, kind, x=x: x.exchange(torch.from_numpy(a.T)))
        locs.append((d, o))

    def run(o):
        try:
            o.step(nsteps)
        except Exception as e:
            errs.append(e)

    ts = [threading.Thread(target=run, args=(o,)) for _, o in locs]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=300)
    assert not errs
    glob = Oracle(NI, NJ, nk, nbt, init_mode=1, bc_fill=False)
    glob.step(nsteps)
    for d, o in locs:
        i0, i1, j0, j1 = o.is_ - 1, o.ie, o.js - 1, o.je
        for name in ("u", "v", "h", "eta", "ubt_av", "vbt_av"):
            a = o.get(name)[i0:i1, j0:j1]
            g = glob.get(name)[i0 + d.i_offset:i1 + d.i_offset, j0 + d.j_offset:j1 + d.j_offset]
            assert np.array_equal(a, g), (d.rank, name)
        o.set_exchange(None)
