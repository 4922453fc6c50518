"""Domain decomposition geometry (mpi_domain_init) and the 8-direction halo
exchange (halo_exchange_3d / _2d) on the host: gloo ranks on the CPU, each
holding its subdomain of a global field with its halo cleared; after one
exchange every halo point whose neighbour exists holds the global field at
its global position, and every other halo point is unchanged."""
import os
import socket

import numpy as np
import pytest

from hackathon_mom6_miniapp_b200.decomp import Decomposition


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("ni,nj,px,py", [(180, 180, 2, 2), (37, 29, 3, 2), (720, 720, 1, 4)])
def test_decomposition_matches_mpi_domain_init(ni, nj, px, py):
    ds = [Decomposition(ni, nj, px, py, r) for r in range(px * py)]
    # local sizes cover the global domain without overlap, remainder to the first positions
    for x in range(px):
        d = next(d for d in ds if d.pos_x == x and d.pos_y == 0)
        base, rem = divmod(ni, px)
        assert d.ni_local == base + (1 if x < rem else 0)
    assert sum(d.ni_local for d in ds if d.pos_y == 0) == ni
    assert sum(d.nj_local for d in ds if d.pos_x == 0) == nj
    for d in ds:
        assert d.rank == d.pos_x * py + d.pos_y
        e = d.neighbour("E")
        if e is not None:
            de = ds[e]
            assert de.i_offset == d.i_offset + d.ni_local and de.j_offset == d.j_offset
        else:
            assert d.pos_x == px - 1
        ne = d.neighbour("NE")
        assert (ne is None) == (d.neighbour("N") is None or d.neighbour("E") is None)
        assert (d.n1, d.n2) == (d.ni_local + 6, d.nj_local + 6)


def _global(ig, jg, k):
    return 1000.0 * ig + jg + 0.25 * k


def _worker(rank, world, px, py, ni, nj, nk, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import torch
    import torch.distributed as dist
    from hackathon_mom6_miniapp_b200.decomp import Decomposition, HaloExchange
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = Decomposition(ni, nj, px, py, rank)
        hw = d.halo
        a = torch.full((nk, d.n2, d.n1), -1.0, dtype=torch.float64)
        for j in range(hw + 1, hw + d.nj_local + 1):
            for i in range(hw + 1, hw + d.ni_local + 1):
                ig, jg = d.global_index(i, j)
                for k in range(nk):
                    a[k, j - 1, i - 1] = _global(ig, jg, k)
        HaloExchange(d).exchange(a)
        bad = 0
        for j in range(1, d.n2 + 1):
            for i in range(1, d.n1 + 1):
                dx = -1 if i <= hw else (1 if i > d.n1 - hw else 0)
                dy = -1 if j <= hw else (1 if j > d.n2 - hw else 0)
                ig, jg = d.global_index(i, j)
                has = (dx == 0 and dy == 0) or d.rank_at(d.pos_x + dx, d.pos_y + dy) is not None
                for k in range(nk):
                    want = _global(ig, jg, k) if has else -1.0
                    bad += int(a[k, j - 1, i - 1].item() != want)
        q.put((rank, bad))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("px,py,ni,nj", [(2, 2, 23, 19), (2, 1, 20, 16), (1, 3, 12, 27)])
def test_halo_exchange_places_every_strip(px, py, ni, nj):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = px * py
    procs = [ctx.Process(target=_worker, args=(r, world, px, py, ni, nj, 2, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(world))
    assert [b for _, b in out] == [0] * world, out


def test_exchange_rejects_a_foreign_shape():
    import torch
    from hackathon_mom6_miniapp_b200.decomp import HaloExchange
    d = Decomposition(20, 20, 1, 1, 0)
    with pytest.raises(ValueError):
        HaloExchange(d).exchange(torch.zeros(2, d.n2, d.n1 + 1, dtype=torch.float64))
