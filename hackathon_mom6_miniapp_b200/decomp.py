"""2-D domain decomposition and the 8-direction halo exchange of the
mini-app's decomposed drivers, over torch.distributed (NCCL between GPUs,
gloo on the host).

`Decomposition` restates mpi_domain_init (mom6_mpi_domain.F90:57-137): an
npes_x x npes_y Cartesian layout of ranks (rank = pos_x * npes_y + pos_y, as
MPI_Cart_create orders a 2-D grid), non-periodic neighbours in the four
cardinal and four diagonal directions (None at the global boundary), local
compute sizes with the remainder given to the first positions, and the
0-based offsets of each rank's compute domain in the global one.  A rank's
arrays hold a halo of `halo` points on every side (init_ocean_grid_mpi:
data domain [1, ni_local + 2 halo], compute domain [halo + 1, ni_local +
halo], mom6_mpi_domain.F90:157-172).

`HaloExchange.exchange` restates halo_exchange_3d / halo_exchange_2d
(mom6_mpi_halo.F90:107-431): every send strip is packed before any receive
is unpacked; east/west strips span the rows [jsd + hw, jed - hw] (and the
halo rows on a side without a north / south neighbour: there the reference's
strips stop at the compute rows, which leaves the corner between a cut and a
wall holding its initial values; the strips here carry the neighbour's
wall-face values there, so that the decomposed step is the single-domain
one), north/south strips the full data width (so they carry the sender's east/west halo columns
as they were before the exchange); received strips are unpacked in the order
E, W, N, S, NE, NW, SE, SW, the corner blocks overwriting the corners of the
north/south strips where a diagonal neighbour exists; nothing is written on a
side without a neighbour.  The strips are placed relative to the data-domain
edge, so only a width equal to the halo lands on the neighbour's matching
global points; the width is therefore the halo here (the reference passes
HALO_WIDTH = 7, mom6_types.F90:85, and 1 between barotropic substeps, on a
halo of 3).

Arrays are the model's Fortran (n1, n2[, nk]) arrays seen as C-order torch
tensors of shape (n2, n1) or (nk, n2, n1): index [..., j - 1, i - 1].
"""

from dataclasses import dataclass
from typing import Optional

# direction -> (send rows, send cols, recv rows, recv cols) as slices builders
_DIRS = ("E", "W", "N", "S", "NE", "NW", "SE", "SW")
_OPPOSITE = {"E": "W", "W": "E", "N": "S", "S": "N",
             "NE": "SW", "SW": "NE", "NW": "SE", "SE": "NW"}


@dataclass
class Decomposition:
    ni_global: int
    nj_global: int
    npes_x: int
    npes_y: int
    rank: int
    halo: int = 3

    def __post_init__(self):
        if self.npes_x < 1 or self.npes_y < 1:
            raise ValueError("npes_x and npes_y must be positive")
        if not 0 <= self.rank < self.npes_x * self.npes_y:
            raise ValueError("rank outside the layout")
        self.pos_x, self.pos_y = divmod(self.rank, self.npes_y)
        self.ni_local, self.i_offset = self._split(self.ni_global, self.npes_x, self.pos_x)
        self.nj_local, self.j_offset = self._split(self.nj_global, self.npes_y, self.pos_y)
        if self.ni_local < self.halo or self.nj_local < self.halo:
            raise ValueError("local domain narrower than the halo")

    @staticmethod
    def _split(n, npes, pos):
        base, rem = divmod(n, npes)
        if pos < rem:
            return base + 1, pos * (base + 1)
        return base, rem * (base + 1) + (pos - rem) * base

    def rank_at(self, px, py) -> Optional[int]:
        if 0 <= px < self.npes_x and 0 <= py < self.npes_y:
            return px * self.npes_y + py
        return None

    def neighbour(self, d) -> Optional[int]:
        dx = (1 if "E" in d else 0) - (1 if "W" in d else 0)
        dy = (1 if "N" in d else 0) - (1 if "S" in d else 0)
        return self.rank_at(self.pos_x + dx, self.pos_y + dy)

    @property
    def n1(self):
        return self.ni_local + 2 * self.halo

    @property
    def n2(self):
        return self.nj_local + 2 * self.halo

    def global_index(self, i, j):
        """0-based global compute indices of the local 1-based data point (i, j)."""
        return (i - self.halo - 1) + self.i_offset, (j - self.halo - 1) + self.j_offset


class HaloExchange:
    """The 8-direction exchange of one rank (see the module docstring)."""

    def __init__(self, decomp: Decomposition, group=None):
        self.d = decomp
        self.group = group
        self.nbr = {k: decomp.neighbour(k) for k in _DIRS}

    def _regions(self, n1, n2):
        hw = self.d.halo
        # east/west strips: the compute rows, and the halo rows of a wall side
        # (no south / north neighbour), whose wall-face values the neighbour
        # computes as the single domain does (vert_visc updates v on the
        # south wall face J = js-1, mom6_vert_visc_serial.F90:394-506)
        rows_in = slice(0 if self.nbr["S"] is None else hw,
                        n2 if self.nbr["N"] is None else n2 - hw)
        e_s, w_s = slice(n1 - 2 * hw, n1 - hw), slice(hw, 2 * hw)
        n_s, s_s = slice(n2 - 2 * hw, n2 - hw), slice(hw, 2 * hw)
        e_r, w_r = slice(n1 - hw, n1), slice(0, hw)
        n_r, s_r = slice(n2 - hw, n2), slice(0, hw)
        full = slice(0, n1)
        send = {"E": (rows_in, e_s), "W": (rows_in, w_s), "N": (n_s, full), "S": (s_s, full),
                "NE": (n_s, e_s), "NW": (n_s, w_s), "SE": (s_s, e_s), "SW": (s_s, w_s)}
        recv = {"E": (rows_in, e_r), "W": (rows_in, w_r), "N": (n_r, full), "S": (s_r, full),
                "NE": (n_r, e_r), "NW": (n_r, w_r), "SE": (s_r, e_r), "SW": (s_r, w_r)}
        return send, recv

    def exchange(self, a):
        """Exchange the halo of `a` ((n2, n1) or (nk, n2, n1)) in place."""
        self.exchange_many([a])
        return a

    def exchange_many(self, arrays):
        """Exchange the halos of several arrays (or (array, kind) pairs, as
        Model.set_exchange(batch=True) passes them) in one round of messages."""
        import torch
        import torch.distributed as dist
        arrays = [x[0] if isinstance(x, tuple) else x for x in arrays]
        plan = []
        for a in arrays:
            n2, n1 = a.shape[-2], a.shape[-1]
            if (n1, n2) != (self.d.n1, self.d.n2):
                raise ValueError(f"array {tuple(a.shape)} does not match the data domain "
                                 f"({self.d.n2}, {self.d.n1})")
            send, recv = self._regions(n1, n2)
            bufs_s, bufs_r = {}, {}
            for k in _DIRS:
                if self.nbr[k] is None:
                    continue
                rs, cs = send[k]
                bufs_s[k] = a[..., rs, cs].contiguous()      # packed before any unpack
                rr, cr = recv[k]
                bufs_r[k] = torch.empty_like(a[..., rr, cr]).contiguous()
            plan.append((a, recv, bufs_s, bufs_r))
        ops = []
        for _, _, bufs_s, bufs_r in plan:
            for k in _DIRS:
                if self.nbr[k] is None:
                    continue
                ops.append(dist.P2POp(dist.irecv, bufs_r[k], self.nbr[k], self.group))
                ops.append(dist.P2POp(dist.isend, bufs_s[k], self.nbr[k], self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for a, recv, _, bufs_r in plan:
            for k in _DIRS:                                    # E, W, N, S, NE, NW, SE, SW
                if self.nbr[k] is None:
                    continue
                rr, cr = recv[k]
                a[..., rr, cr] = bufs_r[k]
        return arrays


class LocalBoard:
    """Where the subdomains held by the threads of one process meet: one slot
    per rank and a barrier (timeout in seconds) for a LocalHaloExchange."""

    def __init__(self, world, timeout=120.0):
        import threading
        self.barrier = threading.Barrier(world, timeout=timeout)
        self.slots = [None] * world


class LocalHaloExchange(HaloExchange):
    """The same 8-direction exchange among subdomains held by threads of one
    process (one model per thread, on one or several GPUs): every rank packs
    its send strips, meets the others at the board's barrier, unpacks its
    neighbours' strips in the order E, W, N, S, NE, NW, SE, SW, and meets them
    again before the strips may change.  CUDA tensors are packed and unpacked
    on the current stream, which is synchronised before each meeting."""

    def __init__(self, decomp: Decomposition, board: LocalBoard):
        super().__init__(decomp)
        self.board = board

    def exchange_many(self, arrays):
        arrays = [x[0] if isinstance(x, tuple) else x for x in arrays]
        packs, recvs = [], []
        for a in arrays:
            n2, n1 = a.shape[-2], a.shape[-1]
            if (n1, n2) != (self.d.n1, self.d.n2):
                raise ValueError(f"array {tuple(a.shape)} does not match the data domain "
                                 f"({self.d.n2}, {self.d.n1})")
            send, recv = self._regions(n1, n2)
            packed = {}
            for k in _DIRS:
                if self.nbr[k] is not None:
                    rs, cs = send[k]
                    packed[k] = a[..., rs, cs].clone()
            packs.append(packed)
            recvs.append(recv)
        for a in arrays:
            self._sync(a)
        self.board.slots[self.d.rank] = packs
        self.board.barrier.wait()
        for f, a in enumerate(arrays):
            for k in _DIRS:
                if self.nbr[k] is not None:
                    rr, cr = recvs[f][k]
                    a[..., rr, cr] = self.board.slots[self.nbr[k]][f][_OPPOSITE[k]].to(a.device)
        for a in arrays:
            self._sync(a)
        self.board.barrier.wait()
        return arrays

    @staticmethod
    def _sync(a):
        if a.is_cuda:
            import torch
            torch.cuda.current_stream(a.device).synchronize()


__all__ = ["Decomposition", "HaloExchange", "LocalBoard", "LocalHaloExchange"]
