"""Spatial domain decomposition of one periodic system over several GPUs.

The reference runs one system on one GPU (``Sim.py:22-25``). Here the box is
cut into slabs along x, one per rank (one process per GPU, ``torch.distributed``
over NCCL; gloo on the CPU for tests). Each rank owns the bodies whose centre
lies in its slab and, every step:

1. receives a halo from both neighbouring slabs: the positions and
   orientations of their bodies within ``halo`` (pair cutoff + Verlet skin) of
   the shared boundary, with ``send``/``recv`` to the neighbours only (no
   collective on the data path). The halo's membership is chosen when the
   Verlet lists are rebuilt and kept until the next rebuild, so that the list
   indices stay valid; in between only the coordinates travel;
2. evaluates the pair forces of every pair with at least one owned body over
   owned + halo bodies (owned bodies first, so that these pairs are the prefix
   of the (i, j)-sorted Verlet list with i < n_owned) and keeps the forces and
   torques of its owned bodies. A pair across a boundary is evaluated on both
   sides ("Newton off"), which needs no reverse exchange of forces;
3. integrates its owned bodies; the thermostat, which needs the kinetic
   energies of the whole system, takes one all-reduce of two numbers.

At each Verlet rebuild bodies that left the slab move to the rank that now
owns them (``migrate``). Positions stay wrapped in the periodic box, and the
minimum image of the force kernels handles pairs across the periodic boundary
(slabs are at least one halo wide).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

FIELDS = ("pos", "quat", "vel", "angmom", "mass", "ids")


@dataclass
class Slab:
    """Slab ``rank`` of ``world`` along x in a periodic box of edge L centred on 0."""
    L: float
    world: int
    rank: int

    @property
    def lo(self) -> float:
        return -0.5 * self.L + self.rank * self.L / self.world

    @property
    def hi(self) -> float:
        return -0.5 * self.L + (self.rank + 1) * self.L / self.world

    def owner(self, x: np.ndarray) -> np.ndarray:
        """Owning rank of each x (wrapped into [-L/2, L/2))."""
        u = (np.asarray(x, np.float64) + 0.5 * self.L) / self.L
        return np.clip(np.floor((u - np.floor(u)) * self.world).astype(np.int64), 0, self.world - 1)

    def near_lo(self, x: np.ndarray, width: float) -> np.ndarray:
        """Owned x within `width` of the lower boundary (periodic distance)."""
        d = np.mod(np.asarray(x, np.float64) - self.lo, self.L)
        return d < width

    def near_hi(self, x: np.ndarray, width: float) -> np.ndarray:
        d = np.mod(self.hi - np.asarray(x, np.float64), self.L)
        return d <= width


class Comm:
    """Point-to-point exchange with the two neighbouring slabs over
    ``torch.distributed`` (any backend with send/recv: NCCL, gloo). For two
    ranks both neighbours are the same rank; the messages keep a fixed order
    (towards the lower neighbour first), so they pair up on both sides."""

    def __init__(self, dist, rank: int, world: int, device):
        self.dist, self.rank, self.world, self.device = dist, rank, world, torch.device(device)
        self.lower, self.upper = (rank - 1) % world, (rank + 1) % world

    def _p2p(self, ops) -> None:
        # one group of sends and receives (NCCL would deadlock on a send whose
        # matching receive sits behind the peer's own send)
        d = self.dist
        for r in d.batch_isend_irecv([d.P2POp(fn, t, peer) for fn, t, peer in ops]):
            r.wait()

    def _exchange(self, send: torch.Tensor, dst: int, src: int) -> torch.Tensor:
        d = self.dist
        n_out = torch.tensor([send.shape[0]], dtype=torch.int64, device=self.device)
        n_in = torch.zeros(1, dtype=torch.int64, device=self.device)
        self._p2p([(d.isend, n_out, dst), (d.irecv, n_in, src)])
        recv = torch.empty((int(n_in.item()),) + tuple(send.shape[1:]), dtype=send.dtype, device=self.device)
        ops = []
        if send.shape[0]:
            ops.append((d.isend, send.contiguous(), dst))
        if recv.shape[0]:
            ops.append((d.irecv, recv, src))
        if ops:
            self._p2p(ops)
        return recv

    def shift(self, to_lower: torch.Tensor, to_upper: torch.Tensor):
        """Send `to_lower` to the lower neighbour and `to_upper` to the upper one;
        returns (from_upper, from_lower): what the upper neighbour sent to its
        lower side and what the lower neighbour sent to its upper side. One rank
        has no neighbour: nothing comes back."""
        if self.world == 1:
            return to_lower[:0].clone(), to_upper[:0].clone()
        from_upper = self._exchange(to_lower, self.lower, self.upper)
        from_lower = self._exchange(to_upper, self.upper, self.lower)
        return from_upper, from_lower

    def sum(self, t: torch.Tensor) -> torch.Tensor:
        if self.world > 1:
            self.dist.all_reduce(t)
        return t


class Halo:
    """Halo bookkeeping of one rank for one Verlet-list period: which owned
    bodies go to each neighbour (chosen at the rebuild) and how many come back.
    ``payload`` / ``receive`` split an exchange into its two halves, so that a
    test can pass the messages of several ranks by hand in one process."""

    def __init__(self, slab: Slab, width: float):
        if slab.world > 1 and slab.L / slab.world < width:
            raise ValueError(f"slabs of {slab.L / slab.world:.3g} are thinner than the halo of {width:.3g}")
        self.slab, self.width = slab, float(width)
        self.to_lower = self.to_upper = None
        self.n_from_upper = self.n_from_lower = 0

    def choose(self, pos_owned: np.ndarray) -> None:
        """Owned bodies within the halo width of each boundary (at a rebuild)."""
        x = np.asarray(pos_owned)[:, 0]
        self.to_lower = np.nonzero(self.slab.near_lo(x, self.width))[0]
        self.to_upper = np.nonzero(self.slab.near_hi(x, self.width))[0]

    def payload(self, pos: torch.Tensor, quat: torch.Tensor):
        """(to_lower, to_upper): (k, 7) float32 rows of position and orientation."""
        pq = torch.cat([pos, quat], dim=1)
        lo = torch.as_tensor(self.to_lower, device=pos.device, dtype=torch.long)
        hi = torch.as_tensor(self.to_upper, device=pos.device, dtype=torch.long)
        return pq[lo], pq[hi]

    def receive(self, pos: torch.Tensor, quat: torch.Tensor, from_upper: torch.Tensor, from_lower: torch.Tensor):
        """Owned + halo arrays: owned bodies first, then the upper neighbour's,
        then the lower neighbour's."""
        self.n_from_upper, self.n_from_lower = int(from_upper.shape[0]), int(from_lower.shape[0])
        ext = torch.cat([torch.cat([pos, quat], dim=1), from_upper, from_lower], dim=0)
        return ext[:, :3].contiguous(), ext[:, 3:].contiguous()

    def exchange(self, comm: Comm, pos: torch.Tensor, quat: torch.Tensor):
        lo, hi = self.payload(pos, quat)
        from_upper, from_lower = comm.shift(lo, hi)
        return self.receive(pos, quat, from_upper, from_lower)


def migrate(comm: Comm, slab: Slab, owned: dict) -> dict:
    """Bodies whose centre left the slab go to the neighbour that owns them now
    (a body moves at most one slab between two rebuilds: slabs are wider than
    the skin). `owned` maps FIELDS to tensors of the owned bodies; returns the
    new owned set (kept bodies first, then arrivals from the upper and the lower
    neighbour)."""
    pos = owned["pos"]
    dest = slab.owner(pos[:, 0].detach().cpu().numpy())
    world, r = slab.world, slab.rank
    lower, upper = (r - 1) % world, (r + 1) % world
    stay = dest == r
    if world > 1 and not np.all(stay | (dest == lower) | (dest == upper)):
        raise RuntimeError("a body moved more than one slab between two Verlet rebuilds")
    rows = torch.cat([owned["pos"].double(), owned["quat"].double(), owned["vel"].double(),
                      owned["angmom"].double(), owned["mass"].double()[:, None], owned["ids"].double()[:, None]],
                     dim=1)
    dev = rows.device
    keep = torch.as_tensor(np.nonzero(stay)[0], device=dev, dtype=torch.long)
    go_lo = torch.as_tensor(np.nonzero((dest == lower) & ~stay)[0], device=dev, dtype=torch.long)
    go_hi = torch.as_tensor(np.nonzero((dest == upper) & ~stay & (dest != lower))[0], device=dev, dtype=torch.long)
    if world == 2:  # one neighbour on both sides: every leaving body goes "down"
        go_lo = torch.as_tensor(np.nonzero(~stay)[0], device=dev, dtype=torch.long)
        go_hi = go_hi[:0]
    from_upper, from_lower = comm.shift(rows[go_lo], rows[go_hi])
    new = torch.cat([rows[keep], from_upper, from_lower], dim=0)
    return {"pos": new[:, 0:3].float().contiguous(), "quat": new[:, 3:7].float().contiguous(),
            "vel": new[:, 7:10].float().contiguous(), "angmom": new[:, 10:14].float().contiguous(),
            "mass": new[:, 14].float().contiguous(), "ids": new[:, 15].round().long()}
