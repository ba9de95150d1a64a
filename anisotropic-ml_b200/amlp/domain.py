"""Spatial domain decomposition of one periodic system over several GPUs.

The reference runs one system on one GPU (``Sim.py:22-25``). Here the box is
cut into a grid of px x py x pz bricks, one per rank (one process per GPU,
``torch.distributed`` over NCCL; gloo on the CPU for tests); slabs along x are
the case py = pz = 1. Each rank owns the bodies whose centre lies in its brick
and, every step:

1. receives a halo: the positions and orientations of the bodies of other
   bricks within ``halo`` (pair cutoff + Verlet skin) of its own, in one pass
   per cut axis with ``send``/``recv`` to the two neighbours along that axis
   (no collective on the data path). A pass forwards what the earlier passes
   received, so the bodies of the edge and corner neighbours arrive through the
   face neighbours (six messages for a 3-D grid, not 26). The halo's membership
   is chosen when the Verlet lists are rebuilt and kept until the next
   rebuild, so that the list indices stay valid; in between only the
   coordinates travel;
2. evaluates the pair forces of every pair with at least one owned body over
   owned + halo bodies (owned bodies first, so that these pairs are the prefix
   of the (i, j)-sorted Verlet list with i < n_owned; each pair then oriented by
   global index, as in the single domain) and keeps the forces and torques of
   its owned bodies. A pair across a boundary is evaluated on both sides
   ("Newton off"), which needs no reverse exchange of forces;
3. integrates its owned bodies; the thermostat, which needs the kinetic
   energies of the whole system, takes one all-reduce of two numbers.

At each Verlet rebuild bodies that left the brick move to the rank that now
owns them (``migrate``, axis by axis). Positions stay wrapped in the periodic
box, and the minimum image of the force kernels handles pairs across the
periodic boundary (bricks are at least two halos wide along every cut axis).
"""
from __future__ import annotations

import numpy as np
import torch

FIELDS = ("pos", "quat", "vel", "angmom", "mass", "ids")


def brick_dims(world: int, L: float, width: float) -> tuple:
    """(px, py, pz) with px py pz = world, as close to a cube as the box allows:
    every cut axis keeps bricks at least 2 * width wide."""
    best = None
    for px in range(1, world + 1):
        if world % px:
            continue
        for py in range(1, world // px + 1):
            if (world // px) % py:
                continue
            dims = (px, py, world // px // py)
            if any(p > 1 and L / p < 2.0 * width for p in dims):
                continue
            # the smallest largest cut, then the most even, then the cuts along x first
            key = (max(dims), -min(dims), tuple(-p for p in dims))
            if best is None or key < best[0]:
                best = (key, dims)
    if best is None:
        raise ValueError(f"{world} bricks of a box of {L:.3g} cannot all be two halos of {width:.3g} wide")
    return best[1]


class Brick:
    """Brick ``rank`` of a px x py x pz grid over a periodic box of edge L centred
    on 0; rank = (cx py + cy) pz + cz for the brick's grid coordinates."""

    def __init__(self, L: float, dims, rank: int):
        self.L, self.dims, self.rank = float(L), tuple(int(p) for p in dims), int(rank)
        self.world = int(np.prod(self.dims))
        px, py, pz = self.dims
        self.coords = (rank // (py * pz), (rank // pz) % py, rank % pz)

    def lo(self, axis: int) -> float:
        return -0.5 * self.L + self.coords[axis] * self.L / self.dims[axis]

    def hi(self, axis: int) -> float:
        return -0.5 * self.L + (self.coords[axis] + 1) * self.L / self.dims[axis]

    def coord(self, x: np.ndarray, axis: int) -> np.ndarray:
        """Grid coordinate along `axis` of each coordinate x (wrapped into [-L/2, L/2))."""
        p = self.dims[axis]
        u = (np.asarray(x, np.float64) + 0.5 * self.L) / self.L
        return np.clip(np.floor((u - np.floor(u)) * p).astype(np.int64), 0, p - 1)

    def rank_of(self, c) -> int:
        px, py, pz = self.dims
        return int((c[0] * py + c[1]) * pz + c[2])

    def owner(self, pos: np.ndarray) -> np.ndarray:
        """Owning rank of each position (rows x, y, z)."""
        pos = np.asarray(pos)
        px, py, pz = self.dims
        return (self.coord(pos[:, 0], 0) * py + self.coord(pos[:, 1], 1)) * pz + self.coord(pos[:, 2], 2)

    def neighbour(self, axis: int, step: int) -> int:
        c = list(self.coords)
        c[axis] = (c[axis] + step) % self.dims[axis]
        return self.rank_of(c)

    def near_lo(self, x: np.ndarray, width: float, axis: int) -> np.ndarray:
        """Coordinates within `width` above the lower face along `axis` (periodic distance)."""
        return np.mod(np.asarray(x, np.float64) - self.lo(axis), self.L) < width

    def near_hi(self, x: np.ndarray, width: float, axis: int) -> np.ndarray:
        return np.mod(self.hi(axis) - np.asarray(x, np.float64), self.L) <= width


class Slab(Brick):
    """Slab ``rank`` of ``world`` along x (a world x 1 x 1 grid of bricks)."""

    def __init__(self, L: float, world: int, rank: int):
        super().__init__(L, (world, 1, 1), rank)


class Comm:
    """Point-to-point exchange with the two neighbouring bricks along an axis of
    a px x py x pz grid, over ``torch.distributed`` (any backend with send/recv:
    NCCL, gloo). When an axis has two bricks both neighbours are the same rank;
    the messages keep a fixed order (towards the lower neighbour first), so they
    pair up on both sides."""

    def __init__(self, dist, rank: int, world: int, device, dims=None):
        self.dist, self.rank, self.world, self.device = dist, rank, world, torch.device(device)
        self.dims = tuple(dims) if dims is not None else (world, 1, 1)
        if int(np.prod(self.dims)) != world:
            raise ValueError(f"a grid of {self.dims} bricks is not {world} ranks")
        self.brick_of_rank = Brick(1.0, self.dims, rank)

    def neighbours(self, axis: int):
        return self.brick_of_rank.neighbour(axis, -1), self.brick_of_rank.neighbour(axis, +1)

    def _p2p(self, ops) -> None:
        # one group of sends and receives (NCCL would deadlock on a send whose
        # matching receive sits behind the peer's own send)
        d = self.dist
        for r in d.batch_isend_irecv([d.P2POp(fn, t, peer) for fn, t, peer in ops]):
            r.wait()

    def _exchange(self, send: torch.Tensor, dst: int, src: int, n_recv: int | None = None) -> torch.Tensor:
        d = self.dist
        if n_recv is None:  # the count first (a host synchronisation), then the rows
            n_out = torch.tensor([send.shape[0]], dtype=torch.int64, device=self.device)
            n_in = torch.zeros(1, dtype=torch.int64, device=self.device)
            self._p2p([(d.isend, n_out, dst), (d.irecv, n_in, src)])
            n_recv = int(n_in.item())
        recv = torch.empty((n_recv,) + tuple(send.shape[1:]), dtype=send.dtype, device=self.device)
        ops = []
        if send.shape[0]:
            ops.append((d.isend, send.contiguous(), dst))
        if recv.shape[0]:
            ops.append((d.irecv, recv, src))
        if ops:
            self._p2p(ops)
        return recv

    def shift(self, to_lower: torch.Tensor, to_upper: torch.Tensor, axis: int = 0, counts=None):
        """Send `to_lower` to the lower neighbour along `axis` and `to_upper` to
        the upper one; returns (from_upper, from_lower): what the upper neighbour
        sent to its lower side and what the lower neighbour sent to its upper
        side. An axis with one brick has no neighbour: nothing comes back. With
        `counts` = (rows from upper, rows from lower) known, the rows travel
        without a count exchange and without a host synchronisation."""
        if self.dims[axis] == 1:
            return to_lower[:0].clone(), to_upper[:0].clone()
        lower, upper = self.neighbours(axis)
        n_up, n_lo = counts if counts is not None else (None, None)
        from_upper = self._exchange(to_lower, lower, upper, n_up)
        from_lower = self._exchange(to_upper, upper, lower, n_lo)
        return from_upper, from_lower

    def sum(self, t: torch.Tensor) -> torch.Tensor:
        if self.world > 1:
            self.dist.all_reduce(t)
        return t


class Halo:
    """Halo bookkeeping of one rank for one Verlet-list period: per cut axis,
    which rows of the extended array (owned bodies, then the halo received so
    far) go to each neighbour along it, chosen at the rebuild and replayed at
    every step until the next one."""

    def __init__(self, brick: Brick, width: float):
        # a body within the halo width of both faces would reach a two-brick
        # neighbour twice, and a halo wider than a brick would need the brick beyond it
        for a, p in enumerate(brick.dims):
            if p > 1 and brick.L / p < 2.0 * width:
                raise ValueError(f"bricks of {brick.L / p:.3g} along axis {a} are thinner than twice the halo "
                                 f"of {width:.3g}")
        self.brick, self.width = brick, float(width)
        self.axes = [a for a, p in enumerate(brick.dims) if p > 1]
        self.sends = []   # per cut axis: (rows to the lower neighbour, rows to the upper neighbour)
        self.counts = []  # per cut axis: (rows from the upper neighbour, rows from the lower one)

    def _select(self, pos: np.ndarray, axis: int):
        x = np.asarray(pos)[:, axis]
        return (np.nonzero(self.brick.near_lo(x, self.width, axis))[0],
                np.nonzero(self.brick.near_hi(x, self.width, axis))[0])

    def _pass(self, comm: Comm, ext: torch.Tensor, k: int, axis: int) -> torch.Tensor:
        lo, hi = (torch.as_tensor(i, device=ext.device, dtype=torch.long) for i in self.sends[k])
        from_upper, from_lower = comm.shift(ext[lo], ext[hi], axis,
                                            self.counts[k] if k < len(self.counts) else None)
        if k == len(self.counts):  # at the rebuild: the counts hold until the next one
            self.counts.append((int(from_upper.shape[0]), int(from_lower.shape[0])))
        return torch.cat([ext, from_upper, from_lower], dim=0)

    def choose_and_exchange(self, comm: Comm, pos: torch.Tensor, quat: torch.Tensor, ids: torch.Tensor):
        """At a rebuild: choose each pass's rows from the positions of the array
        extended so far and exchange them; returns the extended positions,
        orientations and global indices (owned bodies first)."""
        ext = torch.cat([pos, quat], dim=1)
        ext_ids = ids
        self.sends, self.counts = [], []
        for k, axis in enumerate(self.axes):
            self.sends.append(self._select(ext[:, :3].cpu().numpy(), axis))
            lo, hi = (torch.as_tensor(i, device=ids.device, dtype=torch.long) for i in self.sends[k])
            ext = self._pass(comm, ext, k, axis)
            id_up, id_lo = comm.shift(ext_ids[lo], ext_ids[hi], axis, self.counts[k])
            ext_ids = torch.cat([ext_ids, id_up, id_lo])
        return ext[:, :3].contiguous(), ext[:, 3:].contiguous(), ext_ids

    def exchange(self, comm: Comm, pos: torch.Tensor, quat: torch.Tensor):
        """Between rebuilds: the same rows as chosen at the rebuild, current
        coordinates, the counts known (no count exchange, no host synchronisation)."""
        ext = torch.cat([pos, quat], dim=1)
        for k, axis in enumerate(self.axes):
            ext = self._pass(comm, ext, k, axis)
        return ext[:, :3].contiguous(), ext[:, 3:].contiguous()


def migrate(comm: Comm, brick: Brick, owned: dict) -> dict:
    """Bodies whose centre left the brick go to the rank that owns them now,
    one cut axis after the other (a body moves at most one brick along each
    axis between two rebuilds: bricks are wider than the skin; a body leaving
    through an edge or a corner reaches its owner through the face
    neighbours). `owned` maps FIELDS to tensors of the owned bodies; returns the
    new owned set (kept bodies first, then the arrivals of each pass)."""
    rows = torch.cat([owned["pos"].double(), owned["quat"].double(), owned["vel"].double(),
                      owned["angmom"].double(), owned["mass"].double()[:, None], owned["ids"].double()[:, None]],
                     dim=1)
    dev = rows.device
    for axis, p in enumerate(brick.dims):
        if p == 1:
            continue
        c = brick.coords[axis]
        dest = brick.coord(rows[:, axis].detach().cpu().numpy(), axis)
        lower, upper = (c - 1) % p, (c + 1) % p
        stay = dest == c
        if not np.all(stay | (dest == lower) | (dest == upper)):
            raise RuntimeError("a body moved more than one brick between two Verlet rebuilds")
        keep = torch.as_tensor(np.nonzero(stay)[0], device=dev, dtype=torch.long)
        go_lo = torch.as_tensor(np.nonzero((dest == lower) & ~stay)[0], device=dev, dtype=torch.long)
        go_hi = torch.as_tensor(np.nonzero((dest == upper) & ~stay & (dest != lower))[0], device=dev,
                                dtype=torch.long)
        if p == 2:  # one neighbour on both sides: every leaving body goes "down"
            go_lo = torch.as_tensor(np.nonzero(~stay)[0], device=dev, dtype=torch.long)
            go_hi = go_hi[:0]
        from_upper, from_lower = comm.shift(rows[go_lo], rows[go_hi], axis)
        rows = torch.cat([rows[keep], from_upper, from_lower], dim=0)
    return {"pos": rows[:, 0:3].float().contiguous(), "quat": rows[:, 3:7].float().contiguous(),
            "vel": rows[:, 7:10].float().contiguous(), "angmom": rows[:, 10:14].float().contiguous(),
            "mass": rows[:, 14].float().contiguous(), "ids": rows[:, 15].round().long()}


class OwnedForces:
    """Forces and torques on the owned bodies from owned + halo bodies through
    the library's kernels. At a rebuild the Verlet list of owned + halo bodies
    is cut to its pairs with an owned first body (the prefix i < n_owned of the
    (i, j)-sorted list), each pair is oriented by global index as in the single
    domain (the roles of the two bodies enter the rounding of a pair's forces),
    and the list is split into owned-owned pairs and pairs with a halo body;
    each step filters both and runs the force kernel on each. The pair
    energy sums each owned-owned pair once and each cross pair with weight
    1/2, so that the ranks' sums add up to the system's."""

    def __init__(self, shape, hypers, net, L: float, device, method: str = "adjoint", skin: float = 2.0):
        import ctypes
        from ._lib import Nep
        self.ctypes = ctypes
        self.shape, self.hypers, self.net, self.L = shape, hypers, net, float(np.float32(L))
        self.device, self.method = torch.device(device), method
        self.r = float(shape.cutoff) + float(skin)
        self.pts = torch.tensor(shape.pts, dtype=torch.float32, device=self.device)
        n = Nep()
        n.nrad, n.nang, n.lmax = hypers.nrad, hypers.nang, hypers.lmax
        n.npts, n.d_pts = shape.npts, self.pts.data_ptr()
        n.cutoff, n.nep_cutoff = float(shape.cutoff), float(shape.nep_cutoff)
        n.en_min, n.en_max, n.dx, n.dteta = float(shape.en_min), float(shape.en_max), 1e-5, 1e-5
        self.nep = n
        self.lists = []
        self.pe = torch.zeros(2, dtype=torch.float64, device=self.device)

    def _stream(self):
        return torch.cuda.current_stream().cuda_stream

    def rebuild(self, ext_pos: torch.Tensor, n_owned: int, ext_ids: torch.Tensor | None = None) -> None:
        """Verlet lists of the owned bodies' pairs. With the global indices of
        owned + halo bodies (`ext_ids`), every pair is oriented as in the single
        domain (first body = smaller global index), so that each pair's forces
        are computed with the same arithmetic as there."""
        from ._lib import call, size_query
        n = int(ext_pos.shape[0])
        ws = torch.empty(size_query("amlp_nlist_workspace_bytes", n, self.L, self.r), dtype=torch.uint8,
                         device=self.device)
        cnt = torch.zeros(1, dtype=torch.int64, device=self.device)
        cap = max(1024, 64 * n)
        while True:
            out = torch.empty(cap, 2, dtype=torch.int32, device=self.device)
            call("amlp_nlist_build", ext_pos.data_ptr(), n, self.L, self.r, out.data_ptr(), cap, cnt.data_ptr(),
                 ws.data_ptr(), ws.numel(), self._stream())
            k = int(cnt.item())
            if k <= cap:
                break
            cap = k
        vl = out[:k]
        vl = vl[vl[:, 0] < n_owned]                       # a pair of two halo bodies is another rank's
        if ext_ids is not None and vl.shape[0]:
            g = ext_ids.to(self.device)[vl.long()]
            swap = g[:, 0] > g[:, 1]
            vl = torch.where(swap[:, None], vl.flip(1), vl)
            key = vl[:, 0].long() * n + vl[:, 1].long()  # sorted by first body: the scatters merge per body
            vl = vl[torch.argsort(key)].contiguous()
        cross = (vl[:, 0] >= n_owned) | (vl[:, 1] >= n_owned)
        self.lists = []
        for part in (vl[~cross], vl[cross]):
            part = part.contiguous()
            m = max(1, int(part.shape[0]))
            self.lists.append(dict(
                v=part if part.shape[0] else torch.zeros(1, 2, dtype=torch.int32, device=self.device),
                nv=torch.tensor([int(part.shape[0])], dtype=torch.int64, device=self.device),
                f=torch.empty(m, 2, dtype=torch.int32, device=self.device),
                nf=torch.zeros(1, dtype=torch.int64, device=self.device), cap=m,
                ws=torch.empty(max(1, size_query("amlp_filter_workspace_bytes", m)), dtype=torch.uint8,
                               device=self.device),
                adj=(torch.empty(size_query("amlp_adjoint_workspace_bytes", m), dtype=torch.uint8,
                                 device=self.device)
                     if self.method == "adjoint" and (self.net.max_hidden > 64 or self.hypers.D > 48) else None)))

    def forces(self, ext_pos: torch.Tensor, ext_quat: torch.Tensor, n_owned: int):
        """(F, T) of the owned bodies, and this rank's share of the pair energy."""
        from ._lib import call
        c = self.ctypes
        n = int(ext_pos.shape[0])
        F = torch.zeros(n, 3, dtype=torch.float32, device=self.device)
        T = torch.zeros(n, 3, dtype=torch.float32, device=self.device)
        self.pe.zero_()
        st = self._stream()
        for k, lst in enumerate(self.lists):
            call("amlp_pair_filter", ext_pos.data_ptr(), self.L, float(self.shape.cutoff), lst["v"].data_ptr(),
                 lst["nv"].data_ptr(), lst["cap"], lst["f"].data_ptr(), lst["nf"].data_ptr(), lst["ws"].data_ptr(),
                 lst["ws"].numel(), st)
            args = [ext_pos.data_ptr(), ext_quat.data_ptr(), self.L, lst["f"].data_ptr(), lst["nf"].data_ptr(),
                    lst["cap"], c.byref(self.nep), c.byref(self.net.struct), F.data_ptr(), T.data_ptr(),
                    self.pe[k:k + 1].data_ptr()]
            if self.method == "fd":
                call("amlp_forces_fd", *args, st)
            elif lst["adj"] is None:
                call("amlp_forces_adjoint", *args, st)
            else:
                call("amlp_forces_adjoint_wide", *args, lst["adj"].data_ptr(), lst["adj"].numel(), st)
        return F[:n_owned], T[:n_owned], self.pe[0] + 0.5 * self.pe[1]


class DomainSystem:
    """One rank's part of a periodic system decomposed into bricks (see the
    module docstring; the grid is ``comm.dims``, e.g. from ``brick_dims``): owned
    bodies, halo exchange, forces, the NVT halves of the owned bodies and the
    global thermostat. Every rank calls ``step`` in lockstep."""

    def __init__(self, comm: Comm, state, shape, hypers, net, kT: float, dt: float, device, method: str = "adjoint",
                 nlist_every: int = 100, skin: float = 2.0):
        import ctypes
        from ._lib import Nvt, Thermostat, call, size_query
        from .engine import THERMOSTAT_SEED
        self.ctypes, self.call, self.size_query, self.Thermostat = ctypes, call, size_query, Thermostat
        self.comm, self.device = comm, torch.device(device)
        self.L = float(np.float32(state.L))
        self.brick = Brick(self.L, comm.dims, comm.rank)
        self.halo = Halo(self.brick, float(shape.cutoff) + float(skin))
        self.forces_of = OwnedForces(shape, hypers, net, self.L, device, method, skin)
        self.nlist_every, self.timestep, self.N = int(nlist_every), 0, int(state.N)
        mine = np.nonzero(self.brick.owner(np.asarray(state.pos)) == comm.rank)[0]
        f32 = dict(dtype=torch.float32, device=self.device)
        self.owned = {"pos": torch.tensor(np.asarray(state.pos)[mine], **f32),
                      "quat": torch.tensor(np.asarray(state.orient)[mine], **f32),
                      "vel": torch.tensor(np.asarray(state.vel)[mine], **f32),
                      "angmom": torch.tensor(np.asarray(state.angmom)[mine], **f32),
                      "mass": torch.tensor(np.asarray(state.mass)[mine], **f32),
                      "ids": torch.tensor(mine, dtype=torch.long, device=self.device)}
        self.nvt = Nvt()
        self.nvt.dt, self.nvt.tau, self.nvt.kT = float(dt), float(np.float32(100.0 * dt)), float(kT)
        self.nvt.n_dof, self.nvt.rn_dof = float((self.N - 1) * 3), float(3 * self.N)  # the whole system's
        for k in range(3):
            self.nvt.moi[k] = float(np.asarray(state.moi).reshape(-1)[k])
        self.nvt.box, self.nvt.nve = self.L, 0
        th = Thermostat()
        th.xi, th.eta, th.xi_rot, th.eta_rot, th.thermo_fac = THERMOSTAT_SEED
        self.th = torch.frombuffer(bytearray(bytes(th)), dtype=torch.uint8).to(self.device)
        self.pe = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._resize()
        self.call("amlp_nvt_init", self.owned["vel"].data_ptr(), self.owned["quat"].data_ptr(),
                  self.owned["angmom"].data_ptr(), self.owned["mass"].data_ptr(), self.n, ctypes.byref(self.nvt), 0,
                  self.th.data_ptr(), self.ws.data_ptr(), self.ws.numel(), self._stream())
        self._sum_kinetic()

    @property
    def n(self) -> int:
        return int(self.owned["pos"].shape[0])

    def _stream(self):
        return torch.cuda.current_stream().cuda_stream

    def _resize(self) -> None:
        if self.n <= 0:
            raise RuntimeError(f"rank {self.comm.rank} owns no body: too many bricks for this system")
        f32 = dict(dtype=torch.float32, device=self.device)
        self.accel = torch.zeros(self.n, 3, **f32)
        self.dp = torch.zeros(self.n, 4, **f32)
        self.ws = torch.empty(self.size_query("amlp_nvt_workspace_bytes", self.n), dtype=torch.uint8,
                              device=self.device)

    def _sum_kinetic(self) -> None:
        off = self.Thermostat.ke_t.offset
        ke = self.th[off:off + 16].view(torch.float64)  # ke_t, ke_r of the owned bodies -> of the system
        self.comm.sum(ke)

    def step(self) -> None:
        o, c = self.owned, self.ctypes
        if self.timestep % self.nlist_every == 0:
            if self.timestep > 0:
                self.owned = o = migrate(self.comm, self.brick, o)
                self._resize()
            ext_pos, ext_quat, ext_ids = self.halo.choose_and_exchange(self.comm, o["pos"], o["quat"], o["ids"])
            self.forces_of.rebuild(ext_pos, self.n, ext_ids)
        else:
            ext_pos, ext_quat = self.halo.exchange(self.comm, o["pos"], o["quat"])
        F, T, pe = self.forces_of.forces(ext_pos, ext_quat, self.n)
        self.F, self.T = F, T = F.contiguous(), T.contiguous()  # forces and torques of the owned bodies
        self.pe.copy_(pe.reshape(1))
        st = self._stream()
        self.call("amlp_nvt_step_two", o["vel"].data_ptr(), self.accel.data_ptr(), F.data_ptr(), o["mass"].data_ptr(),
                  o["quat"].data_ptr(), T.data_ptr(), o["angmom"].data_ptr(), self.dp.data_ptr(), self.n,
                  c.byref(self.nvt), self.th.data_ptr(), st)
        self.call("amlp_nvt_step_one", o["pos"].data_ptr(), o["vel"].data_ptr(), self.accel.data_ptr(),
                  o["quat"].data_ptr(), o["angmom"].data_ptr(), self.dp.data_ptr(), o["mass"].data_ptr(), self.n,
                  c.byref(self.nvt), self.th.data_ptr(), self.ws.data_ptr(), self.ws.numel(), st)
        self._sum_kinetic()
        self.timestep += 1

    def run(self, nsteps: int) -> None:
        for _ in range(nsteps):
            self.step()

    def gather(self) -> dict:
        """The owned bodies' arrays on the host, with their global indices."""
        return {k: v.detach().cpu().numpy() for k, v in self.owned.items()}
