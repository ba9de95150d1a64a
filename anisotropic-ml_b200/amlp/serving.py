"""Continuous-batching server for many independent rigid-body NVT systems on one GPU.

Requests (particle count, shape, packing fraction, kT, number of steps) arrive
over time. Each is admitted, in arrival order, as soon as its memory fits a
fixed HBM budget. Admitted systems stay resident on the device until they
finish.

Systems of one shape share a bucket, buffers of a fixed capacity:
- each system owns a contiguous range of body slots and one system slot; a
  per-body system index points at per-system box, temperature, degrees of
  freedom and thermostat; free body slots (index -1) and free system slots are
  skipped by the kernels;
- one time step of a bucket is: the pair filter, the adjoint force kernel
  (net on the tensor cores), and the two NVT halves, each a single launch over
  the bucket's capacity (``amlp_multi_*``), with the same arguments whatever
  systems are resident.

The server advances all buckets in segments of ``segment`` steps (100, the
Verlet rebuild period of the reference, ``Sim.py:87``). Each segment:
- rebuilds every system's Verlet list;
- replays one CUDA graph holding all steps of all buckets, one branch per
  bucket so that the buckets' kernels run concurrently. It is captured once
  and captured again only when a bucket's capacity grows, so admissions and
  departures cost a few small copies, not a capture;
- then admits new arrivals and retires finished systems. This is the only time
  the set of systems can change.

Throughput (particle-steps/s over the wall time), per-segment latency
percentiles (device time of the replay, and wall time of lists + replay) and
per-request completion latencies are recorded. Admissions and request latencies
run on the device time of the segments (plus jumps over idle gaps), so a seeded
stream is served the same way every run.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import Nvt, Thermostat, call, size_query
from .configs import make_state
from .engine import THERMOSTAT_SEED, EnergyNet, Hypers
from .shapes import get_shape


Replica = _lib.Replica


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


@dataclass
class Request:
    rid: int
    n: int
    shape: str
    phi: float
    kT: float
    steps: int
    arrival: float = 0.0      # seconds after the start of the run
    seed: int = 0


@dataclass
class _System:
    req: Request
    state: object
    done: int = 0
    th: bytes = b""            # thermostat bytes carried across re-packs
    admitted_at: float = 0.0
    finished_at: float = 0.0
    mem: int = 0


def verlet_capacity(n: int, shape, phi: float, r: float) -> int:
    """Capacity for the Verlet list: 1.5x the ideal-gas estimate plus slack."""
    rho = phi / shape.volume
    est = 0.5 * n * rho * 4.0 / 3.0 * math.pi * r ** 3
    return int(1.5 * est) + 4 * n + 1024


def system_bytes(n: int, shape, phi: float) -> int:
    """Device memory of one resident system (state, pair lists, workspaces)."""
    cap = verlet_capacity(n, shape, phi, shape.cutoff + 2.0)
    return n * 128 + cap * 16 + size_query("amlp_nlist_workspace_bytes", n, 10.0 * shape.cutoff, shape.cutoff + 2.0)


class _Bucket:
    """All active systems of one shape, in buffers of a fixed capacity.

    Every admitted system gets a system slot r (its box, temperature, degrees of
    freedom and thermostat in row r of ``rp`` / ``th``) and a contiguous range of
    body slots; free body slots have ``rep = -1`` and free system slots
    ``n_dof = 0``, which the multi-system kernels skip. The launches of a step
    therefore have the same arguments whatever the active set, and one captured
    CUDA graph serves every segment until a capacity has to grow."""

    def __init__(self, shape_name: str, net: EnergyNet, hypers: Hypers, dt: float, device,
                 body_cap: int = 1 << 16, sys_cap: int = 64):
        self.shape = get_shape(shape_name)
        self.net, self.hypers, self.dt, self.device = net, hypers, dt, device
        self.systems: list[_System] = []
        self.pts = torch.tensor(self.shape.pts, dtype=torch.float32, device=device)
        self.nep = _lib.Nep()
        self.nep.nrad, self.nep.nang, self.nep.lmax = hypers.nrad, hypers.nang, hypers.lmax
        self.nep.npts = self.shape.npts
        self.nep.d_pts = self.pts.data_ptr()
        self.nep.cutoff = float(self.shape.cutoff)
        self.nep.nep_cutoff = float(self.shape.nep_cutoff)
        self.nep.en_min, self.nep.en_max = float(self.shape.en_min), float(self.shape.en_max)
        self.nep.dx = self.nep.dteta = 1e-5
        self.prm = Nvt()
        self.prm.dt = float(dt)
        self.prm.tau = float(np.float32(100.0 * dt))
        for k in range(3):
            self.prm.moi[k] = float(self.shape.moi[k])
        self.r_verlet = float(self.shape.cutoff) + 2.0
        self.where = {}            # rid -> (system slot, first body slot)
        self.generation = 0        # bumped whenever the buffers are reallocated
        self._alloc(body_cap, sys_cap, 1 << 20)

    # -------------------------------------------------------------- buffers
    def _alloc(self, body_cap: int, sys_cap: int, pair_cap: int) -> None:
        """(Re)allocate every buffer at the given capacities, keeping the
        resident systems' state."""
        keep = self._snapshot_states() if getattr(self, "systems", None) and hasattr(self, "pos") else {}
        keep_th = {s.req.rid: self._thermostat_bytes(s) for s in self.systems} if keep else {}
        f32 = dict(dtype=torch.float32, device=self.device)
        self.body_cap, self.sys_cap, self.cap = int(body_cap), int(sys_cap), int(pair_cap)
        self.pos = torch.zeros(self.body_cap, 3, **f32)
        self.quat = torch.zeros(self.body_cap, 4, **f32)
        self.quat[:, 0] = 1.0
        self.vel = torch.zeros(self.body_cap, 3, **f32)
        self.angmom = torch.zeros(self.body_cap, 4, **f32)
        self.mass = torch.ones(self.body_cap, **f32)
        self.rep = torch.full((self.body_cap,), -1, dtype=torch.int32, device=self.device)
        self.F = torch.zeros(self.body_cap, 3, **f32)
        self.T = torch.zeros(self.body_cap, 3, **f32)
        self.accel = torch.zeros(self.body_cap, 3, **f32)
        self.dp = torch.zeros(self.body_cap, 4, **f32)
        self.rp = torch.zeros(self.sys_cap * ctypes.sizeof(Replica), dtype=torch.uint8, device=self.device)
        self.th = torch.zeros(self.sys_cap * ctypes.sizeof(Thermostat), dtype=torch.uint8, device=self.device)
        self.pe = torch.zeros(self.sys_cap, dtype=torch.float64, device=self.device)
        self.vpairs = torch.empty(self.cap, 2, dtype=torch.int32, device=self.device)
        self.vgap = torch.empty(self.cap, 2, dtype=torch.int32, device=self.device)
        self.fpairs = torch.empty(self.cap, 2, dtype=torch.int32, device=self.device)
        self.nv = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.nf = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.counts = torch.zeros(self.sys_cap, dtype=torch.int64, device=self.device)
        self.nl_ws = torch.empty(0, dtype=torch.uint8, device=self.device)
        self.f_ws = torch.empty(size_query("amlp_filter_workspace_bytes", self.cap), dtype=torch.uint8,
                                device=self.device)
        self.adj_ws = None
        if self.net.max_hidden > 64 or self.hypers.D > 48:  # beyond the fused adjoint kernel: the wide path
            self.adj_ws = torch.empty(size_query("amlp_adjoint_workspace_bytes", self.cap), dtype=torch.uint8,
                                      device=self.device)
        self.free_sys = list(range(self.sys_cap))
        self.free_bodies = [(0, self.body_cap)]   # (first, length), sorted by first
        self.where = {}
        self.generation += 1
        old = self.systems
        self.systems = []
        if old:
            self._place([(s, keep[s.req.rid], keep_th[s.req.rid]) for s in old])

    def _take_bodies(self, n: int) -> int | None:
        for k, (a, m) in enumerate(self.free_bodies):
            if m >= n:
                self.free_bodies[k] = (a + n, m - n)
                if m == n:
                    del self.free_bodies[k]
                return a
        return None

    def _give_bodies(self, a: int, n: int) -> None:
        self.free_bodies.append((a, n))
        self.free_bodies.sort()
        merged = []
        for b, m in self.free_bodies:
            if merged and merged[-1][0] + merged[-1][1] == b:
                merged[-1] = (merged[-1][0], merged[-1][1] + m)
            else:
                merged.append((b, m))
        self.free_bodies = merged

    # -------------------------------------------------------------- admission
    def _thermostat_bytes(self, s: _System) -> bytes:
        r = self.where[s.req.rid][0]
        tsz = ctypes.sizeof(Thermostat)
        return self.th[r * tsz:(r + 1) * tsz].cpu().numpy().tobytes()

    def _place(self, entries) -> None:
        """Put (system, host state, thermostat bytes or b"") entries into free slots."""
        tsz, rsz = ctypes.sizeof(Thermostat), ctypes.sizeof(Replica)
        for s, st, thb in entries:
            n = s.req.n
            r = self.free_sys.pop(0)
            a = self._take_bodies(n)
            for name, t in (("pos", self.pos), ("orient", self.quat), ("vel", self.vel), ("angmom", self.angmom),
                            ("mass", self.mass)):
                t[a:a + n].copy_(torch.from_numpy(np.ascontiguousarray(getattr(st, name), np.float32)))
            self.rep[a:a + n] = r
            q = Replica()
            q.kT, q.n_dof, q.rn_dof, q.box, q.nve = s.req.kT, float((n - 1) * 3), float(n * 3), float(st.L), 0
            self.rp[r * rsz:(r + 1) * rsz].copy_(torch.frombuffer(bytearray(bytes(q)), dtype=torch.uint8))
            if not thb:
                t = Thermostat()
                t.xi, t.eta, t.xi_rot, t.eta_rot, t.thermo_fac = THERMOSTAT_SEED
                thb = bytes(t)
            self.th[r * tsz:(r + 1) * tsz].copy_(torch.frombuffer(bytearray(thb), dtype=torch.uint8))
            self.where[s.req.rid] = (r, a)
            s.state = st
            self.systems.append(s)
        # kinetic energies of every system from its current state (the value step one
        # would have left), so that step two of the next segment starts right
        call("amlp_multi_nvt_init", self.vel.data_ptr(), self.quat.data_ptr(), self.angmom.data_ptr(),
             self.mass.data_ptr(), self.rep.data_ptr(), self.body_cap, self.sys_cap, ctypes.byref(self.prm),
             self.th.data_ptr(), _stream())

    def _verlet_cap(self, s: _System) -> int:
        return verlet_capacity(s.req.n, self.shape, s.req.phi, self.r_verlet)

    def admit(self, new: list[_System]) -> None:
        """Admit systems (their states from their requests); grows the buffers
        (a new generation) when a capacity is short."""
        if not new:
            return
        bodies = sum(m for _, m in self.free_bodies)
        need_b = sum(s.req.n for s in new)
        need_s = len(self.systems) + len(new)
        need_p = sum(self._verlet_cap(s) for s in self.systems + new)
        fits = need_s <= self.sys_cap and need_p <= self.cap and bodies >= need_b
        if fits:  # a contiguous range for each new system, tried on a copy of the free list
            trial = list(self.free_bodies)
            for s in new:
                k = next((k for k, (_, m) in enumerate(trial) if m >= s.req.n), None)
                if k is None:
                    fits = False
                    break
                a, m = trial[k]
                trial[k] = (a + s.req.n, m - s.req.n)
        if not fits:
            used = sum(s.req.n for s in self.systems)
            bc, sc, pc = self.body_cap, self.sys_cap, self.cap
            while bc < 2 * (used + need_b):  # headroom against fragmentation
                bc *= 2
            while sc < need_s:
                sc *= 2
            while pc < need_p:
                pc *= 2
            self._alloc(bc, sc, pc)
        self._place([(s, s.state, b"") for s in new])

    def retire(self, gone: list[_System]) -> dict:
        """Remove systems; returns their host states {rid: State}."""
        if not gone:
            return {}
        states = self._snapshot_states([s.req.rid for s in gone])
        rsz = ctypes.sizeof(Replica)
        for s in gone:
            r, a = self.where.pop(s.req.rid)
            self.rep[a:a + s.req.n] = -1
            self.rp[r * rsz:(r + 1) * rsz].zero_()  # n_dof = 0: a free system slot
            self.free_sys.append(r)
            self._give_bodies(a, s.req.n)
        self.free_sys.sort()
        ids = {s.req.rid for s in gone}
        self.systems = [s for s in self.systems if s.req.rid not in ids]
        return states

    def _snapshot_states(self, rids=None) -> dict:
        out = {}
        if not self.systems:
            return out
        pos, quat, vel, ang, mass = (t.cpu().numpy() for t in (self.pos, self.quat, self.vel, self.angmom, self.mass))
        for s in self.systems:
            if rids is not None and s.req.rid not in rids:
                continue
            _, a = self.where[s.req.rid]
            b = a + s.req.n
            out[s.req.rid] = type(s.state)(pos=pos[a:b].copy(), orient=quat[a:b].copy(), vel=vel[a:b].copy(),
                                           angmom=ang[a:b].copy(), mass=mass[a:b].copy(), moi=s.state.moi,
                                           L=s.state.L)
        return out

    def unpack(self, s: _System):
        """Host copy of system s's state (positions, orientations, velocities, angular momenta)."""
        return self._snapshot_states([s.req.rid])[s.req.rid]

    # -------------------------------------------------------------- stepping
    def rebuild_lists(self) -> None:
        """Verlet list of every system (``amlp_nlist_build`` per system into its
        own slot), then one contiguous list with global body indices."""
        if not self.systems:
            self.nv.zero_()
            return
        st = _stream()
        caps = [self._verlet_cap(s) for s in self.systems]
        slot = np.concatenate([[0], np.cumsum(caps)[:-1]]).astype(np.int64)
        ws = max(size_query("amlp_nlist_workspace_bytes", s.req.n, float(s.state.L), self.r_verlet)
                 for s in self.systems)
        if self.nl_ws.numel() < ws:
            self.nl_ws = torch.empty(ws, dtype=torch.uint8, device=self.device)
        firsts = []
        for k, s in enumerate(self.systems):
            _, a = self.where[s.req.rid]
            firsts.append(a)
            call("amlp_nlist_build", self.pos[a:a + s.req.n].data_ptr(), s.req.n, float(s.state.L), self.r_verlet,
                 self.vgap[int(slot[k]):].data_ptr(), caps[k], self.counts[k:k + 1].data_ptr(),
                 self.nl_ws.data_ptr(), self.nl_ws.numel(), st)
        counts = self.counts[:len(self.systems)].cpu().numpy()
        if np.any(counts > np.asarray(caps)):
            raise RuntimeError("Verlet list of a served system exceeds its capacity")
        parts = [self.vgap[int(slot[k]):int(slot[k]) + int(counts[k])] + int(firsts[k])
                 for k in range(len(self.systems)) if counts[k]]
        total = int(counts.sum())
        if parts:
            torch.cat(parts, out=self.vpairs[:total])
        self.nv.fill_(total)

    def step_kernels(self) -> None:
        """One step of every system of the bucket: the same launches whatever the active set."""
        st = _stream()
        self.F.zero_()
        self.T.zero_()
        self.pe.zero_()
        call("amlp_multi_pair_filter", self.pos.data_ptr(), self.rep.data_ptr(), self.rp.data_ptr(),
             float(self.shape.cutoff), self.vpairs.data_ptr(), self.nv.data_ptr(), self.cap, self.fpairs.data_ptr(),
             self.nf.data_ptr(), self.f_ws.data_ptr(), self.f_ws.numel(), st)
        args = [self.pos.data_ptr(), self.quat.data_ptr(), self.rep.data_ptr(), self.rp.data_ptr(),
                self.fpairs.data_ptr(), self.nf.data_ptr(), self.cap, ctypes.byref(self.nep),
                ctypes.byref(self.net.struct), self.F.data_ptr(), self.T.data_ptr(), self.pe.data_ptr()]
        if self.adj_ws is None:
            call("amlp_multi_forces_adjoint", *args, st)
        else:
            call("amlp_multi_forces_adjoint_wide", *args, self.adj_ws.data_ptr(), self.adj_ws.numel(), st)
        call("amlp_multi_nvt_step_two", self.vel.data_ptr(), self.accel.data_ptr(), self.F.data_ptr(),
             self.mass.data_ptr(), self.quat.data_ptr(), self.T.data_ptr(), self.angmom.data_ptr(),
             self.dp.data_ptr(), self.rep.data_ptr(), self.body_cap, self.sys_cap, self.rp.data_ptr(),
             ctypes.byref(self.prm), self.th.data_ptr(), st)
        call("amlp_multi_nvt_step_one", self.pos.data_ptr(), self.vel.data_ptr(), self.accel.data_ptr(),
             self.quat.data_ptr(), self.angmom.data_ptr(), self.dp.data_ptr(), self.mass.data_ptr(),
             self.rep.data_ptr(), self.body_cap, self.rp.data_ptr(), ctypes.byref(self.prm), self.th.data_ptr(), st)


@dataclass
class ServeStats:
    segments_ms: list = field(default_factory=list)
    completions: list = field(default_factory=list)    # (rid, latency s)
    body_steps: int = 0
    wall_s: float = 0.0
    max_active: int = 0
    graphs_captured: int = 0

    segments_wall_ms: list = field(default_factory=list)
    server_clock_s: float = 0.0

    def summary(self) -> dict:
        seg = np.asarray(self.segments_ms) if self.segments_ms else np.zeros(1)
        wall = np.asarray(self.segments_wall_ms) if self.segments_wall_ms else np.zeros(1)
        lat = np.asarray([c[1] for c in self.completions]) if self.completions else np.zeros(1)
        return {"particle_steps_per_s": self.body_steps / self.wall_s if self.wall_s else 0.0,
                "particle_steps_per_s_server_clock": (self.body_steps / self.server_clock_s
                                                      if self.server_clock_s else 0.0),
                "server_clock_s": self.server_clock_s,
                "segment_ms_p50": float(np.percentile(seg, 50)), "segment_ms_p99": float(np.percentile(seg, 99)),
                "segment_wall_ms_p50": float(np.percentile(wall, 50)),
                "segment_wall_ms_p99": float(np.percentile(wall, 99)),
                "request_latency_s_p50": float(np.percentile(lat, 50)),
                "request_latency_s_p99": float(np.percentile(lat, 99)),
                "segments": len(self.segments_ms), "requests": len(self.completions),
                "max_concurrent": self.max_active, "graphs_captured": self.graphs_captured,
                "wall_s": self.wall_s, "particle_steps": self.body_steps}


class Server:
    """Continuous-batching NVT server (see the module docstring)."""

    def __init__(self, nets: dict, hbm_budget: int, dt: float = 0.005, segment: int = 100, device="cuda",
                 hypers: Hypers | None = None, use_graphs: bool = True, clock: str = "device"):
        if clock not in ("device", "wall"):
            raise ValueError(f"clock must be 'device' or 'wall', not {clock!r}")
        self.clock = clock
        self.device = torch.device(device)
        self.hypers = hypers or Hypers()
        self.buckets = {k: _Bucket(k, v, self.hypers, dt, self.device) for k, v in nets.items()}
        self.budget = int(hbm_budget)
        self.segment = int(segment)
        self.use_graphs = use_graphs
        self.used = 0
        self._graph = None
        self._graph_key = None
        self._branches = {}
        self.results = {}

    def _branch(self, b) -> torch.cuda.Stream:
        """The side stream that bucket b's steps are captured on."""
        if id(b) not in self._branches:
            self._branches[id(b)] = torch.cuda.Stream(device=self.device)
        return self._branches[id(b)]

    def _admit(self, req: Request, now: float) -> _System:
        shape = get_shape(req.shape)
        st = make_state(req.n, shape, req.phi, kT=req.kT, seed=req.seed)
        return _System(req=req, state=st, admitted_at=now, mem=system_bytes(req.n, shape, req.phi))

    def _segment(self, steps: int) -> tuple[float, float]:
        """Run `steps` steps of every bucket: the Verlet lists, then one graph
        replay. Returns (device ms of the replay, wall ms of lists + replay). The
        graph is captured again only when a bucket's buffers were reallocated."""
        key = tuple(b.generation for b in self.buckets.values()) + (steps,)
        if self.use_graphs and key != self._graph_key:
            self._graph = None
            for b in self.buckets.values():
                b.rebuild_lists()
            for b in self.buckets.values():   # warm-up launch sets kernel attributes outside capture
                snap = [t.clone() for t in (b.pos, b.quat, b.vel, b.angmom, b.th)]
                b.step_kernels()
                torch.cuda.synchronize()
                for t, v in zip((b.pos, b.quat, b.vel, b.angmom, b.th), snap):
                    t.copy_(v)
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    # one branch per bucket: the buckets share no buffer, so their steps run
                    # concurrently and fill each other's idle SMs (a persistent force kernel with
                    # few tiles leaves most of the GPU free at its tail)
                    for b in self.buckets.values():
                        bs = self._branch(b)
                        bs.wait_stream(s)
                        with torch.cuda.stream(bs):
                            for _ in range(steps):
                                b.step_kernels()
                        s.wait_stream(bs)
            torch.cuda.current_stream().wait_stream(s)
            torch.cuda.synchronize()
            self._graph, self._graph_key = g, key
            self.stats.graphs_captured += 1
        t0 = time.perf_counter()
        for b in self.buckets.values():
            b.rebuild_lists()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        if self.use_graphs:
            self._graph.replay()
        else:
            for _ in range(steps):
                for b in self.buckets.values():
                    b.step_kernels()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1), (time.perf_counter() - t0) * 1e3

    def run(self, requests: list[Request], keep_states: bool = False) -> ServeStats:
        """Serve `requests` (arrival times in seconds from the start) to completion.

        The server's clock (admissions, request latencies) is the device time of
        the segments served so far, plus the jumps over idle gaps to the next
        arrival: it does not see host work or graph captures, so the same stream
        gives the same admissions, resident sets and segment sizes from run to
        run. ``clock="wall"`` uses the host's clock instead. The aggregate
        throughput is over the wall time either way."""
        self.stats = ServeStats()
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        active: list[_System] = []
        t0 = time.perf_counter()
        shift = 0.0
        device_s = 0.0

        def clock() -> float:
            return (device_s if self.clock == "device" else time.perf_counter() - t0) + shift

        while pending or active:
            now = clock()
            if not active and pending and pending[0].arrival > now:
                shift += pending[0].arrival - now    # idle: jump to the next arrival
                now = pending[0].arrival
            admitted = []
            while pending and pending[0].arrival <= now:
                shape = get_shape(pending[0].shape)
                need = system_bytes(pending[0].n, shape, pending[0].phi)
                if need > self.budget:
                    raise ValueError(f"request {pending[0].rid} needs {need} B, above the whole budget")
                if self.used + need > self.budget:
                    break                           # first-come first-served: wait for memory
                sysm = self._admit(pending.pop(0), now)
                self.used += sysm.mem
                active.append(sysm)
                admitted.append(sysm)
            if admitted:
                for name, b in self.buckets.items():
                    b.admit([s for s in admitted if s.req.shape == name])
            if not active:
                continue
            self.stats.max_active = max(self.stats.max_active, len(active))
            steps = min(self.segment, min(s.req.steps - s.done for s in active))
            ms, wall_ms = self._segment(steps)
            device_s += ms / 1e3
            self.stats.segments_ms.append(ms * self.segment / steps)
            self.stats.segments_wall_ms.append(wall_ms * self.segment / steps)
            self.stats.body_steps += steps * sum(s.req.n for s in active)
            finished = []
            for s in active:
                s.done += steps
                if s.done >= s.req.steps:
                    finished.append(s)
            if finished:
                now = clock()
                for name, b in self.buckets.items():
                    gone = [s for s in b.systems if s in finished]
                    if gone:
                        states = b.retire(gone)
                        for s in gone:
                            s.finished_at = now
                            self.stats.completions.append((s.req.rid, now - s.req.arrival))
                            if keep_states:
                                self.results[s.req.rid] = states[s.req.rid]
                            self.used -= s.mem
                active = [s for s in active if s not in finished]
        self.stats.wall_s = time.perf_counter() - t0
        self.stats.server_clock_s = clock()
        return self.stats


def request_stream(n_requests: int, seed: int, steps: int, rate: float, n_range=(500, 50000),
                   shapes=("cube26", "tetra16", "cyl24"), phi_range=(0.25, 0.45), kT_range=(0.5, 2.0)) -> list:
    """Seeded stream: Poisson arrivals at `rate` per second, N log-uniform,
    shape uniform, packing fraction and kT uniform."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n_requests):
        t += rng.exponential(1.0 / rate)
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        out.append(Request(rid=k, n=n, shape=str(rng.choice(shapes)), phi=float(rng.uniform(*phi_range)),
                           kT=float(rng.uniform(*kT_range)), steps=steps, arrival=t, seed=int(rng.integers(1 << 30))))
    return out
