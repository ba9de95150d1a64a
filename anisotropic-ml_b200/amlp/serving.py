"""Continuous-batching server for many independent rigid-body NVT systems on one GPU.

Requests (particle count, shape, packing fraction, kT, number of steps) arrive
over time. Each is admitted, in arrival order, as soon as its memory fits a
fixed HBM budget. Admitted systems stay resident on the device until they
finish.

Systems of one shape are packed into a bucket:
- bodies are concatenated, and a per-body system index points at per-system
  box, temperature, degrees of freedom and thermostat;
- one time step of a bucket is: the pair filter, the adjoint force kernel
  (net on the tensor cores), and the two NVT halves, each a single launch over
  every system of the bucket (``amlp_multi_*``).

The server advances all buckets in segments of ``segment`` steps (100, the
Verlet rebuild period of the reference, ``Sim.py:87``). Each segment:
- rebuilds every system's Verlet list;
- replays one captured CUDA graph holding all steps of all buckets;
- then admits new arrivals and retires finished systems. This is the only time
  the set of systems can change.

Throughput (particle-steps/s), per-segment latency percentiles and
per-request completion latencies are recorded.
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
    """All active systems of one shape, packed for multi-system launches."""

    def __init__(self, shape_name: str, net: EnergyNet, hypers: Hypers, dt: float, device):
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
        self.N = 0

    # -------------------------------------------------------------- packing
    def pack(self, systems: list[_System]) -> None:
        """Lay out `systems` (states from the previous packing or new) contiguously."""
        old = self._snapshot_states() if self.N else {}
        self.systems = systems
        f32 = dict(dtype=torch.float32, device=self.device)
        ns = [s.req.n for s in systems]
        self.N = sum(ns)
        self.first = np.concatenate([[0], np.cumsum(ns)[:-1]]).astype(np.int64) if ns else np.zeros(0, np.int64)
        if not systems:
            return
        host = {k: [] for k in ("pos", "orient", "vel", "angmom", "mass")}
        for s in systems:
            st = old.get(s.req.rid, s.state)
            for k in host:
                host[k].append(np.asarray(getattr(st, k), np.float32))
        self.pos = torch.tensor(np.concatenate(host["pos"]), **f32)
        self.quat = torch.tensor(np.concatenate(host["orient"]), **f32)
        self.vel = torch.tensor(np.concatenate(host["vel"]), **f32)
        self.angmom = torch.tensor(np.concatenate(host["angmom"]), **f32)
        self.mass = torch.tensor(np.concatenate(host["mass"]), **f32)
        self.rep = torch.tensor(np.repeat(np.arange(len(systems), dtype=np.int32), ns), device=self.device)
        self.F = torch.zeros(self.N, 3, **f32)
        self.T = torch.zeros(self.N, 3, **f32)
        self.accel = torch.zeros(self.N, 3, **f32)
        self.dp = torch.zeros(self.N, 4, **f32)
        rp = (Replica * len(systems))()
        th = bytearray()
        for r, s in enumerate(systems):
            rp[r].kT = s.req.kT
            rp[r].n_dof = float((s.req.n - 1) * 3)
            rp[r].rn_dof = float(s.req.n * 3)
            rp[r].box = float(s.state.L)
            rp[r].nve = 0
            if s.th:
                th += s.th
            else:
                t = Thermostat()
                t.xi, t.eta, t.xi_rot, t.eta_rot, t.thermo_fac = THERMOSTAT_SEED
                th += bytes(t)
        self.rp = torch.frombuffer(bytearray(bytes(rp)), dtype=torch.uint8).to(self.device)
        self.th = torch.frombuffer(th, dtype=torch.uint8).to(self.device)
        self.pe = torch.zeros(len(systems), dtype=torch.float64, device=self.device)
        caps = [verlet_capacity(s.req.n, self.shape, s.req.phi, self.r_verlet) for s in systems]
        self.caps = caps
        self.cap = sum(caps)
        self.vpairs = torch.empty(self.cap, 2, dtype=torch.int32, device=self.device)
        self.vgap = torch.empty(self.cap, 2, dtype=torch.int32, device=self.device)
        self.fpairs = torch.empty(self.cap, 2, dtype=torch.int32, device=self.device)
        self.nv = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.nf = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.counts = torch.zeros(len(systems), dtype=torch.int64, device=self.device)
        self.nl_ws = torch.empty(max(size_query("amlp_nlist_workspace_bytes", s.req.n, float(s.state.L), self.r_verlet)
                                     for s in systems), dtype=torch.uint8, device=self.device)
        self.f_ws = torch.empty(size_query("amlp_filter_workspace_bytes", self.cap), dtype=torch.uint8,
                                device=self.device)
        self.adj_ws = None
        if self.net.max_hidden > 64:  # wider nets take the three-kernel adjoint path
            self.adj_ws = torch.empty(size_query("amlp_adjoint_workspace_bytes", self.cap), dtype=torch.uint8,
                                      device=self.device)
        call("amlp_multi_nvt_init", self.vel.data_ptr(), self.quat.data_ptr(), self.angmom.data_ptr(),
             self.mass.data_ptr(), self.rep.data_ptr(), self.N, len(systems), ctypes.byref(self.prm),
             self.th.data_ptr(), _stream())

    def _snapshot_states(self) -> dict:
        out = {}
        if not self.systems:
            return out
        pos, quat, vel, ang, mass = (t.cpu().numpy() for t in (self.pos, self.quat, self.vel, self.angmom, self.mass))
        thb = self.th.cpu().numpy().tobytes()
        tsz = ctypes.sizeof(Thermostat)
        for r, s in enumerate(self.systems):
            a, b = int(self.first[r]), int(self.first[r]) + s.req.n
            s.th = thb[r * tsz:(r + 1) * tsz]
            out[s.req.rid] = type(s.state)(pos=pos[a:b], orient=quat[a:b], vel=vel[a:b], angmom=ang[a:b],
                                           mass=mass[a:b], moi=s.state.moi, L=s.state.L)
        return out

    def unpack(self, s: _System):
        """Host copy of system s's state (positions, orientations, velocities, angular momenta)."""
        return self._snapshot_states()[s.req.rid]

    # -------------------------------------------------------------- stepping
    def rebuild_lists(self) -> None:
        """Verlet list of every system (``amlp_nlist_build`` per system into its
        own slot), then one contiguous list with global body indices."""
        if not self.systems:
            return
        st = _stream()
        slot = np.concatenate([[0], np.cumsum(self.caps)[:-1]]).astype(np.int64)
        for r, s in enumerate(self.systems):
            a, n = int(self.first[r]), s.req.n
            call("amlp_nlist_build", self.pos[a:a + n].data_ptr(), n, float(s.state.L), self.r_verlet,
                 self.vgap[int(slot[r]):].data_ptr(), self.caps[r], self.counts[r:r + 1].data_ptr(),
                 self.nl_ws.data_ptr(), self.nl_ws.numel(), st)
        counts = self.counts.cpu().numpy()
        if np.any(counts > np.asarray(self.caps)):
            raise RuntimeError("Verlet list of a served system exceeds its capacity")
        parts = [self.vgap[int(slot[r]):int(slot[r]) + int(counts[r])] + int(self.first[r])
                 for r in range(len(self.systems)) if counts[r]]
        total = int(counts.sum())
        if parts:
            torch.cat(parts, out=self.vpairs[:total])
        self.nv.fill_(total)

    def step_kernels(self) -> None:
        if not self.systems:
            return
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
             self.dp.data_ptr(), self.rep.data_ptr(), self.N, len(self.systems), self.rp.data_ptr(),
             ctypes.byref(self.prm), self.th.data_ptr(), st)
        call("amlp_multi_nvt_step_one", self.pos.data_ptr(), self.vel.data_ptr(), self.accel.data_ptr(),
             self.quat.data_ptr(), self.angmom.data_ptr(), self.dp.data_ptr(), self.mass.data_ptr(),
             self.rep.data_ptr(), self.N, self.rp.data_ptr(), ctypes.byref(self.prm), self.th.data_ptr(), st)


@dataclass
class ServeStats:
    segments_ms: list = field(default_factory=list)
    completions: list = field(default_factory=list)    # (rid, latency s)
    body_steps: int = 0
    wall_s: float = 0.0
    max_active: int = 0
    graphs_captured: int = 0

    def summary(self) -> dict:
        seg = np.asarray(self.segments_ms) if self.segments_ms else np.zeros(1)
        lat = np.asarray([c[1] for c in self.completions]) if self.completions else np.zeros(1)
        return {"particle_steps_per_s": self.body_steps / self.wall_s if self.wall_s else 0.0,
                "segment_ms_p50": float(np.percentile(seg, 50)), "segment_ms_p99": float(np.percentile(seg, 99)),
                "request_latency_s_p50": float(np.percentile(lat, 50)),
                "request_latency_s_p99": float(np.percentile(lat, 99)),
                "segments": len(self.segments_ms), "requests": len(self.completions),
                "max_concurrent": self.max_active, "graphs_captured": self.graphs_captured,
                "wall_s": self.wall_s, "particle_steps": self.body_steps}


class Server:
    """Continuous-batching NVT server (see the module docstring)."""

    def __init__(self, nets: dict, hbm_budget: int, dt: float = 0.005, segment: int = 100, device="cuda",
                 hypers: Hypers | None = None, use_graphs: bool = True):
        self.device = torch.device(device)
        self.hypers = hypers or Hypers()
        self.buckets = {k: _Bucket(k, v, self.hypers, dt, self.device) for k, v in nets.items()}
        self.budget = int(hbm_budget)
        self.segment = int(segment)
        self.use_graphs = use_graphs
        self.used = 0
        self._graph = None
        self._graph_key = None
        self.results = {}

    def _admit(self, req: Request, now: float) -> _System:
        shape = get_shape(req.shape)
        st = make_state(req.n, shape, req.phi, kT=req.kT, seed=req.seed)
        return _System(req=req, state=st, admitted_at=now, mem=system_bytes(req.n, shape, req.phi))

    def _segment(self, steps: int) -> float:
        """Run `steps` steps of every bucket; returns device milliseconds."""
        for b in self.buckets.values():
            b.rebuild_lists()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        key = tuple((k, tuple(s.req.rid for s in b.systems)) for k, b in self.buckets.items()) + (steps,)
        if self.use_graphs and key != self._graph_key:
            self._graph = None
            for b in self.buckets.values():   # warm-up launch sets kernel attributes outside capture
                if b.systems:
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
                    for _ in range(steps):
                        for b in self.buckets.values():
                            b.step_kernels()
            torch.cuda.current_stream().wait_stream(s)
            self._graph, self._graph_key = g, key
            self.stats.graphs_captured += 1
        ev0.record()
        if self.use_graphs:
            self._graph.replay()
        else:
            for _ in range(steps):
                for b in self.buckets.values():
                    b.step_kernels()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1)

    def run(self, requests: list[Request], keep_states: bool = False) -> ServeStats:
        """Serve `requests` (arrival times in seconds from now) to completion."""
        self.stats = ServeStats()
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        active: list[_System] = []
        t0 = time.perf_counter()
        shift = 0.0
        while pending or active:
            now = time.perf_counter() - t0 + shift
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
                    new = [s for s in admitted if s.req.shape == name]
                    if new:
                        b.pack(b.systems + new)
            if not active:
                continue
            self.stats.max_active = max(self.stats.max_active, len(active))
            steps = min(self.segment, min(s.req.steps - s.done for s in active))
            ms = self._segment(steps)
            self.stats.segments_ms.append(ms * self.segment / steps)
            self.stats.body_steps += steps * sum(s.req.n for s in active)
            finished = []
            for s in active:
                s.done += steps
                if s.done >= s.req.steps:
                    finished.append(s)
            if finished:
                now = time.perf_counter() - t0 + shift
                for name, b in self.buckets.items():
                    gone = [s for s in b.systems if s in finished]
                    if gone:
                        states = b._snapshot_states()
                        for s in gone:
                            s.finished_at = now
                            self.stats.completions.append((s.req.rid, now - s.req.arrival))
                            if keep_states:
                                self.results[s.req.rid] = states[s.req.rid]
                            self.used -= s.mem
                        b.pack([s for s in b.systems if s not in finished])
                active = [s for s in active if s not in finished]
        self.stats.wall_s = time.perf_counter() - t0
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
