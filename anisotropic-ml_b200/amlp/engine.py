"""Device-resident rigid-body NVT system driving ``libamlp`` (host side).

``System`` owns the state in torch tensors on one GPU and sequences the C-ABI
calls of one time step exactly as ``Sim.step`` does (``Sim.py:257-285``):
force pass (pair filter, descriptors, net, forces/torques), then
``integrate_step_two``, then ``integrate_step_one``; the Verlet list is rebuilt
every ``nlist_every`` steps (100, ``Sim.py:87``). ``run`` replays segments of
steps as CUDA graphs.

Verlet-list policies: ``"every"`` (the reference's fixed schedule) and
``"displacement"``: every step checks on the device whether some body has moved
more than half the skin since the list was built and rebuilds only then (the
check and the gated build sit inside the graphs). A rebuild that overflows the
list's capacity is detected after the segment, which is then run again from a
snapshot with a larger list.

Force methods:
* ``"fd"``       -- the reference's finite differences, one fused kernel;
* ``"fd_split"`` -- the same through the three kernels that keep g_all in HBM
                    (the reference's own data flow; any net width);
* ``"adjoint"``  -- analytic forces/torques (one descriptor pass per pair).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import ACT, Mlp, Nep, Nvt, Thermostat, call, size_query
from .configs import State
from .shapes import Shape, get_shape

THERMOSTAT_SEED = (-0.0317711, 0.108609, 0.00814227, -0.014238, 1.00011)  # Sim.setkT, Sim.py:101-105


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class EnergyNet:
    """FFNN pair energy (``TheEnergyNet``, ``ForceEvaluator.py:6-26``) with its
    weights packed for the library: per layer W (out x in, row-major) then b."""

    def __init__(self, layers, act: str = "relu", device="cuda"):
        if act not in ACT:
            raise ValueError(f"activation {act!r} not in {sorted(ACT)}")
        self.layers = [(np.asarray(W, np.float32), np.asarray(b, np.float32).reshape(-1)) for W, b in layers]
        self.act = act
        dims = [self.layers[0][0].shape[1]] + [W.shape[0] for W, _ in self.layers]
        for k, (W, b) in enumerate(self.layers):
            if W.shape != (dims[k + 1], dims[k]) or b.shape != (dims[k + 1],):
                raise ValueError(f"layer {k}: weight {W.shape} / bias {b.shape} do not chain")
        if dims[-1] != 1:
            raise ValueError("the last layer must have one output")
        if len(self.layers) > _lib.MAX_LAYERS:
            raise ValueError(f"at most {_lib.MAX_LAYERS} layers")
        self.dims = dims
        packed = np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in self.layers]).astype(np.float32)
        self.device = torch.device(device)
        self.d_w = torch.from_numpy(packed).to(self.device)
        self.struct = Mlp()
        self.struct.n_layers = len(self.layers)
        for k, d in enumerate(dims):
            self.struct.dims[k] = d
        self.struct.act = ACT[act]
        self.struct.d_w = self.d_w.data_ptr()

    @property
    def n_inputs(self) -> int:
        return self.dims[0]

    @property
    def max_hidden(self) -> int:
        return max(self.dims[1:-1]) if len(self.dims) > 2 else 0

    @classmethod
    def from_state_dict(cls, sd, act: str = "relu", device="cuda"):
        """Weights stored with the reference's key names (``layer_first``,
        ``layer_hidden.k``, ``layer_last``)."""
        sd = {k: (v.detach().cpu().numpy() if hasattr(v, "detach") else np.asarray(v)) for k, v in sd.items()}
        nh = len([k for k in sd if k.startswith("layer_hidden.") and k.endswith(".weight")])
        names = ["layer_first"] + [f"layer_hidden.{k}" for k in range(nh)] + ["layer_last"]
        return cls([(sd[n + ".weight"], sd[n + ".bias"]) for n in names], act, device)

    @classmethod
    def xavier(cls, D: int, widths, act: str, seed: int, device="cuda"):
        """Xavier-uniform weights, zero biases, from ``seed``."""
        rng = np.random.default_rng(seed)
        dims = [D] + list(widths) + [1]
        layers = []
        for k in range(len(dims) - 1):
            a = math.sqrt(6.0 / (dims[k] + dims[k + 1]))
            layers.append((rng.uniform(-a, a, (dims[k + 1], dims[k])).astype(np.float32),
                           np.zeros(dims[k + 1], np.float32)))
        return cls(layers, act, device)


@dataclass
class Hypers:
    nrad: int = 10
    nang: int = 8
    lmax: int = 4

    @property
    def D(self) -> int:
        return (self.nrad + 1) + (self.nang + 1) * self.lmax


class System:
    """One periodic system of identical rigid bodies, resident on one GPU."""

    def __init__(self, state: State, shape: Shape | str, hypers: Hypers, net: EnergyNet, kT: float, dt: float,
                 device="cuda", nve: bool = False, initial_ke_quirk: bool = False, nlist_every: int = 100,
                 skin: float = 2.0, dx: float = 1e-5, dteta: float = 1e-5, tau: float | None = None,
                 moi=None, nlist_policy: str = "every"):
        if isinstance(shape, str):
            shape = get_shape(shape)
        if net.n_inputs != hypers.D:
            raise ValueError(f"net takes {net.n_inputs} inputs, descriptor has {hypers.D}")
        self.device = torch.device(device)
        self.shape, self.hypers, self.net = shape, hypers, net
        self.N = state.N
        self.L = float(np.float32(state.L))
        f32 = dict(dtype=torch.float32, device=self.device)
        self.pos = torch.tensor(np.asarray(state.pos, np.float32), **f32).contiguous()
        self.quat = torch.tensor(np.asarray(state.orient, np.float32), **f32).contiguous()
        self.vel = torch.tensor(np.asarray(state.vel, np.float32), **f32).contiguous()
        self.angmom = torch.tensor(np.asarray(state.angmom, np.float32), **f32).contiguous()
        self.mass = torch.tensor(np.asarray(state.mass, np.float32), **f32).contiguous()
        self.accel = torch.zeros(self.N, 3, **f32)
        self.dp = torch.zeros(self.N, 4, **f32)
        self.F = torch.zeros(self.N, 3, **f32)
        self.T = torch.zeros(self.N, 3, **f32)
        self.pts = torch.tensor(shape.pts, **f32).contiguous()
        moi = np.asarray(state.moi if moi is None else moi, np.float32).reshape(-1)[:3]
        self.kT, self.dt = float(kT), float(dt)
        self.nve = bool(nve)
        self.nlist_every = int(nlist_every)
        self.r_verlet = float(shape.cutoff) + float(skin)  # Sim.py:86
        if nlist_policy not in ("every", "displacement"):
            raise ValueError(f"unknown Verlet-list policy {nlist_policy!r}")
        self.nlist_policy = nlist_policy
        self.max_disp = 0.5 * float(skin)
        if nlist_policy == "displacement":
            self.nl_ref = torch.zeros(self.N, 3, **f32)
            self.nl_gate = torch.zeros(3, dtype=torch.int32, device=self.device)

        self.nep = Nep()
        self.nep.nrad, self.nep.nang, self.nep.lmax = hypers.nrad, hypers.nang, hypers.lmax
        self.nep.npts = shape.npts
        self.nep.d_pts = self.pts.data_ptr()
        self.nep.cutoff = float(shape.cutoff)
        self.nep.nep_cutoff = float(shape.nep_cutoff)
        self.nep.en_min, self.nep.en_max = float(shape.en_min), float(shape.en_max)
        self.nep.dx, self.nep.dteta = float(dx), float(dteta)

        self.nvt = Nvt()
        self.nvt.dt = self.dt
        self.nvt.tau = float(np.float32(100.0 * dt) if tau is None else tau)
        self.nvt.kT = self.kT
        self.nvt.n_dof = float((self.N - 1) * 3)
        self.nvt.rn_dof = float(self.N * 3)
        for k in range(3):
            self.nvt.moi[k] = float(moi[k])
        self.nvt.box = self.L
        self.nvt.nve = int(self.nve)

        th = Thermostat()
        if self.nve:
            th.thermo_fac = 1.0
        else:
            th.xi, th.eta, th.xi_rot, th.eta_rot, th.thermo_fac = THERMOSTAT_SEED
        self.th = torch.frombuffer(bytearray(bytes(th)), dtype=torch.uint8).to(self.device)
        self.nvt_ws = torch.empty(size_query("amlp_nvt_workspace_bytes", self.N), dtype=torch.uint8,
                                  device=self.device)
        self.nl_ws = torch.empty(size_query("amlp_nlist_workspace_bytes", self.N, self.L, self.r_verlet),
                                 dtype=torch.uint8, device=self.device)
        self.nv = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.nf = torch.zeros(1, dtype=torch.int64, device=self.device)
        self.cap = 0
        self.vpairs = None
        self.fpairs = None
        self.f_ws = None
        self._split_g = self._split_e = None
        self.timestep = 0
        self._graphs = {}
        self.build_nlist()
        call("amlp_nvt_init", self.vel.data_ptr(), self.quat.data_ptr(), self.angmom.data_ptr(),
             self.mass.data_ptr(), self.N, ctypes.byref(self.nvt), int(initial_ke_quirk), self.th.data_ptr(),
             self.nvt_ws.data_ptr(), self.nvt_ws.numel(), _stream())

    # ------------------------------------------------------------------ pairs
    def _alloc_pairs(self, cap: int) -> None:
        self.cap = int(cap)
        self.vpairs = torch.empty(self.cap, 2, dtype=torch.int32, device=self.device)
        self.fpairs = torch.empty(self.cap, 2, dtype=torch.int32, device=self.device)
        self.f_ws = torch.empty(max(1, size_query("amlp_filter_workspace_bytes", self.cap)), dtype=torch.uint8,
                                device=self.device)
        self.adj_ws = None
        self._split_g = self._split_e = None  # g_all and e_all of the split path (grown on demand)
        if self.net.max_hidden > 64 or self.hypers.D > 48:  # beyond the fused adjoint kernel: the wide path
            self.adj_ws = torch.empty(size_query("amlp_adjoint_workspace_bytes", self.cap), dtype=torch.uint8,
                                      device=self.device)
        self._graphs.clear()

    def build_nlist(self, check: bool = True) -> int:
        """Rebuild the Verlet list (``Sim.refreshNList``); grows the buffers if
        needed. Returns the number of pairs (one device-to-host read)."""
        if self.vpairs is None:
            self._alloc_pairs(1024)
        while True:
            call("amlp_nlist_build", self.pos.data_ptr(), self.N, self.L, self.r_verlet, self.vpairs.data_ptr(),
                 self.cap, self.nv.data_ptr(), self.nl_ws.data_ptr(), self.nl_ws.numel(), _stream())
            if not check:
                return -1
            n = int(self.nv.item())
            _lib.check_device()  # the count read has synchronised: the check costs one small copy
            if n <= self.cap:
                if self.nlist_policy == "displacement":
                    self.nl_ref.copy_(self.pos)
                return n
            self._alloc_pairs(int(n * 1.25) + 1024)

    def verlet_pairs(self) -> np.ndarray:
        n = int(self.nv.item())
        return self.vpairs[:n].cpu().numpy()

    def filter_pairs(self) -> None:
        call("amlp_pair_filter", self.pos.data_ptr(), self.L, float(self.shape.cutoff), self.vpairs.data_ptr(),
             self.nv.data_ptr(), self.cap, self.fpairs.data_ptr(), self.nf.data_ptr(), self.f_ws.data_ptr(),
             self.f_ws.numel(), _stream())

    def filtered_pairs(self) -> np.ndarray:
        n = int(self.nf.item())
        return self.fpairs[:n].cpu().numpy()

    # ------------------------------------------------------------------ forces
    def _pe_ptr(self) -> int:
        return self.th.data_ptr() + Thermostat.pe.offset

    def compute_forces(self, method: str = "fd") -> None:
        """Zero F, T and the pair-energy sum, filter the pairs, run the force pass."""
        self.F.zero_()
        self.T.zero_()
        self.th[Thermostat.pe.offset:Thermostat.pe.offset + 8].zero_()
        self.filter_pairs()
        args = (self.pos.data_ptr(), self.quat.data_ptr(), self.L, self.fpairs.data_ptr(), self.nf.data_ptr(),
                self.cap, ctypes.byref(self.nep), ctypes.byref(self.net.struct), self.F.data_ptr(),
                self.T.data_ptr(), self._pe_ptr(), _stream())
        if method == "fd":
            call("amlp_forces_fd", *args)
        elif method == "adjoint":
            if self.adj_ws is None:
                call("amlp_forces_adjoint", *args)
            else:
                call("amlp_forces_adjoint_wide", *args[:-1], self.adj_ws.data_ptr(), self.adj_ws.numel(), args[-1])
        elif method == "fd_split":
            self._forces_split()
        else:
            raise ValueError(f"unknown force method {method!r}")

    def _forces_split(self) -> None:
        P = int(self.nf.item())  # the reference's data-dependent pair count (cp.where sync)
        D = self.hypers.D
        rows = 10 * max(P, 1)
        if self._split_e is None or self._split_e.numel() < rows:
            # g_all and e_all kept between steps, a quarter above the largest pair count so far:
            # a new block per step (pair counts move a little every step) would go back to
            # cudaMalloc, a synchronous call, whenever the count grows
            keep = rows + rows // 4
            self._split_g = self._split_e = None
            self._split_g = torch.empty(keep * D, dtype=torch.float32, device=self.device)
            self._split_e = torch.empty(keep, dtype=torch.float32, device=self.device)
        g, e = self._split_g, self._split_e
        call("amlp_descriptors", self.pos.data_ptr(), self.quat.data_ptr(), self.L, self.fpairs.data_ptr(), P,
             ctypes.byref(self.nep), g.data_ptr(), _stream())
        call("amlp_mlp_energy", g.data_ptr(), 10 * P, ctypes.byref(self.net.struct), e.data_ptr(), _stream())
        call("amlp_fd_scatter", e.data_ptr(), P, self.fpairs.data_ptr(), ctypes.byref(self.nep), self.F.data_ptr(),
             self.T.data_ptr(), self._pe_ptr(), _stream())

    # ------------------------------------------------------------------ integration
    def integrate_step_two(self) -> None:
        call("amlp_nvt_step_two", self.vel.data_ptr(), self.accel.data_ptr(), self.F.data_ptr(),
             self.mass.data_ptr(), self.quat.data_ptr(), self.T.data_ptr(), self.angmom.data_ptr(),
             self.dp.data_ptr(), self.N, ctypes.byref(self.nvt), self.th.data_ptr(), _stream())

    def integrate_step_one(self) -> None:
        call("amlp_nvt_step_one", self.pos.data_ptr(), self.vel.data_ptr(), self.accel.data_ptr(),
             self.quat.data_ptr(), self.angmom.data_ptr(), self.dp.data_ptr(), self.mass.data_ptr(), self.N,
             ctypes.byref(self.nvt), self.th.data_ptr(), self.nvt_ws.data_ptr(), self.nvt_ws.numel(), _stream())

    def _gated_rebuild(self) -> None:
        call("amlp_nlist_check_displacement", self.pos.data_ptr(), self.nl_ref.data_ptr(), self.N, self.L,
             self.max_disp, self.nl_gate.data_ptr(), _stream())
        call("amlp_nlist_build_gated", self.pos.data_ptr(), self.N, self.L, self.r_verlet, self.vpairs.data_ptr(),
             self.cap, self.nv.data_ptr(), self.nl_ws.data_ptr(), self.nl_ws.numel(), self.nl_gate.data_ptr(),
             self.nl_ref.data_ptr(), _stream())

    @property
    def rebuilds(self) -> int:
        """Gated rebuilds so far (displacement policy)."""
        return int(self.nl_gate[1].item()) if self.nlist_policy == "displacement" else -1

    def _step_kernels(self, method: str) -> None:
        if self.nlist_policy == "displacement":
            self._gated_rebuild()
        self.compute_forces(method)
        self.integrate_step_two()
        self.integrate_step_one()

    def step(self, method: str = "fd") -> None:
        """One time step, host-driven (``Sim.step``)."""
        if self.nlist_policy == "displacement":
            self._run_checked(1, method, graph=False)
            return
        if self.timestep % self.nlist_every == 0 and self.timestep > 0:
            self.build_nlist()
        self._step_kernels(method)
        self.timestep += 1

    def _run_checked(self, seg: int, method: str, graph: bool) -> None:
        """``seg`` steps under the displacement policy; rerun from a snapshot
        with a larger list if a rebuild inside them overflowed."""
        snap = self.snapshot_tensors()
        while True:
            if graph and method != "fd_split":
                self._graph(method, seg).replay()
            else:
                for _ in range(seg):
                    self._step_kernels(method)
            if not int(self.nl_gate[2].item()):
                break
            self.restore_tensors(snap)
            self.nl_gate[2] = 0
            self._alloc_pairs(int(self.cap * 1.5) + 1024)
            self.build_nlist()
        self.timestep += seg

    def run(self, nsteps: int, method: str = "fd", graph: bool = True) -> None:
        """``nsteps`` steps; between Verlet rebuilds the steps replay as one CUDA graph.
        Raises ``AmlpDeviceError`` (after the steps) if a bounded device wait gave up."""
        self._run(nsteps, method, graph)
        _lib.check_device()

    def _run(self, nsteps: int, method: str, graph: bool) -> None:
        end = self.timestep + nsteps
        if self.nlist_policy == "displacement":
            while self.timestep < end:
                self._run_checked(min(end - self.timestep, self.nlist_every), method, graph)
            return
        while self.timestep < end:
            if self.timestep % self.nlist_every == 0 and self.timestep > 0:
                self.build_nlist()
            seg = min(end - self.timestep, self.nlist_every - self.timestep % self.nlist_every)
            if not graph or method == "fd_split":
                for _ in range(seg):
                    self._step_kernels(method)
                    self.timestep += 1
                continue
            self._graph(method, seg).replay()
            self.timestep += seg

    def _graph(self, method: str, seg: int) -> torch.cuda.CUDAGraph:
        key = (method, seg, self.cap)
        g = self._graphs.get(key)
        if g is None:
            # warm-up outside capture (sets kernel attributes), on a snapshot of the state
            snap = self.snapshot_tensors()
            self._step_kernels(method)
            torch.cuda.synchronize()
            self.restore_tensors(snap)
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                snap = self.snapshot_tensors()
                with torch.cuda.graph(g, stream=s):
                    for _ in range(seg):
                        self._step_kernels(method)
                self.restore_tensors(snap)
            torch.cuda.current_stream().wait_stream(s)
            self._graphs[key] = g
        return g

    def snapshot_tensors(self):
        return [t.clone() for t in (self.pos, self.quat, self.vel, self.angmom, self.accel, self.dp, self.th)]

    def restore_tensors(self, snap) -> None:
        for t, s in zip((self.pos, self.quat, self.vel, self.angmom, self.accel, self.dp, self.th), snap):
            t.copy_(s)

    # ------------------------------------------------------------------ host views
    def set_thermostat(self, integrator_vars, thermo_fac) -> None:
        """Set xi, eta, xi_rot, eta_rot and the translational factor (resume)."""
        raw = bytes(self.th.cpu().numpy().tobytes())
        th = Thermostat.from_buffer_copy(raw)
        th.xi, th.eta, th.xi_rot, th.eta_rot = (float(v) for v in integrator_vars)
        th.thermo_fac = float(thermo_fac)
        self.th.copy_(torch.frombuffer(bytearray(bytes(th)), dtype=torch.uint8))

    def thermostat(self) -> dict:
        raw = bytes(self.th.cpu().numpy().tobytes())
        th = Thermostat.from_buffer_copy(raw)
        return dict(xi=th.xi, eta=th.eta, xi_rot=th.xi_rot, eta_rot=th.eta_rot, thermo_fac=th.thermo_fac,
                    ke_t=th.ke_t, ke_r=th.ke_r, pe=th.pe)

    def state(self) -> State:
        return State(pos=self.pos.cpu().numpy(), orient=self.quat.cpu().numpy(), vel=self.vel.cpu().numpy(),
                     angmom=self.angmom.cpu().numpy(), mass=self.mass.cpu().numpy(),
                     moi=np.array(list(self.nvt.moi), np.float32), L=self.L)

    def conserved_quantity(self) -> float:
        """KE_t + KE_r + PE + MTK thermostat energy, FP64 (HOOMD's NVT-MTK form:
        dof kT (xi^2 tau^2 / 2 + eta) for translation and rotation)."""
        t = self.thermostat()
        e = t["ke_t"] + t["ke_r"] + t["pe"]
        if not self.nve:
            tau = float(self.nvt.tau)
            e += self.nvt.n_dof * self.kT * (t["xi"] ** 2 * tau * tau / 2 + t["eta"])
            e += self.nvt.rn_dof * self.kT * (t["xi_rot"] ** 2 * tau * tau / 2 + t["eta_rot"])
        return e
