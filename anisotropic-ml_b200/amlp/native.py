"""Python handles over the library's own runtimes (``amlp_sim``, ``amlp_pool``).

``NativeSystem`` drives one system through the C ABI's simulation handle: the
handle owns the device state and buffers, sequences the time step of
``Sim.step`` (``Sim.py:257-285``) in C++, rebuilds the Verlet list every
``nlist_every`` steps and replays the steps in between as one CUDA graph.
``System`` in ``engine.py`` does the same with the buffers in torch tensors;
the two run the same kernels in the same order.

``NativePool`` is the serving pool of the C ABI. Systems of one shape and one
net are admitted and evicted between segments and advanced together by
multi-system launches.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import FORCES, AmlpError, Mlp, PoolConfig, PoolSystem, SimConfig, Thermostat
from .configs import State
from .engine import EnergyNet, Hypers
from .shapes import Shape, get_shape


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _f32(a, shape) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, np.float32).reshape(shape))


class NativeSystem:
    """One periodic system of identical rigid bodies in an ``amlp_sim`` handle
    (same arguments as ``engine.System``)."""

    def __init__(self, state: State, shape: Shape | str, hypers: Hypers, net: EnergyNet, kT: float, dt: float,
                 device="cuda", nve: bool = False, initial_ke_quirk: bool = False, nlist_every: int = 100,
                 skin: float = 2.0, dx: float = 1e-5, dteta: float = 1e-5, tau: float | None = None, moi=None):
        if isinstance(shape, str):
            shape = get_shape(shape)
        self.device = torch.device(device)
        self.N = state.N
        self.L = float(np.float32(state.L))
        self.shape, self.net = shape, net
        cfg = SimConfig()
        cfg.n, cfg.nrad, cfg.nang, cfg.lmax = self.N, hypers.nrad, hypers.nang, hypers.lmax
        cfg.kT, cfg.dt, cfg.tau = float(kT), float(dt), float(tau) if tau is not None else 0.0
        cfg.nve, cfg.initial_ke_quirk, cfg.nlist_every = int(nve), int(initial_ke_quirk), int(nlist_every)
        cfg.skin, cfg.dx, cfg.dteta = float(skin), float(dx), float(dteta)
        h = ctypes.c_void_p()
        self._h = None
        self._call("amlp_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        pts = _f32(shape.pts, (-1, 3))
        self._call("amlp_set_shape", self._h, pts.ctypes.data, shape.npts, float(shape.en_min), float(shape.en_max),
                   float(shape.cutoff), float(shape.nep_cutoff))
        self._call("amlp_set_model", self._h, ctypes.byref(net.struct), _stream())
        f32 = dict(dtype=torch.float32, device=self.device)
        t = {k: torch.tensor(_f32(getattr(state, k), shp), **f32)
             for k, shp in (("pos", (-1, 3)), ("orient", (-1, 4)), ("vel", (-1, 3)), ("angmom", (-1, 4)),
                            ("mass", (-1,)))}
        moi = _f32(state.moi if moi is None else moi, (-1,))[:3].copy()
        self._call("amlp_set_state", self._h, t["pos"].data_ptr(), t["orient"].data_ptr(), t["vel"].data_ptr(),
                   t["angmom"].data_ptr(), t["mass"].data_ptr(), moi.ctypes.data, self.L, _stream())
        torch.cuda.current_stream().synchronize()

    def _call(self, name: str, *args) -> None:
        st = getattr(_lib.lib, name)(*args)
        if st != _lib.AMLP_OK:
            detail = _lib.lib.amlp_last_error(self._h).decode() if self._h else ""
            raise AmlpError(name, st, detail)

    def close(self) -> None:
        if self._h:
            torch.cuda.synchronize()
            _lib.lib.amlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def timestep(self) -> int:
        return int(_lib.lib.amlp_timestep(self._h))

    def build_nlist(self) -> None:
        self._call("amlp_build_nlist", self._h, _stream())

    def run(self, nsteps: int, method: str = "fd") -> None:
        self._call("amlp_step", self._h, int(nsteps), FORCES[method], _stream())

    def forces(self, method: str = "fd"):
        """(F, T) of the current state, one force pass."""
        F = torch.empty(self.N, 3, dtype=torch.float32, device=self.device)
        T = torch.empty_like(F)
        self._call("amlp_forces", self._h, F.data_ptr(), T.data_ptr(), FORCES[method], _stream())
        return F, T

    def descriptors(self, cap: int):
        """(g_all (10 P, D), filtered pairs (P, 2) int32, P) of the current state."""
        D = self.net.n_inputs
        g = torch.empty(10 * max(cap, 1), D, dtype=torch.float32, device=self.device)
        pairs = torch.empty(max(cap, 1), 2, dtype=torch.int32, device=self.device)
        P = ctypes.c_longlong(0)
        self._call("amlp_sim_descriptors", self._h, g.data_ptr(), pairs.data_ptr(), int(cap), ctypes.byref(P),
                   _stream())
        n = int(P.value)
        return g[:10 * n], pairs[:n], n

    def state(self) -> dict:
        f32 = dict(dtype=torch.float32, device=self.device)
        out = {"pos": torch.empty(self.N, 3, **f32), "quat": torch.empty(self.N, 4, **f32),
               "vel": torch.empty(self.N, 3, **f32), "angmom": torch.empty(self.N, 4, **f32)}
        self._call("amlp_get_state", self._h, out["pos"].data_ptr(), out["quat"].data_ptr(), out["vel"].data_ptr(),
                   out["angmom"].data_ptr(), _stream())
        return out

    def thermostat(self) -> dict:
        th = Thermostat()
        self._call("amlp_get_thermostat", self._h, ctypes.byref(th), _stream())
        return dict(xi=th.xi, eta=th.eta, xi_rot=th.xi_rot, eta_rot=th.eta_rot, thermo_fac=th.thermo_fac,
                    ke_t=th.ke_t, ke_r=th.ke_r, pe=th.pe)


class NativePool:
    """``amlp_pool``: systems of one shape and one net advanced together."""

    def __init__(self, shape: Shape | str, hypers: Hypers, net: EnergyNet, dt: float, tau: float | None = None,
                 skin: float = 2.0):
        if isinstance(shape, str):
            shape = get_shape(shape)
        self.shape, self.net = shape, net
        self._pts = _f32(shape.pts, (-1, 3))
        self._moi = _f32(shape.moi, (-1,))[:3].copy()
        cfg = PoolConfig()
        cfg.nrad, cfg.nang, cfg.lmax = hypers.nrad, hypers.nang, hypers.lmax
        cfg.dt, cfg.tau = float(dt), float(tau) if tau is not None else 0.0
        cfg.h_pts, cfg.npts = self._pts.ctypes.data, shape.npts
        cfg.en_min, cfg.en_max = float(shape.en_min), float(shape.en_max)
        cfg.cutoff, cfg.nep_cutoff, cfg.skin = float(shape.cutoff), float(shape.nep_cutoff), float(skin)
        cfg.h_moi = self._moi.ctypes.data
        self._mlp = Mlp.from_buffer_copy(bytes(net.struct))
        cfg.mlp = ctypes.pointer(self._mlp)
        h = ctypes.c_void_p()
        self._h = None
        self._call("amlp_pool_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        self.sizes = {}

    def _call(self, name: str, *args) -> None:
        st = getattr(_lib.lib, name)(*args)
        if st != _lib.AMLP_OK:
            detail = _lib.lib.amlp_pool_last_error(self._h).decode() if self._h else ""
            raise AmlpError(name, st, detail)

    def close(self) -> None:
        if self._h:
            torch.cuda.synchronize()
            _lib.lib.amlp_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return int(_lib.lib.amlp_pool_size(self._h))

    def admit(self, state: State, kT: float, nve: bool = False, verlet_cap: int = 0) -> int:
        arr = [_f32(state.pos, (-1, 3)), _f32(state.orient, (-1, 4)), _f32(state.vel, (-1, 3)),
               _f32(state.angmom, (-1, 4)), _f32(state.mass, (-1,))]
        x = PoolSystem()
        x.n, x.box, x.kT, x.nve, x.verlet_cap = state.N, float(np.float32(state.L)), float(kT), int(nve), verlet_cap
        x.h_pos, x.h_quat, x.h_vel, x.h_angmom, x.h_mass = (a.ctypes.data for a in arr)
        rid = ctypes.c_int(-1)
        self._call("amlp_pool_admit", self._h, ctypes.byref(x), ctypes.byref(rid))
        self.sizes[rid.value] = state.N
        return rid.value

    def evict(self, rid: int) -> dict:
        n = self.sizes.pop(rid)
        out = {"pos": np.empty((n, 3), np.float32), "quat": np.empty((n, 4), np.float32),
               "vel": np.empty((n, 3), np.float32), "angmom": np.empty((n, 4), np.float32)}
        th = Thermostat()
        self._call("amlp_pool_evict", self._h, rid, out["pos"].ctypes.data, out["quat"].ctypes.data,
                   out["vel"].ctypes.data, out["angmom"].ctypes.data, ctypes.byref(th))
        out["thermostat"] = dict(xi=th.xi, eta=th.eta, xi_rot=th.xi_rot, eta_rot=th.eta_rot,
                                 thermo_fac=th.thermo_fac, ke_t=th.ke_t, ke_r=th.ke_r, pe=th.pe)
        return out

    def step_segment(self, nsteps: int) -> None:
        self._call("amlp_pool_step_segment", self._h, int(nsteps), _stream())

    def status(self, rid: int) -> dict:
        st, done, th = ctypes.c_int(-1), ctypes.c_longlong(0), Thermostat()
        self._call("amlp_pool_system_status", self._h, rid, ctypes.byref(st), ctypes.byref(done), ctypes.byref(th))
        return dict(status=st.value, steps_done=done.value, xi=th.xi, eta=th.eta, pe=th.pe, ke_t=th.ke_t)
