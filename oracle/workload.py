"""Seeded benchmark workloads and the timed CPU run of the reference's step.

TEST INFRASTRUCTURE ONLY: used by the reference arm and the ``cpu_baseline``
leg of ``bench.py``. Those legs must not import the product package, so the
benchmark's initial state and Xavier net are generated here as well;
``tests/test_cpu_host.py`` checks that ``make_state`` and ``xavier_layers``
give the product's arrays bit for bit (``amlp.configs.make_state``,
``amlp.engine.EnergyNet.xavier``).

``CpuStep`` runs one step of the reference's algorithm on the host cores: the
force pass of ``Sim.step`` (``nep_simulator/Sim.py:261-266``: ten
finite-difference clouds, FP32 descriptors, torch-CPU net, differences, clip,
scatter) through ``oracle.nep`` on a process pool (one worker per host core,
each on a contiguous chunk of the pairs), then both NVT halves on every body
(``NVT.py:12-64``). The oracle's FP32 path is bit-identical to the reference's
own classes on the golden cases.
"""
from __future__ import annotations

import math
import multiprocessing as mp
import os
import time
from dataclasses import dataclass

import numpy as np

from . import nep, nlist
from .shapes import SHAPES

# solid-body volume and principal moments (unit mass) of the shapes without a reference table
_R = 0.4
SOLID = {
    "cube26": (1.0, (1 / 6, 1 / 6, 1 / 6)),
    "tetra16": (1.0 / (6.0 * math.sqrt(2.0)), (0.05, 0.05, 0.05)),
    "cyl24": (math.pi * _R * _R * 2.0, ((3 * _R * _R + 4.0) / 12.0, (3 * _R * _R + 4.0) / 12.0, 0.5 * _R * _R)),
}


@dataclass
class State:
    pos: np.ndarray
    orient: np.ndarray
    vel: np.ndarray
    angmom: np.ndarray
    mass: np.ndarray
    moi: np.ndarray
    L: float

    @property
    def N(self) -> int:
        return int(self.pos.shape[0])


def _quat_mul(a, b):
    w = a[..., 0] * b[..., 0] - np.sum(a[..., 1:] * b[..., 1:], axis=-1)
    v = a[..., :1] * b[..., 1:] + b[..., :1] * a[..., 1:] + np.cross(a[..., 1:], b[..., 1:])
    return np.concatenate([w[..., None], v], axis=-1)


def make_state(n: int, shape: str, phi: float, kT: float = 1.0, seed: int = 0) -> State:
    """Jittered simple-cubic lattice (n = ceil(N^(1/3)) sites per side, jitter
    +-0.1), Shoemake unit quaternions, Maxwell-Boltzmann velocities and angular
    momenta p = 2 q (x) (0, L_body), L_body ~ N(0, I kT), box (N V / phi)^(1/3);
    every draw from ``default_rng(seed)`` in that order."""
    vol, moi = SOLID[shape]
    rng = np.random.default_rng(seed)
    L = float(np.float32((n * vol / phi) ** (1.0 / 3.0)))
    m = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
    while m ** 3 < n:
        m += 1
    a = L / m
    g = np.arange(m, dtype=np.float64)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)[:n]
    pos = ((sites + 0.5) * a - 0.5 * L + rng.uniform(-0.1, 0.1, size=(n, 3))).astype(np.float32)
    Lf = np.float32(L)
    pos = np.where(pos >= 0.5 * Lf, pos - Lf, pos)
    pos = np.where(pos < -0.5 * Lf, pos + Lf, pos).astype(np.float32)
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    s1, s2 = np.sqrt(1 - u1), np.sqrt(u1)
    orient = np.stack([s2 * np.cos(2 * np.pi * u3), s1 * np.sin(2 * np.pi * u2), s1 * np.cos(2 * np.pi * u2),
                       s2 * np.sin(2 * np.pi * u3)], axis=1).astype(np.float32)
    vel = (rng.standard_normal((n, 3)) * math.sqrt(kT)).astype(np.float32)
    moi = np.asarray(moi, np.float64)
    Lb = rng.standard_normal((n, 3)) * np.sqrt(moi * kT)
    p = 2.0 * _quat_mul(orient.astype(np.float64), np.concatenate([np.zeros((n, 1)), Lb], axis=1))
    return State(pos=pos, orient=orient, vel=vel, angmom=p.astype(np.float32), mass=np.ones(n, np.float32),
                 moi=moi.astype(np.float32), L=L)


def xavier_layers(D: int, widths, seed: int):
    """Xavier-uniform weights and zero biases, D -> widths -> 1, from ``seed``."""
    rng = np.random.default_rng(seed)
    dims = [D] + list(widths) + [1]
    out = []
    for k in range(len(dims) - 1):
        a = math.sqrt(6.0 / (dims[k] + dims[k + 1]))
        out.append((rng.uniform(-a, a, (dims[k + 1], dims[k])).astype(np.float32),
                    np.zeros(dims[k + 1], np.float32)))
    return out


# ----------------------------------------------------------------------------- pool workers
_W = {}


def _init_worker(shape_name, hypers, layers, act):
    import torch
    torch.set_num_threads(1)
    _W.update(shape=SHAPES[shape_name], hypers=hypers, layers=layers, act=act)


def _chunk_forces(args):
    """Per-pair F, T_i, T_j of a chunk of filtered pairs; the chunk carries only
    the bodies it touches (pairs re-indexed into them)."""
    pos, orient, pairs, L = args
    o = nep.pair_forces(pos, orient, pairs, L, _W["shape"], _W["hypers"], _W["layers"], _W["act"])
    return o["F_pair"], o["T_i"], o["T_j"], o["e_all"][:o["P"]]


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class CpuStep:
    """One NVT step of the reference's algorithm on the host cores (see the
    module docstring). ``step(bodies)`` runs, for the given bodies (None: all),
    the pair filter of the Verlet pairs (i, j) they own (i is the body, j > i)
    and the force pass of the filtered ones; then both NVT halves on all
    bodies. It returns the step's wall time. Every body owns P / N filtered pairs
    on average, so a random sample of bodies is an unbiased share of the force
    work; the NVT halves on all bodies are more than that share."""

    def __init__(self, state: State, shape_name: str, hypers, layers, act: str, kT: float, dt: float,
                 workers: int | None = None):
        self.state, self.shape = state, SHAPES[shape_name]
        self.workers = max(1, min(workers or host_cores(), 64))
        t0 = time.perf_counter()
        vl = nlist.reference_pairs(state.pos, state.L, self.shape["cutoff"] + 2.0)
        self.t_nlist = time.perf_counter() - t0
        self.vl = nlist.sorted_pairs(vl)
        self.start = np.searchsorted(self.vl[:, 0], np.arange(state.N + 1))
        self.st = nep.NVTState(state.pos, state.vel, state.orient, state.angmom, state.mass, state.moi, state.L,
                               kT, dt)
        self.pairs_last = 0
        self.pool = mp.get_context("spawn").Pool(self.workers, initializer=_init_worker,
                                                 initargs=(shape_name, tuple(hypers), layers, act))
        self.pool.map(_chunk_forces, [])  # workers up before any timing

    def close(self):
        self.pool.terminate()
        self.pool.join()

    def _tasks(self, pairs):
        out = []
        for chunk in np.array_split(pairs, self.workers):
            if len(chunk) == 0:
                continue
            bodies, inv = np.unique(chunk.reshape(-1), return_inverse=True)
            out.append((self.st.pos[bodies], self.st.orient[bodies], inv.reshape(-1, 2).astype(np.int64),
                        self.state.L))
        return out

    def step(self, bodies=None) -> float:
        t0 = time.perf_counter()
        if bodies is None:
            vsub = self.vl
        else:
            vsub = np.concatenate([self.vl[self.start[i]:self.start[i + 1]] for i in bodies] or
                                  [np.zeros((0, 2), np.int64)])
        _, pairs, _ = nep.min_image_filter(self.st.pos, vsub, self.state.L, self.shape["cutoff"])
        res = self.pool.map(_chunk_forces, self._tasks(pairs))
        N = self.state.N
        if res:
            Fp, Ti, Tj = (np.concatenate([r[k] for r in res]) for k in range(3))
            F, T = nep.scatter(pairs, Fp, Ti, Tj, N)
        else:
            F, T = np.zeros((N, 3), np.float32), np.zeros((N, 3), np.float32)
        self.st.step_two(F, T)
        self.st.step_one()
        self.pairs_last = len(pairs)
        return time.perf_counter() - t0
