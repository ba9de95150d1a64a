"""Seeded synthetic initial states.

* centres: jittered simple-cubic lattice, n = ceil(N^(1/3)) sites per side,
  spacing L/n, uniform jitter +-0.1 per coordinate, the first N sites;
* box: L = (N * V_body / phi)^(1/3) for packing fraction phi;
* orientations: uniform random unit quaternions (Shoemake), (w, x, y, z);
* velocities: Maxwell-Boltzmann, v ~ N(0, kT/m);
* angular momenta: HOOMD quaternion convention p = 2 q (x) (0, L_body) with
  L_body,k ~ N(0, I_k kT), so that s = 1/2 conj(q) (x) p has vector part L_body
  (the rotational kinetic energy of ``Sim.getRotKin``, ``Sim.py:171-180``).

All draws come from ``numpy.random.default_rng(seed)`` in a fixed order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .shapes import Shape, get_shape


@dataclass
class State:
    pos: np.ndarray       # (N,3) float32 in [-L/2, L/2)
    orient: np.ndarray    # (N,4) float32, unit, w first
    vel: np.ndarray       # (N,3) float32
    angmom: np.ndarray    # (N,4) float32
    mass: np.ndarray      # (N,)  float32
    moi: np.ndarray       # (3,)  float32
    L: float              # cubic box edge (float32 value)

    @property
    def N(self) -> int:
        return int(self.pos.shape[0])


def quat_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Hamilton product of (w, x, y, z) quaternions, batched."""
    w = a[..., 0] * b[..., 0] - np.sum(a[..., 1:] * b[..., 1:], axis=-1)
    v = a[..., :1] * b[..., 1:] + b[..., :1] * a[..., 1:] + np.cross(a[..., 1:], b[..., 1:])
    return np.concatenate([w[..., None], v], axis=-1)


def random_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform unit quaternions (Shoemake's subgroup algorithm), w first."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    a, b = np.sqrt(1 - u1), np.sqrt(u1)
    q = np.stack([b * np.cos(2 * np.pi * u3), a * np.sin(2 * np.pi * u2),
                  a * np.cos(2 * np.pi * u2), b * np.sin(2 * np.pi * u3)], axis=1)
    return q.astype(np.float32)


def box_for(n: int, shape: Shape, phi: float) -> float:
    return float(np.float32((n * shape.volume / phi) ** (1.0 / 3.0)))


def jittered_lattice(rng: np.random.Generator, n: int, L: float, jitter: float = 0.1) -> np.ndarray:
    m = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
    while m ** 3 < n:
        m += 1
    a = L / m
    g = np.arange(m, dtype=np.float64)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)[:n]
    pos = (sites + 0.5) * a - 0.5 * L + rng.uniform(-jitter, jitter, size=(n, 3))
    pos = pos.astype(np.float32)
    Lf = np.float32(L)
    pos = np.where(pos >= 0.5 * Lf, pos - Lf, pos)
    pos = np.where(pos < -0.5 * Lf, pos + Lf, pos)
    return pos.astype(np.float32)


def make_state(n: int, shape: Shape | str, phi: float, kT: float = 1.0, seed: int = 0,
               L: float | None = None) -> State:
    """Seeded initial state of ``n`` rigid bodies of ``shape`` at packing fraction ``phi``."""
    if isinstance(shape, str):
        shape = get_shape(shape)
    rng = np.random.default_rng(seed)
    L = box_for(n, shape, phi) if L is None else float(np.float32(L))
    pos = jittered_lattice(rng, n, L)
    orient = random_quaternions(rng, n)
    mass = np.ones(n, np.float32)
    vel = (rng.standard_normal((n, 3)) * math.sqrt(kT)).astype(np.float32)
    moi = np.asarray(shape.moi, np.float64)
    Lb = rng.standard_normal((n, 3)) * np.sqrt(moi * kT)
    p = 2.0 * quat_mul(orient.astype(np.float64), np.concatenate([np.zeros((n, 1)), Lb], axis=1))
    return State(pos=pos, orient=orient, vel=vel, angmom=p.astype(np.float32), mass=mass,
                 moi=moi.astype(np.float32), L=L)
