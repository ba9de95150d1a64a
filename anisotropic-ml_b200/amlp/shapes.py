"""Shape tables: body-frame interaction points and per-shape constants.

Reference shapes come from ``DescriptorGenerator.setShape``
(``nep_simulator/DescriptorGenerator.py:58-125``): ``cube_v2`` (6 points),
``th_v1`` (4 points), ``pbp_v3`` (7 points).

The reference has no table for the large-scale shapes; they are defined here
and fixed:

* ``cube26``  -- cube of edge 1: 8 vertices, 12 edge midpoints, 6 face centres;
* ``tetra16`` -- regular tetrahedron of edge 1 centred on its centroid: 4
  vertices, 6 edge midpoints, and for every edge (a, b), a < b, the point one
  third of the way from vertex a to vertex b;
* ``cyl24``   -- twisted cylinder of length 2 and radius 0.4 along z: 3 rings of
  8 points at z = -1, 0, 1, each ring turned 45 degrees further (90 degrees of
  twist end to end).

All three use pair cutoff 2.5 (Verlet radius 4.5), NEP cutoff 2.5 and the
energy range of ``cube_v2`` (-5.1, 15.0). ``moi`` and ``volume`` are those of
the solid body with unit mass.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Shape:
    name: str
    pts: np.ndarray          # (npts, 3) float32, body frame
    en_min: float
    en_max: float
    cutoff: float            # pair filter cutoff on centre distance
    nep_cutoff: float        # descriptor cutoff radius r_c
    moi: tuple               # (Ix, Iy, Iz) of the solid body, unit mass
    volume: float            # solid-body volume (packing fraction -> box)

    @property
    def npts(self) -> int:
        return int(self.pts.shape[0])

    @property
    def nd(self) -> int:
        return 2 * self.npts


def _cube26():
    h = 0.5
    return np.array([(x, y, z) for x in (-h, 0.0, h) for y in (-h, 0.0, h) for z in (-h, 0.0, h)
                     if (x, y, z) != (0.0, 0.0, 0.0)], np.float32)


def _tetra16():
    s = 1.0 / (2.0 * math.sqrt(2.0))
    v = np.array([[s, s, s], [s, -s, -s], [-s, s, -s], [-s, -s, s]], np.float64)
    edges = [(a, b) for a in range(4) for b in range(a + 1, 4)]
    pts = list(v) + [(v[a] + v[b]) / 2 for a, b in edges] + [v[a] + (v[b] - v[a]) / 3 for a, b in edges]
    return np.array(pts, np.float32)


def _cyl24():
    pts = []
    for k, z in enumerate((-1.0, 0.0, 1.0)):
        for j in range(8):
            phi = 2 * math.pi * j / 8 + math.radians(45.0 * k)
            pts.append((0.4 * math.cos(phi), 0.4 * math.sin(phi), z))
    return np.array(pts, np.float32)


_R = 0.4
_TETRA_VOL = 1.0 / (6.0 * math.sqrt(2.0))

SHAPES = {
    "cube_v2": Shape("cube_v2", np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]],
                                         np.float32) * np.float32(1.7),
                     -5.1, 15.0, 5.80, 4.5, (1.0, 1.0, 1.0), 1.0),
    "th_v1": Shape("th_v1", np.array([[-0.45, -0.45, -0.45], [-0.45, 0.45, 0.45], [0.45, -0.45, 0.45],
                                      [0.45, 0.45, -0.45]], np.float32),
                   -6.7, 15.0, 5.75, 4.5, (1.0, 1.0, 1.0), _TETRA_VOL),
    "pbp_v3": Shape("pbp_v3", np.array([[-1.46946, 2.02254, 0.0], [-2.37764, -0.77254, 0.0], [-0.0, -2.5, 0.0],
                                        [2.37764, -0.77254, 0.0], [1.46946, 2.02254, 0.0], [0.0, 0.0, 3.5],
                                        [0.0, 0.0, -3.5]], np.float32),
                    -2.5, 15.0, 8.1, 7.5, (1.0, 1.0, 1.0), 1.0),
    "cube26": Shape("cube26", _cube26(), -5.1, 15.0, 2.5, 2.5, (1 / 6, 1 / 6, 1 / 6), 1.0),
    "tetra16": Shape("tetra16", _tetra16(), -5.1, 15.0, 2.5, 2.5, (0.05, 0.05, 0.05), _TETRA_VOL),
    "cyl24": Shape("cyl24", _cyl24(), -5.1, 15.0, 2.5, 2.5,
                   ((3 * _R * _R + 4.0) / 12.0, (3 * _R * _R + 4.0) / 12.0, 0.5 * _R * _R),
                   math.pi * _R * _R * 2.0),
}


def get_shape(name: str) -> Shape:
    """Shape by name; unknown names raise ``KeyError`` (the reference prints and
    calls ``exit()``, ``DescriptorGenerator.py:121-123``)."""
    try:
        return SHAPES[name]
    except KeyError:
        raise KeyError(f"shape {name!r} not found; known shapes: {sorted(SHAPES)}") from None
