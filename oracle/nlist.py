"""Neighbour list of the reference, by the reference's own call (test infrastructure only).

``Sim.setNeighborList`` / ``Sim.refreshNList`` (``nep_simulator/Sim.py:85-92``,
``:192-198``) build the Verlet list with
``cKDTree(pos + Lx/2, leafsize=12, boxsize=Lx + 0.0001).query_pairs(r=cutoff + 2.0,
output_type='ndarray')``. scipy's order of pairs is its tree traversal order;
``sorted_pairs`` returns them sorted by (i, j), the canonical order used to
compare lists.
"""
from __future__ import annotations

import numpy as np
from scipy.spatial import cKDTree


def reference_pairs(pos, L, r):
    """The reference's call; ``pos`` float32 in [-L/2, L/2], ``L`` float32."""
    pos = np.asarray(pos, np.float32)
    L = np.float32(L)
    tree = cKDTree(data=pos + L * np.float32(0.5), leafsize=12, boxsize=L + 0.0001)
    return tree.query_pairs(r=r, output_type="ndarray")


def sorted_pairs(p):
    p = np.asarray(p, np.int64).reshape(-1, 2)
    return p[np.lexsort((p[:, 1], p[:, 0]))]


def brute_force_pairs(pos, L, r):
    """Same criterion written out: FP64 periodic distance of float32(pos + L/2),
    box float32(L + 1e-4), folded once per axis, squared distance summed x, y, z
    and compared inclusively with r*r."""
    x = (np.asarray(pos, np.float32) + np.float32(L) * np.float32(0.5)).astype(np.float64)
    fb = float(np.float32(L) + 0.0001)
    hb = 0.5 * fb
    n = len(x)
    out = []
    for i in range(n - 1):
        d = x[i] - x[i + 1:]
        d = np.where(d < -hb, fb + d, np.where(d > hb, d - fb, d))
        s = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
        js = np.nonzero(s <= r * r)[0] + i + 1
        out.extend((i, j) for j in js)
    return np.asarray(out, np.int64).reshape(-1, 2)
