"""Oracle copy of the shape tables (test infrastructure only).

Kept independent of the product's table so that a mistake in one shows up as a
mismatch in ``tests/test_shapes.py``.

Reference shapes: ``nep_simulator/DescriptorGenerator.py:63-117``.
New shapes (cube26, tetra16, cyl24) have no reference table; their definition
is fixed here and in the product identically.
"""
import numpy as np


def _ref(points, scale, en_min, en_max, cutoff, nep_cutoff):
    return dict(pts=np.asarray(points, np.float32) * np.float32(scale), en_min=en_min,
                en_max=en_max, cutoff=cutoff, nep_cutoff=nep_cutoff)


def cube26():
    h = 0.5
    pts = []
    for x in (-h, 0.0, h):
        for y in (-h, 0.0, h):
            for z in (-h, 0.0, h):
                if (x, y, z) != (0.0, 0.0, 0.0):
                    pts.append((x, y, z))
    return np.asarray(pts, np.float32)


def tetra16():
    s = 1.0 / (2.0 * np.sqrt(2.0))
    v = np.array([[s, s, s], [s, -s, -s], [-s, s, -s], [-s, -s, s]], np.float64)
    pts = list(v)
    edges = [(a, b) for a in range(4) for b in range(a + 1, 4)]
    pts += [(v[a] + v[b]) / 2 for a, b in edges]
    pts += [v[a] + (v[b] - v[a]) / 3 for a, b in edges]
    return np.asarray(pts, np.float32)


def cyl24():
    pts = []
    for k, z in enumerate((-1.0, 0.0, 1.0)):
        tw = np.deg2rad(45.0 * k)
        for j in range(8):
            phi = 2 * np.pi * j / 8 + tw
            pts.append((0.4 * np.cos(phi), 0.4 * np.sin(phi), z))
    return np.asarray(pts, np.float32)


SHAPES = {
    "cube_v2": _ref([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]],
                    1.7, -5.1, 15.0, 5.80, 4.5),
    "th_v1": _ref([[-0.45, -0.45, -0.45], [-0.45, 0.45, 0.45], [0.45, -0.45, 0.45], [0.45, 0.45, -0.45]],
                  1.0, -6.7, 15.0, 5.75, 4.5),
    "pbp_v3": _ref([[-1.46946, 2.02254, 0.0], [-2.37764, -0.77254, 0.0], [-0.0, -2.5, 0.0],
                    [2.37764, -0.77254, 0.0], [1.46946, 2.02254, 0.0], [0.0, 0.0, 3.5], [0.0, 0.0, -3.5]],
                   1.0, -2.5, 15.0, 8.1, 7.5),
    "cube26": _ref(cube26(), 1.0, -5.1, 15.0, 2.5, 2.5),
    "tetra16": _ref(tetra16(), 1.0, -5.1, 15.0, 2.5, 2.5),
    "cyl24": _ref(cyl24(), 1.0, -5.1, 15.0, 2.5, 2.5),
}
