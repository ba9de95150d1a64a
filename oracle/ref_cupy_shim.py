"""Numpy-backed stand-in for CuPy, used to run the reference's own Python classes
on the CPU of the development container (TEST INFRASTRUCTURE ONLY).

``install()`` registers stand-ins for ``cupy``, ``gsd.hoomd`` and
``matplotlib.pyplot`` in ``sys.modules`` and a loader that executes the
reference modules from their ``.py`` source (never from a cached bytecode
file). ``cupy.RawKernel`` launches the host-compiled kernel of
``oracle/ref_kernels.py``; ``radial_grad``, whose block-level shared-memory sum
cannot run one thread after another, runs through the oracle's restatement
``oracle.nep.radial`` and writes the kernel's output buffers in the kernel's
layout.

Differences from running on a GPU, all below FP32 rounding: host libm instead
of CUDA's cosf/sinf/expf, no FMA contraction, numpy/BLAS summation order in
``cp.sum``/``cp.matmul``, and the FFNN on torch's CPU path.
"""
from __future__ import annotations

import ctypes
import importlib.abc
import importlib.util
import os
import sys
import types

import numpy as np

from . import ref_kernels
from . import nep as onep


class ndarray(np.ndarray):
    """numpy array with CuPy's ``.get()``."""

    def get(self):
        return np.array(self)


def _wrap(a):
    if isinstance(a, np.ndarray):
        return a.view(ndarray)
    return np.asarray(a).view(ndarray)


def _make_cupy():
    cp = types.ModuleType("cupy")
    cp.ndarray = ndarray
    cp.float32, cp.float64, cp.int32, cp.int64 = np.float32, np.float64, np.int32, np.int64

    def asarray(a, dtype=None):
        if isinstance(a, ndarray):
            return a if dtype is None or a.dtype == np.dtype(dtype) else _wrap(a.astype(dtype))
        return _wrap(np.array(a, dtype=dtype, copy=True))

    cp.asarray = asarray
    cp.array = lambda a, dtype=None: _wrap(np.array(a, dtype=dtype, copy=True))
    cp.empty = lambda shape, dtype=np.float32: _wrap(np.zeros(shape, dtype))
    cp.zeros = lambda shape, dtype=np.float32: _wrap(np.zeros(shape, dtype))
    cp.ones = lambda shape, dtype=np.float32: _wrap(np.ones(shape, dtype))
    cp.empty_like = lambda a: _wrap(np.zeros_like(a))
    cp.zeros_like = lambda a: _wrap(np.zeros_like(a))
    cp.copy = lambda a: _wrap(np.array(a, copy=True))
    cp.vstack = lambda t: _wrap(np.vstack(t))
    cp.hstack = lambda t: _wrap(np.hstack(t))
    cp.einsum = lambda s, *a: _wrap(np.einsum(s, *a))
    cp.matmul = lambda a, b: _wrap(np.matmul(a, b))
    cp.cross = lambda a, b: _wrap(np.cross(a, b))

    def where(c, a=None, b=None):
        if a is None:
            return tuple(_wrap(x) for x in np.where(c))
        return _wrap(np.where(c, a, b))

    cp.where = where

    def csum(a, axis=None):
        return _wrap(np.asarray(np.sum(np.asarray(a), axis=axis)))

    cp.sum = csum
    linalg = types.ModuleType("cupy.linalg")
    linalg.norm = lambda a, axis=None: _wrap(np.asarray(np.linalg.norm(np.asarray(a), axis=axis)))
    cp.linalg = linalg
    cp.from_dlpack = lambda t: _wrap(np.from_dlpack(t))

    cuda = types.ModuleType("cupy.cuda")

    class Device:
        def __init__(self, i=0):
            self.id = i

        def use(self):
            pass

    class _Null:
        @staticmethod
        def synchronize():
            pass

    class Stream:
        null = _Null()

    cuda.Device, cuda.Stream = Device, Stream
    cp.cuda = cuda
    cp.RawKernel = RawKernel
    return cp


class RawKernel:
    """Launch of a reference kernel on the host (see module docstring)."""

    def __init__(self, code, name, **kw):
        self.code, self.name = code, name
        self._fn = None

    def __call__(self, grid, block, args):
        if self.name == "radial_grad":
            return _radial_grad(*args)
        if self._fn is None:
            self._fn, self._params = ref_kernels.load(self.name)
        cargs = []
        for (t, n), a in zip(self._params, args):
            if "*" in t:
                arr = np.asarray(a)
                want = np.float32 if "float" in t else np.int32
                if arr.dtype != want:
                    raise TypeError(f"{self.name}: {n} has dtype {arr.dtype}, kernel wants {want}")
                if not arr.flags.c_contiguous:
                    raise TypeError(f"{self.name}: {n} is not contiguous")
                cargs.append(arr.ctypes.data_as(ctypes.c_void_p))
            else:
                cargs.append(int(a))
        self._fn(int(grid[0]), int(block[0]), *cargs)


def _radial_grad(pos, r_ij, r_ij_norm, chebo, g_rad, nep_cutoff, n_pairs, n_cheb, Nd):
    """Intended semantics of ``radial_grad`` written into its output buffers."""
    n_pairs, n_cheb, Nd = int(n_pairs), int(n_cheb), int(Nd)
    pts = np.asarray(pos)[:n_pairs].reshape(n_pairs, Nd, 3)
    r, norm, ch, g = onep.radial(pts, n_cheb - 1, float(np.asarray(nep_cutoff).reshape(-1)[0]))
    np.asarray(r_ij)[:n_pairs] = r
    np.asarray(r_ij_norm)[:n_pairs] = norm
    np.asarray(chebo)[:n_pairs] = ch
    np.asarray(g_rad)[:n_pairs] = g


# ----------------------------------------------------------------------------- gsd stand-in
def _make_gsd():
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(repo, "anisotropic-ml_b200"))
    from amlp import gsd as g

    gsd = types.ModuleType("gsd")
    hoomd = types.ModuleType("gsd.hoomd")

    class _NS:
        pass

    class Frame:
        def __init__(self):
            self.configuration = _NS()
            self.configuration.step = 0
            self.configuration.box = [1, 1, 1, 0, 0, 0]
            self.particles = _NS()
            p = self.particles
            p.N = 0
            p.types = ["A"]
            for k in ("position", "typeid", "mass", "orientation", "angmom", "velocity",
                      "moment_inertia", "body", "charge"):
                setattr(p, k, None)

    def _to_frame(f):
        fr = Frame()
        fr.configuration.step = f.step
        fr.configuration.box = f.box
        fr.particles.N = f.N
        fr.particles.types = f.types
        for k in ("position", "typeid", "mass", "orientation", "angmom", "velocity",
                  "moment_inertia", "body", "charge"):
            setattr(fr.particles, k, f.get(k))
        return fr

    class _File:
        def __init__(self, name, mode="r"):
            self._g = g.GsdFile(name, {"w": "w", "r": "r", "r+": "r+", "a": "a"}[mode])

        def __len__(self):
            return len(self._g)

        def __getitem__(self, k):
            return _to_frame(self._g[k])

        def append(self, fr):
            f = g.Frame()
            f.step = int(fr.configuration.step)
            f.box = np.asarray([float(np.asarray(x)) for x in fr.configuration.box], np.float32)
            f.N = int(fr.particles.N)
            f.types = list(fr.particles.types)
            for k in ("position", "typeid", "mass", "orientation", "angmom", "velocity", "moment_inertia"):
                v = getattr(fr.particles, k)
                if v is not None:
                    f.particles[k] = np.asarray(v)
            self._g.append(f)

        def __enter__(self):
            return self

        def __exit__(self, *e):
            self._g.close()

    hoomd.Frame = Frame
    hoomd.open = lambda name, mode="r": _File(name, mode)
    gsd.hoomd = hoomd
    return gsd, hoomd


class _SourceOnlyFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    """Imports the reference modules by compiling their .py source."""

    def __init__(self, root):
        self.root = root

    def find_spec(self, name, path, target=None):
        parts = name.split(".")
        base = os.path.join(self.root, *parts)
        if os.path.isfile(base + ".py"):
            return importlib.util.spec_from_loader(name, self, origin=base + ".py")
        if os.path.isdir(base) and parts[0] == "cudakernels":
            spec = importlib.util.spec_from_loader(name, self, origin=base, is_package=True)
            spec.submodule_search_locations = [base]
            return spec
        return None

    def create_module(self, spec):
        return None

    def exec_module(self, module):
        origin = module.__spec__.origin
        if os.path.isdir(origin):
            module.__path__ = [origin]
            return
        with open(origin) as fh:
            src = fh.read()
        module.__file__ = origin
        exec(compile(src, origin, "exec"), module.__dict__)


def install(reference_root: str = ref_kernels.REF_ROOT):
    """Register the stand-ins; returns the reference's ``nep_simulator`` dir."""
    ref_kernels.build()
    sys.modules["cupy"] = _make_cupy()
    sys.modules["cupy.cuda"] = sys.modules["cupy"].cuda
    gsd, hoomd = _make_gsd()
    sys.modules["gsd"], sys.modules["gsd.hoomd"] = gsd, hoomd
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt
    sys.modules["matplotlib"], sys.modules["matplotlib.pyplot"] = mpl, plt
    root = os.path.join(reference_root, "nep_simulator")
    sys.meta_path.insert(0, _SourceOnlyFinder(root))
    import torch
    if not getattr(torch.nn.Module.to, "_amlp_cpu", False):
        orig = torch.nn.Module.to

        def to(self, *a, **k):
            if a and isinstance(a[0], str) and a[0].startswith("cuda"):
                return self
            return orig(self, *a, **k)

        to._amlp_cpu = True
        torch.nn.Module.to = to
    return root
