"""Drop-in ``DescriptorGenerator`` (reference: ``nep_simulator/DescriptorGenerator.py``).

Same methods, argument order and return values; arrays are torch CUDA tensors
instead of CuPy arrays. ``generate_nep_descriptors`` returns the reference's
``(g_all (10P, D) float32, pp (P, 2) int64, P)`` with rows ``v*P + p`` for
finite-difference variant v of filtered pair p (``DescriptorGenerator.py:136-161``),
computed by ``amlp_pair_filter`` + ``amlp_descriptors``.

Differences: an unknown shape raises ``KeyError`` instead of ``exit()``
(``:121-123``); descriptors use every point of the cloud for any point count
(the reference's fixed launch shapes only cover clouds of <= 12 points, ``:336-337``).
"""
import ctypes
import time

import numpy as np
import torch

import _amlp_path  # noqa: F401  (puts the amlp package on sys.path)
from amlp import _lib
from amlp._lib import Nep, call
from amlp.shapes import get_shape


class DescriptorGenerator:
    def set_timers(self):
        self.t_pos_to_pts = 0
        self.t_dx = 0
        self.t_pts_to_nep = 0
        self.t_nep1 = self.t_nep2 = self.t_nep3 = self.t_nep4 = self.t_nep5 = 0
        self.is_sync = 0

    def setDevice(self, gpu_id):
        self.set_timers()
        if isinstance(gpu_id, torch.device):
            self.device = gpu_id
        else:
            self.device = torch.device("cuda", int(getattr(gpu_id, "index", gpu_id) or 0))
        self.gpu_id = self.device.index or 0

    def setHyperParameters(self, hypers):
        self.nrad = int(hypers[0])
        self.nang = int(hypers[1])
        self.lmax = int(hypers[2])
        self.cutoff_nep = hypers[3] if len(hypers) > 3 else None  # stored, unused (as in the reference)
        self.N_descriptors = (self.nrad + 1) + (self.nang + 1) * self.lmax

    def setSync(self, is_sync):
        self.is_sync = is_sync

    def getN_descriptor(self):
        return self.N_descriptors

    def setBoxSize(self, Lx):
        self.Lx = float(np.float32(Lx))

    def set_dx_dteta(self, dx, dteta):
        self.dx = float(dx)
        self.dteta = float(dteta)

    def setShape(self, shape_str):
        s = get_shape(shape_str)
        self.shape = s
        self.pts_rep = torch.tensor(s.pts, dtype=torch.float32, device=self.device)
        self.Npts = s.npts
        self.Nd = s.nd
        self.en_min, self.en_max = s.en_min, s.en_max
        self.cutoff = s.cutoff
        self.nep_cutoff = s.nep_cutoff

    def get_en_min_max(self):
        return self.en_min, self.en_max

    def move_data_to_device(self):
        self.pts_rep = self.pts_rep.to(self.device).contiguous()

    def nep_struct(self):
        n = Nep()
        n.nrad, n.nang, n.lmax = self.nrad, self.nang, self.lmax
        n.npts = self.Npts
        n.d_pts = self.pts_rep.data_ptr()
        n.cutoff = float(self.cutoff)
        n.nep_cutoff = float(self.nep_cutoff)
        n.en_min, n.en_max = float(self.en_min), float(self.en_max)
        n.dx, n.dteta = self.dx, self.dteta
        return n

    def _sync(self):
        if self.is_sync == 1:
            torch.cuda.synchronize(self.device)

    def generate_nep_descriptors(self, central_pos, orientations, Nlist):
        """(g_all, pp, N_pair) for the current positions/orientations (``:136-161``)."""
        self._sync()
        t0 = time.time()
        self.pos_to_pts(central_pos, orientations, Nlist)
        self._sync()
        t1 = time.time()
        self.pts_to_nep_descriptors()
        self._sync()
        t2 = time.time()
        self.t_pos_to_pts += t1 - t0
        self.t_pts_to_nep += t2 - t1
        return self.g_all, self.pp, self.N_pair

    def pos_to_pts(self, central_pos, orientations, Nlist):
        """Minimum image and pair filter (``:163-182``); keeps the inputs for the
        descriptor pass, which builds the rotated point clouds on chip."""
        self._pos = central_pos.contiguous()
        self._quat = orientations.contiguous()
        nl = Nlist if isinstance(Nlist, torch.Tensor) else torch.as_tensor(np.asarray(Nlist))
        nl = nl.to(self.device, torch.int32).contiguous()
        nv = nl.shape[0]
        self._nv = torch.tensor([nv], dtype=torch.int64, device=self.device)
        cap = max(nv, 1)
        self._pairs = torch.empty(cap, 2, dtype=torch.int32, device=self.device)
        self._np = torch.zeros(1, dtype=torch.int64, device=self.device)
        ws = torch.empty(max(1, _lib.size_query("amlp_filter_workspace_bytes", cap)), dtype=torch.uint8,
                         device=self.device)
        if nv:
            call("amlp_pair_filter", self._pos.data_ptr(), self.Lx, float(self.cutoff), nl.data_ptr(),
                 self._nv.data_ptr(), nv, self._pairs.data_ptr(), self._np.data_ptr(), ws.data_ptr(), ws.numel(),
                 torch.cuda.current_stream(self.device).cuda_stream)
        self.N_pair = int(self._np.item())  # data-dependent count, as cp.where (:172)
        self.pairs = self._pairs[:self.N_pair]
        self.pp = self.pairs.to(torch.int64)

    def pts_to_nep_descriptors(self):
        P = self.N_pair
        self.g_all = torch.empty(10 * P, self.N_descriptors, dtype=torch.float32, device=self.device)
        self._nep = self.nep_struct()
        if P:
            call("amlp_descriptors", self._pos.data_ptr(), self._quat.data_ptr(), self.Lx, self.pairs.data_ptr(), P,
                 ctypes.byref(self._nep), self.g_all.data_ptr(), torch.cuda.current_stream(self.device).cuda_stream)
