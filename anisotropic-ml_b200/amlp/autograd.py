"""Pair energies as a ``torch.autograd.Function`` over libamlp.

``PairEnergy.apply(pos, quat, w, pairs, box, model, clip)`` returns the energy
of every listed pair, E_p = en_min + (en_max - en_min) net(g_p) with g_p the
descriptor of the unperturbed pair (``DescriptorGenerator.py:136-161`` variant
0 and ``ForceEvaluator.py:80-83``). Its backward is the adjoint of descriptor
and net:

* positions and orientations: ``amlp_pair_energy_vjp`` recomputes each pair's
  descriptor (nothing per pair is kept from the forward), runs the net forward
  and backward on the tensor cores and the descriptor backward, and scatters
  F = -sum_p w_p dE_p/dx and T = -sum_p w_p dE_p/dtheta for the upstream
  gradient w. The position gradient is -F; the quaternion gradient is the
  tangent vector G = -2 sum_k T_k ((0, e_k) (x) q), so that a world-frame
  rotation of the body by a small angle vector theta, q -> q + 1/2 (0, theta)
  (x) q, changes the energy by G . dq = -T . theta (``torque_from_quat_grad``
  inverts it). With ``clip`` the per-pair terms are clipped to [-100, 100] as
  the force path does (``ForceEvaluator.py:119-132``), so that the gradient of
  the summed energy is the simulation's force; without it the product is exact.
* weights: ``amlp_mlp_backward`` over the recomputed descriptors, FP32.

``mse_loss_grad`` is the training loss of ``05/FFNN.py:95-106`` (MSELoss on
energies normalised as ``05/FFNN.py:59-63``) and its weight gradient in one call.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import ACT, Mlp, Nep, call, size_query
from .shapes import Shape, get_shape


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


class PairModel:
    """Descriptor constants of one body shape and the structure of its net
    (layer widths and activation); the weights are passed per call."""

    def __init__(self, shape: Shape | str, hypers, dims, act: str, device="cuda"):
        if isinstance(shape, str):
            shape = get_shape(shape)
        if act not in ACT:
            raise ValueError(f"activation {act!r} not in {sorted(ACT)}")
        self.shape = shape
        self.device = torch.device(device)
        self.dims = [int(d) for d in dims]
        self.act = act
        self.D = (hypers.nrad + 1) + (hypers.nang + 1) * hypers.lmax
        if self.dims[0] != self.D or self.dims[-1] != 1:
            raise ValueError(f"net dims {self.dims} do not map {self.D} descriptors to one energy")
        self.n_weights = sum(self.dims[k + 1] * (self.dims[k] + 1) for k in range(len(self.dims) - 1))
        self.pts = torch.tensor(np.asarray(shape.pts, np.float32), device=self.device).contiguous()
        self.nep = Nep()
        self.nep.nrad, self.nep.nang, self.nep.lmax = hypers.nrad, hypers.nang, hypers.lmax
        self.nep.npts = shape.npts
        self.nep.d_pts = self.pts.data_ptr()
        self.nep.cutoff = float(shape.cutoff)
        self.nep.nep_cutoff = float(shape.nep_cutoff)
        self.nep.en_min, self.nep.en_max = float(shape.en_min), float(shape.en_max)
        self.nep.dx = self.nep.dteta = 1e-5
        self.en_min = float(np.float32(shape.en_min))
        self.en_range = float(np.float32(np.float32(shape.en_max) - np.float32(shape.en_min)))

    def mlp(self, w: torch.Tensor) -> Mlp:
        if w.dtype != torch.float32 or not w.is_contiguous() or w.numel() != self.n_weights:
            raise ValueError(f"weights must be a contiguous float32 vector of {self.n_weights} values")
        m = Mlp()
        m.n_layers = len(self.dims) - 1
        for k, d in enumerate(self.dims):
            m.dims[k] = d
        m.act = ACT[self.act]
        m.d_w = w.data_ptr()
        return m

    def descriptors(self, pos, quat, pairs, box: float) -> torch.Tensor:
        """(P, D) descriptors of the unperturbed pairs."""
        P = pairs.shape[0]
        g = torch.empty(max(P, 1), self.D, dtype=torch.float32, device=self.device)
        if P == 0:
            return g[:0]
        npairs = torch.tensor([P], dtype=torch.int64, device=self.device)
        call("amlp_pair_descriptors", pos.data_ptr(), quat.data_ptr(), float(box), pairs.data_ptr(),
             npairs.data_ptr(), max(P, 1), ctypes.byref(self.nep), g.data_ptr(), self.D, _stream())
        return g[:P]


def _check_inputs(model: PairModel, pos, quat, w, pairs):
    for name, t, dt in (("pos", pos, torch.float32), ("quat", quat, torch.float32), ("w", w, torch.float32),
                        ("pairs", pairs, torch.int32)):
        if t.device != model.device or t.dtype != dt or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous {dt} tensor on {model.device}")
    if pos.dim() != 2 or pos.shape[1] != 3 or quat.shape != (pos.shape[0], 4):
        raise ValueError("pos must be (N, 3) and quat (N, 4)")
    if pairs.dim() != 2 or pairs.shape[1] != 2:
        raise ValueError("pairs must be (P, 2)")


class PairEnergy(torch.autograd.Function):
    """Energies of listed pairs, differentiable in positions, orientations and
    net weights (see the module docstring)."""

    @staticmethod
    def forward(ctx, pos, quat, w, pairs, box: float, model: PairModel, clip: bool = False):
        _check_inputs(model, pos, quat, w, pairs)
        P = pairs.shape[0]
        mlp = model.mlp(w)
        g = model.descriptors(pos, quat, pairs, box)
        y = torch.empty(max(P, 1), dtype=torch.float32, device=model.device)
        if P:
            call("amlp_mlp_energy", g.data_ptr(), P, ctypes.byref(mlp), y.data_ptr(), _stream())
        ctx.save_for_backward(pos, quat, w, pairs)
        ctx.box, ctx.model, ctx.clip = float(box), model, bool(clip)
        return y[:P] * model.en_range + model.en_min

    @staticmethod
    def backward(ctx, dE):
        pos, quat, w, pairs = ctx.saved_tensors
        model: PairModel = ctx.model
        P = pairs.shape[0]
        dE = dE.to(torch.float32).contiguous()
        mlp = model.mlp(w)
        g_pos = g_quat = g_w = None
        if (ctx.needs_input_grad[0] or ctx.needs_input_grad[1]) and P:
            N = pos.shape[0]
            F = torch.zeros(N, 3, dtype=torch.float32, device=model.device)
            T = torch.zeros(N, 3, dtype=torch.float32, device=model.device)
            npairs = torch.tensor([P], dtype=torch.int64, device=model.device)
            ws = torch.empty(size_query("amlp_adjoint_workspace_bytes", P), dtype=torch.uint8, device=model.device)
            call("amlp_pair_energy_vjp", pos.data_ptr(), quat.data_ptr(), ctx.box, pairs.data_ptr(),
                 npairs.data_ptr(), P, ctypes.byref(model.nep), ctypes.byref(mlp), dE.data_ptr(), int(ctx.clip),
                 F.data_ptr(), T.data_ptr(), None, ws.data_ptr(), ws.numel(), _stream())
            g_pos = -F if ctx.needs_input_grad[0] else None
            g_quat = quat_grad_from_torque(quat, T) if ctx.needs_input_grad[1] else None
        elif ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            g_pos = torch.zeros_like(pos) if ctx.needs_input_grad[0] else None
            g_quat = torch.zeros_like(quat) if ctx.needs_input_grad[1] else None
        if ctx.needs_input_grad[2]:
            g_w = torch.zeros_like(w)
            if P:
                g = model.descriptors(pos, quat, pairs, ctx.box)
                dy = (dE * model.en_range).contiguous()
                call("amlp_mlp_backward", g.data_ptr(), dy.data_ptr(), P, ctypes.byref(mlp), g_w.data_ptr(),
                     _stream())
        return g_pos, g_quat, g_w, None, None, None, None


def pair_energies(pos, quat, w, pairs, box: float, model: PairModel, clip: bool = False) -> torch.Tensor:
    return PairEnergy.apply(pos, quat, w, pairs, box, model, clip)


def quat_grad_from_torque(quat: torch.Tensor, T: torch.Tensor) -> torch.Tensor:
    """G = -2 (0, T) (x) q for q = (w, u): (2 T.u, -2 (w T + T x u))."""
    w, u = quat[:, :1], quat[:, 1:]
    G = torch.empty_like(quat)
    G[:, 0] = 2.0 * (T * u).sum(1)
    G[:, 1:] = -2.0 * (w * T + torch.cross(T, u, dim=1))
    return G


def torque_from_quat_grad(quat: torch.Tensor, G: torch.Tensor) -> torch.Tensor:
    """T_k = -1/2 G . ((0, e_k) (x) q) (unit q), the inverse of quat_grad_from_torque."""
    w, u = quat[:, :1], quat[:, 1:]
    T = torch.empty(quat.shape[0], 3, dtype=quat.dtype, device=quat.device)
    eye = torch.eye(3, dtype=quat.dtype, device=quat.device)
    for k in range(3):
        e = eye[k].expand_as(u)
        b0 = -u[:, k]
        bv = w * e + torch.cross(e, u, dim=1)
        T[:, k] = -0.5 * (G[:, 0] * b0 + (G[:, 1:] * bv).sum(1))
    return T


def normalised_energies(E: torch.Tensor, en_min: float, en_max: float) -> torch.Tensor:
    """Training labels of ``05/FFNN.py:59-63``: E capped at en_max, mapped to
    (E - en_min) / (en_max - en_min), clamped to [0, 1]."""
    y = (torch.clamp(E, max=en_max) - en_min) / (en_max - en_min)
    return torch.clamp(y, 0.0, 1.0)


def mse_loss_grad(model: PairModel, w: torch.Tensor, g: torch.Tensor, y: torch.Tensor):
    """Mean squared error of net(g) against normalised labels y and its gradient
    with respect to the packed weights (one kernel). Returns (loss, grad)."""
    g = g.to(torch.float32).contiguous()
    y = y.to(torch.float32).contiguous()
    if g.dim() != 2 or g.shape[1] != model.D or y.shape != (g.shape[0],):
        raise ValueError("g must be (B, D) and y (B,)")
    grad = torch.zeros_like(w)
    loss = torch.zeros(1, dtype=torch.float64, device=model.device)
    call("amlp_mlp_loss_grad", g.data_ptr(), y.data_ptr(), g.shape[0], ctypes.byref(model.mlp(w)), grad.data_ptr(),
         loss.data_ptr(), _stream())
    return loss, grad
