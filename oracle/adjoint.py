"""Exact pair forces and torques in FP64 by automatic differentiation
(test infrastructure only).

The reference approximates them by forward differences
(``ForceEvaluator.py:86-112``): F = -(E(x_i + dx) - E)/dx along x/y/z,
T_i = -(E(rot_i dteta) - E)/dteta, T_j likewise for body j. Here the same
quantities are the exact derivatives at zero displacement: the pair energy
E(cloud1) of the unperturbed cloud (body i at the origin, body j at the
minimum-image translation t) is differentiated with respect to every point,
then
  F_pair = -sum_{a in i} dE/dp_a,
  T_i    = -sum_{a in i} p_a x dE/dp_a              (rotation about the centre of i),
  T_j    = -sum_{a in j} (p_a - t) x dE/dp_a        (rotation about the centre of j),
each multiplied by (en_max - en_min) and clipped to [-100, 100] as the
reference does (``ForceEvaluator.py:119-132``).
"""
from __future__ import annotations

import numpy as np
import torch

from . import nep


def _act(name):
    return {"relu": torch.relu, "tanh": torch.tanh, "silu": torch.nn.functional.silu}[name]


def descriptor_torch(pts, nrad, nang, lmax, rc):
    """Differentiable FP64 descriptor (direct O(Nd^2) form of
    ``NepDescriptorKernels.py:3-144``). pts (P, Nd, 3)."""
    r = pts - pts.mean(dim=1, keepdim=True)
    d = torch.sqrt((r * r).sum(-1))
    u = d / rc
    x = 2.0 * (u - 1.0) ** 2 - 1.0
    fc = 0.5 * (1.0 + torch.cos(np.pi * u))
    T = [torch.ones_like(x), x]
    for _ in range(1, nrad):
        T.append(2.0 * x * T[-1] - T[-2])
    f = torch.stack([(1.0 + t) / 2.0 * fc for t in T[:nrad + 1]], dim=1)  # (P, nrad+1, Nd)
    rh = r / d[..., None]
    cos = torch.einsum("pak,pbk->pab", rh, rh)
    leg = [torch.ones_like(cos), cos]
    for l in range(1, lmax):
        leg.append(((2 * l + 1) * cos * leg[-1] - l * leg[-2]) / (l + 1))
    fa = f[:, :nang + 1]
    g_ang = torch.stack([torch.einsum("pna,pnb,pab->pn", fa, fa, leg[l]) for l in range(1, lmax + 1)], dim=-1)
    return torch.cat([f.sum(-1), g_ang.reshape(len(pts), -1)], dim=1)


def pair_energy_net(g, layers, act):
    h = g
    for k, (W, b) in enumerate(layers):
        h = torch.nn.functional.linear(h, torch.as_tensor(np.asarray(W, np.float64)),
                                       torch.as_tensor(np.asarray(b, np.float64)))
        if k < len(layers) - 1:
            h = _act(act)(h)
    return h[:, 0]


def exact_pair_forces(pos, quat, pairs, L, shape, hypers, layers, act, chunk=512, clip=True):
    """Per-pair (F_pair, T_i, T_j) in FP64, scaled by en_range (and clipped), the
    per-body sums (F, T) and the pair energies E = en_min + en_range * y."""
    nrad, nang, lmax = (int(h) for h in hypers[:3])
    pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
    _, _, t = nep.min_image_filter(pos, pairs, L, 1e30, np.float64)
    c1, _ = nep.pair_clouds(quat, pairs, t, shape["pts"], np.float64)
    rng = shape["en_max"] - shape["en_min"]
    h = c1.shape[1] // 2
    out_F, out_Ti, out_Tj, out_E = [], [], [], []
    for s in range(0, len(pairs), chunk):
        p = torch.tensor(c1[s:s + chunk], dtype=torch.float64, requires_grad=True)
        y = pair_energy_net(descriptor_torch(p, nrad, nang, lmax, float(shape["nep_cutoff"])), layers, act)
        (grad,) = torch.autograd.grad(y.sum(), p)
        grad = grad.numpy()
        pts = c1[s:s + chunk]
        tt = t[s:s + chunk][:, None, :]
        F = -grad[:, :h].sum(1)
        Ti = -np.cross(pts[:, :h], grad[:, :h]).sum(1)
        Tj = -np.cross(pts[:, h:] - tt, grad[:, h:]).sum(1)
        out_F.append(F * rng)
        out_Ti.append(Ti * rng)
        out_Tj.append(Tj * rng)
        out_E.append(shape["en_min"] + rng * y.detach().numpy())
    F, Ti, Tj = (np.concatenate(a) if a else np.zeros((0, 3)) for a in (out_F, out_Ti, out_Tj))
    E = np.concatenate(out_E) if out_E else np.zeros(0)
    if clip:
        F, Ti, Tj = (np.clip(a, -100.0, 100.0) for a in (F, Ti, Tj))
    N = len(pos)
    Fn, Tn = nep.scatter(pairs, F, Ti, Tj, N, np.float64)
    return dict(F_pair=F, T_i=Ti, T_j=Tj, forces=Fn, torques=Tn, E=E, pairs=pairs)


def relu_margin(pos, quat, pairs, L, shape, hypers, layers, chunk=2048):
    """Per pair, the smallest |z| over all hidden pre-activations of the net,
    in units of that layer's mean |z| over all pairs (FP64).

    A ReLU net's forces jump where a pre-activation crosses zero, so an FP32
    evaluation matches the FP64 one only on pairs whose every z stays clear of
    zero by more than the FP32 path's own error."""
    nrad, nang, lmax = (int(h) for h in hypers[:3])
    pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
    _, _, t = nep.min_image_filter(pos, pairs, L, 1e30, np.float64)
    c1, _ = nep.pair_clouds(quat, pairs, t, shape["pts"], np.float64)
    with torch.no_grad():
        g = descriptor_torch(torch.tensor(c1, dtype=torch.float64), nrad, nang, lmax, float(shape["nep_cutoff"]))
        h, margin = g, None
        for W, b in layers[:-1]:
            z = torch.nn.functional.linear(h, torch.as_tensor(np.asarray(W, np.float64)),
                                           torch.as_tensor(np.asarray(b, np.float64)))
            m = (z.abs() / z.abs().mean()).min(dim=1).values
            margin = m if margin is None else torch.minimum(margin, m)
            h = torch.relu(z)
    return margin.numpy()


def _qmul(a, b):
    w = a[..., 0] * b[..., 0] - np.sum(a[..., 1:] * b[..., 1:], axis=-1)
    v = a[..., :1] * b[..., 1:] + b[..., :1] * a[..., 1:] + np.cross(a[..., 1:], b[..., 1:])
    return np.concatenate([w[..., None], v], axis=-1)


def _pair_energies64(pos_i, pos_j, q_i, q_j, L, shape, hypers, layers, act, chunk=4096):
    """FP64 energies E = en_min + en_range * net(g) of pairs given per row by
    both bodies' centres and orientations (minimum image in a cubic box L)."""
    nrad, nang, lmax = (int(h) for h in hypers[:3])
    d = pos_j - pos_i
    t = d - L * np.round(d / L)
    R = len(t)
    pos2 = np.zeros((2 * R, 3))
    pos2[1::2] = t
    quat2 = np.empty((2 * R, 4))
    quat2[0::2], quat2[1::2] = q_i, q_j
    pr = np.arange(2 * R, dtype=np.int64).reshape(-1, 2)
    c1, _ = nep.pair_clouds(quat2, pr, t, shape["pts"], np.float64)
    rng = shape["en_max"] - shape["en_min"]
    out = []
    with torch.no_grad():
        for s in range(0, R, chunk):
            p = torch.tensor(c1[s:s + chunk], dtype=torch.float64)
            y = pair_energy_net(descriptor_torch(p, nrad, nang, lmax, float(shape["nep_cutoff"])), layers, act)
            out.append(shape["en_min"] + rng * y.numpy())
    return np.concatenate(out) if out else np.zeros(0)


def central_difference_forces(pos, quat, pairs, L, shape, hypers, layers, act, bodies, h=1e-4):
    """Forces and torques on ``bodies`` by FP64 central differences of the summed
    energy of their pairs: F_k = -(U(x + h e_k) - U(x - h e_k)) / 2h and
    T_k = -(U(R_k(h) q) - U(R_k(-h) q)) / 2h with R_k(a) the world-frame
    rotation by angle a about axis k applied on the left of the body's
    quaternion (rotation about the body's centre). Unclipped. The pair set is
    held fixed (the filtered list at the unperturbed positions)."""
    pos = np.asarray(pos, np.float64)
    quat = np.asarray(quat, np.float64)
    pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
    bodies = np.asarray(bodies, np.int64)
    eye = np.eye(3)
    dq = []
    for k in range(3):
        for sgn in (1.0, -1.0):
            dq.append(np.concatenate([[np.cos(sgn * h / 2)], np.sin(sgn * h / 2) * eye[k]]))
    rows_i, rows_j, rows_qi, rows_qj, owner, kind = [], [], [], [], [], []
    for n, b in enumerate(bodies):
        sel = np.nonzero((pairs[:, 0] == b) | (pairs[:, 1] == b))[0]
        for m in range(12):
            pi, pj = pos[pairs[sel, 0]].copy(), pos[pairs[sel, 1]].copy()
            qi, qj = quat[pairs[sel, 0]].copy(), quat[pairs[sel, 1]].copy()
            is_i = pairs[sel, 0] == b
            if m < 6:
                delta = (1.0 if m % 2 == 0 else -1.0) * h * eye[m // 2]
                pi[is_i] += delta
                pj[~is_i] += delta
            else:
                r = dq[m - 6]
                qi[is_i] = _qmul(r, qi[is_i])
                qj[~is_i] = _qmul(r, qj[~is_i])
            rows_i.append(pi)
            rows_j.append(pj)
            rows_qi.append(qi)
            rows_qj.append(qj)
            owner.append(np.full(len(sel), n))
            kind.append(np.full(len(sel), m))
    E = _pair_energies64(np.concatenate(rows_i), np.concatenate(rows_j), np.concatenate(rows_qi),
                         np.concatenate(rows_qj), L, shape, hypers, layers, act)
    U = np.zeros((len(bodies), 12))
    np.add.at(U, (np.concatenate(owner), np.concatenate(kind)), E)
    F = -(U[:, 0:6:2] - U[:, 1:6:2]) / (2 * h)
    T = -(U[:, 6:12:2] - U[:, 7:12:2]) / (2 * h)
    return F, T
