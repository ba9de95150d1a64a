"""Thin wrappers that call single libamlp entry points on torch tensors (tests only)."""
import ctypes

import numpy as np
import torch

from amlp import _lib
from amlp._lib import Mlp, Nep, call, size_query
from amlp.engine import EnergyNet

DEV = torch.device("cuda:0")


def stream():
    return torch.cuda.current_stream().cuda_stream


def t32(a):
    return torch.tensor(np.asarray(a, np.float32), device=DEV).contiguous()


def nlist(pos, L, r, cap=None):
    pos_t = t32(pos)
    n = len(pos)
    ws = torch.empty(size_query("amlp_nlist_workspace_bytes", n, float(L), float(r)), dtype=torch.uint8, device=DEV)
    cnt = torch.zeros(1, dtype=torch.int64, device=DEV)
    cap_given = cap
    cap = cap if cap is not None else max(16, n * 64)
    out = torch.empty(cap, 2, dtype=torch.int32, device=DEV)
    call("amlp_nlist_build", pos_t.data_ptr(), n, float(L), float(r), out.data_ptr(), cap, cnt.data_ptr(),
         ws.data_ptr(), ws.numel(), stream())
    k = int(cnt.item())
    if k > cap and cap_given is None:
        return nlist(pos, L, r, cap=k)
    return out[:min(k, cap)].cpu().numpy().astype(np.int64), k


def nep_struct(shape, hypers, pts_t, dx=1e-5, dteta=1e-5):
    n = Nep()
    n.nrad, n.nang, n.lmax = (int(h) for h in hypers[:3])
    n.npts = len(shape["pts"])
    n.d_pts = pts_t.data_ptr()
    n.cutoff = float(shape["cutoff"])
    n.nep_cutoff = float(shape["nep_cutoff"])
    n.en_min, n.en_max = float(shape["en_min"]), float(shape["en_max"])
    n.dx, n.dteta = float(dx), float(dteta)
    return n


def pair_filter(pos, L, cutoff, vpairs):
    pos_t = t32(pos)
    vp = torch.tensor(np.asarray(vpairs, np.int32).reshape(-1, 2), device=DEV).contiguous()
    nv = torch.tensor([len(vp)], dtype=torch.int64, device=DEV)
    cap = max(1, len(vp))
    out = torch.empty(cap, 2, dtype=torch.int32, device=DEV)
    npairs = torch.zeros(1, dtype=torch.int64, device=DEV)
    ws = torch.empty(size_query("amlp_filter_workspace_bytes", cap), dtype=torch.uint8, device=DEV)
    call("amlp_pair_filter", pos_t.data_ptr(), float(L), float(cutoff), vp.data_ptr(), nv.data_ptr(), cap,
         out.data_ptr(), npairs.data_ptr(), ws.data_ptr(), ws.numel(), stream())
    k = int(npairs.item())
    return out[:k].cpu().numpy().astype(np.int64)


def descriptors(pos, quat, L, pairs, shape, hypers):
    pts_t = t32(shape["pts"])
    D = (hypers[0] + 1) + (hypers[1] + 1) * hypers[2]
    P = len(pairs)
    g = torch.empty(10 * P, D, dtype=torch.float32, device=DEV)
    pr = torch.tensor(np.asarray(pairs, np.int32).reshape(-1, 2), device=DEV).contiguous()
    n = nep_struct(shape, hypers, pts_t)
    pos_t, quat_t = t32(pos), t32(quat)  # keep the inputs alive across the asynchronous call
    call("amlp_descriptors", pos_t.data_ptr(), quat_t.data_ptr(), float(L), pr.data_ptr(), P, ctypes.byref(n),
         g.data_ptr(), stream())
    return g.cpu().numpy()


def pair_descriptors(pos, quat, L, pairs, shape, hypers, ld=None):
    """amlp_pair_descriptors: one descriptor row per pair (the adjoint path's forward)."""
    pts_t = t32(shape["pts"])
    D = (hypers[0] + 1) + (hypers[1] + 1) * hypers[2]
    ld = ld or D
    P = len(pairs)
    g = torch.full((max(P, 1), ld), float("nan"), dtype=torch.float32, device=DEV)
    pr = torch.tensor(np.asarray(pairs, np.int32).reshape(-1, 2), device=DEV).contiguous()
    npairs = torch.tensor([P], dtype=torch.int64, device=DEV)
    n = nep_struct(shape, hypers, pts_t)
    pos_t, quat_t = t32(pos), t32(quat)
    call("amlp_pair_descriptors", pos_t.data_ptr(), quat_t.data_ptr(), float(L), pr.data_ptr(), npairs.data_ptr(),
         max(P, 1), ctypes.byref(n), g.data_ptr(), ld, stream())
    return g[:P].cpu().numpy()


def mlp_energy(layers, act, g):
    net = EnergyNet(layers, act, DEV)
    gt = t32(g)
    e = torch.empty(len(g), dtype=torch.float32, device=DEV)
    call("amlp_mlp_energy", gt.data_ptr(), len(g), ctypes.byref(net.struct), e.data_ptr(), stream())
    return e.cpu().numpy()


def fd_scatter(e, pairs, N, shape):
    pts_t = t32(shape["pts"])
    n = nep_struct(shape, (10, 8, 4), pts_t)
    P = len(pairs)
    F = torch.zeros(N, 3, dtype=torch.float32, device=DEV)
    T = torch.zeros(N, 3, dtype=torch.float32, device=DEV)
    pe = torch.zeros(1, dtype=torch.float64, device=DEV)
    pr = torch.tensor(np.asarray(pairs, np.int32).reshape(-1, 2), device=DEV).contiguous()
    e_t = t32(e)
    call("amlp_fd_scatter", e_t.data_ptr(), P, pr.data_ptr(), ctypes.byref(n), F.data_ptr(), T.data_ptr(),
         pe.data_ptr(), stream())
    return F.cpu().numpy(), T.cpu().numpy(), float(pe.item())


def fused_forces(pos, quat, L, pairs, shape, hypers, layers, act, method="amlp_forces_fd"):
    pts_t = t32(shape["pts"])
    n = nep_struct(shape, hypers, pts_t)
    net = EnergyNet(layers, act, DEV)
    N = len(pos)
    P = len(pairs)
    F = torch.zeros(N, 3, dtype=torch.float32, device=DEV)
    T = torch.zeros(N, 3, dtype=torch.float32, device=DEV)
    pe = torch.zeros(1, dtype=torch.float64, device=DEV)
    pr = torch.zeros(max(P, 1), 2, dtype=torch.int32, device=DEV)
    if P:
        pr[:P] = torch.tensor(np.asarray(pairs, np.int32).reshape(-1, 2), device=DEV)
    npairs = torch.tensor([P], dtype=torch.int64, device=DEV)
    pos_t, quat_t = t32(pos), t32(quat)
    args = [pos_t.data_ptr(), quat_t.data_ptr(), float(L), pr.data_ptr(), npairs.data_ptr(), max(P, 1),
            ctypes.byref(n), ctypes.byref(net.struct), F.data_ptr(), T.data_ptr(), pe.data_ptr()]
    if method == "amlp_forces_adjoint_wide":
        ws = torch.empty(size_query("amlp_adjoint_workspace_bytes", max(P, 1)), dtype=torch.uint8, device=DEV)
        args += [ws.data_ptr(), ws.numel()]
    e = None
    if method == "amlp_forces_fd_energies":
        e = torch.full((10 * max(P, 1),), float("nan"), dtype=torch.float32, device=DEV)
        args += [e.data_ptr()]
    call(method, *args, stream())
    out = (F.cpu().numpy(), T.cpu().numpy(), float(pe.item()))
    return out + (e[:10 * P].cpu().numpy(),) if e is not None else out
