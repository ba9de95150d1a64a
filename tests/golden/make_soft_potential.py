"""Train the SiLU pair-energy nets of the twisted-cylinder (``cyl24``,
47->128->128->1) and tetrahedron (``tetra16``, 47->128->128->128->1) workloads and
write them to ``model_<shape>_soft.npz`` in this directory.

A random net has no meaning as a potential: its pair energy at the 2.5 pair
cutoff is far from zero, so every pair that crosses the cutoff changes the
total energy by a jump. This net is fitted instead to a smooth, short-ranged
ground truth, so that it can drive NVE runs whose energy drift means something:

    E_ij = sum_{a in i, b in j} eps (1 - r_ab / r_c)^3   for r_ab < r_c,

the soft repulsion of the two bodies' interaction points, eps = 10. For the
cylinders r_c = 0.34: with points at most sqrt(1 + 0.4^2) = 1.077 from a
cylinder's centre, E_ij is exactly 0 beyond a centre distance of
2 * 1.077 + 0.34 = 2.494, inside the 2.5 cutoff. For the tetrahedra (points at
most sqrt(3/8) = 0.612 from the centre) r_c = 0.5, so E_ij vanishes beyond 1.72.

Training data: 262,144 pairs, three quarters with the centre distance uniform
in [0.4, 3.0] and one quarter uniform in [zero_from - 0.3, 3.0] (where the label
is 0 or nearly so; zero_from is the distance beyond which E_ij vanishes),
uniform random orientations (seed 0); labels in FP64 from the
formula above, normalised as the reference's training code does
(``05/FFNN.py:59-63``); descriptors from ``amlp_pair_descriptors`` on the GPU.
The net sees standardised descriptors during training; the standardisation is
folded into the first layer before saving, so the saved net takes raw
descriptors like the reference's. Loss: mean squared error as in
``05/FFNN.py:95-106``, with pairs beyond zero_from - 0.2 weighted 20x so that
the fitted energy is close to zero where pairs cross the cutoff (a jump there
breaks energy conservation); forward by ``amlp_mlp_energy``, the
weighted output gradient formed in torch, weight gradient by
``amlp_mlp_backward``. Adam (lr 2e-3, cosine decay), batch 4,096, 120 epochs.
A held-out set of 16,384 pairs gives the fit error and the net's energy at the
cutoff (centre distances 2.45-2.55), written to ``model_<shape>_soft.json``.

Usage (needs a CUDA device): ``python tests/golden/make_soft_potential.py [cyl24|tetra16] [out.npz]``.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "anisotropic-ml_b200"))

EPS = 10.0
# per shape: hidden widths, point-point interaction range r_c, centre distance beyond which E_ij = 0
SHAPE_CFG = {
    "cyl24": dict(widths=(128, 128), rc=0.34, zero_from=2.494),
    "tetra16": dict(widths=(128, 128, 128), rc=0.5, zero_from=1.72),
}
RC = SHAPE_CFG["cyl24"]["rc"]
WIDTHS = SHAPE_CFG["cyl24"]["widths"]


def _rotate(q, p):
    """Rotate body-frame points p (n, 3) by unit quaternions q (P, 4), (w, x, y, z)."""
    w, u = q[:, None, :1], q[:, None, 1:]
    t = 2.0 * np.cross(u, p[None])
    return p[None] + w * t + np.cross(u, t)


def soft_energy(pts, d_vec, qi, qj, chunk=16384, rc=None):
    """Ground-truth pair energy in FP64 (formula in the module docstring)."""
    rc = RC if rc is None else rc
    out = np.empty(len(d_vec))
    pts = np.asarray(pts, np.float64)
    for s in range(0, len(d_vec), chunk):
        pi = _rotate(qi[s:s + chunk], pts)
        pj = _rotate(qj[s:s + chunk], pts) + d_vec[s:s + chunk, None, :]
        r = np.linalg.norm(pi[:, :, None, :] - pj[:, None, :, :], axis=-1)
        x = np.clip(1.0 - r / rc, 0.0, None)
        out[s:s + chunk] = EPS * (x ** 3).sum((1, 2))
    return out


def sample_pairs(n, seed, far_fraction=0.25, far_from=2.2):
    """Pair k = bodies (2k, 2k+1): 2k on a lattice of spacing 8, 2k+1 at a
    random centre distance in a random direction (distribution in the module
    docstring)."""
    from amlp.configs import random_quaternions
    rng = np.random.default_rng(seed)
    m = int(math.ceil(n ** (1.0 / 3.0) - 1e-9))
    L = float(np.float32(8.0 * m))
    grid = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3)[:n]
    a = grid * 8.0 - L / 2 + 4.0
    d = np.where(rng.random(n) < far_fraction, rng.uniform(far_from, 3.0, n), rng.uniform(0.4, 3.0, n))
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pos = np.empty((2 * n, 3), np.float32)
    pos[0::2], pos[1::2] = a, a + d[:, None] * u
    quat = random_quaternions(rng, 2 * n)
    pairs = np.stack([np.arange(0, 2 * n, 2), np.arange(1, 2 * n, 2)], 1).astype(np.int32)
    # labels from the float32 positions and orientations the descriptors see
    d_vec = pos[1::2].astype(np.float64) - pos[0::2].astype(np.float64)
    q64 = quat.astype(np.float64)
    return pos, quat, pairs, L, d, d_vec, q64[0::2], q64[1::2]


def main(shape_name: str, out_path: str) -> None:
    import ctypes

    import torch
    from amlp._lib import call
    from amlp.autograd import PairModel, mse_loss_grad, normalised_energies
    from amlp.engine import EnergyNet, Hypers
    from amlp.shapes import get_shape

    dev = torch.device("cuda:0")
    cfg = SHAPE_CFG[shape_name]
    widths = cfg["widths"]
    shape = get_shape(shape_name)
    model = PairModel(shape, Hypers(), [47, *widths, 1], "silu", dev)

    def dataset(n, seed):
        pos, quat, pairs, L, d, d_vec, qi, qj = sample_pairs(n, seed, far_from=cfg["zero_from"] - 0.3)
        E = soft_energy(shape.pts, d_vec, qi, qj, rc=cfg["rc"])
        g = model.descriptors(torch.tensor(pos, device=dev), torch.tensor(quat, device=dev),
                              torch.tensor(pairs, device=dev), L).clone()
        y = normalised_energies(torch.tensor(E), shape.en_min, shape.en_max).to(dev, torch.float32)
        return g, y, E, d

    g, y, E, d = dataset(262144, 0)
    gv, yv, Ev, dv = dataset(16384, 1)
    mu = g.mean(0)
    sd = g.std(0).clamp_min(1e-6)
    gs, gvs = ((g - mu) / sd).contiguous(), ((gv - mu) / sd).contiguous()

    net0 = EnergyNet.xavier(47, widths, "silu", seed=0, device="cpu")
    w = torch.cat([torch.cat([torch.tensor(W).reshape(-1), torch.tensor(b)]) for W, b in net0.layers]).to(dev)
    wt = torch.where(torch.tensor(d) > cfg["zero_from"] - 0.2, 20.0, 1.0).to(dev, torch.float32)
    opt = torch.optim.Adam([w], lr=2e-3)
    B, epochs = 4096, 120
    steps = epochs * (len(gs) // B)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, steps)
    gen = torch.Generator(device=dev).manual_seed(0)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.empty(B, dtype=torch.float32, device=dev)
    for ep in range(epochs):
        perm = torch.randperm(len(gs), device=dev, generator=gen)
        for k in range(len(gs) // B):
            idx = perm[k * B:(k + 1) * B]
            gb, yb, wb = gs[idx].contiguous(), y[idx], wt[idx]
            mlp = model.mlp(w)
            call("amlp_mlp_energy", gb.data_ptr(), B, ctypes.byref(mlp), out.data_ptr(), stream)
            dy = (2.0 * wb * (out - yb) / wb.sum()).contiguous()
            grad = torch.zeros_like(w)
            call("amlp_mlp_backward", gb.data_ptr(), dy.data_ptr(), B, ctypes.byref(mlp), grad.data_ptr(), stream)
            w.grad = grad
            opt.step()
            sched.step()
        if ep % 20 == 19 or ep == epochs - 1:
            tl, _ = mse_loss_grad(model, w, gs[:16384].contiguous(), y[:16384].contiguous())
            vl, _ = mse_loss_grad(model, w, gvs, yv)
            print(f"epoch {ep + 1}: train {tl.item():.3e} held-out {vl.item():.3e} (unweighted)", flush=True)

    # fold the standardisation into the first layer: W0 (g - mu)/sd + b0 = (W0/sd) g + (b0 - W0 mu/sd)
    dims = [47, *widths, 1]
    layers, off = [], 0
    for k in range(len(dims) - 1):
        n_w = dims[k + 1] * dims[k]
        W = w[off:off + n_w].reshape(dims[k + 1], dims[k]).double()
        b = w[off + n_w:off + n_w + dims[k + 1]].double()
        off += n_w + dims[k + 1]
        if k == 0:
            b = b - W @ (mu.double() / sd.double())
            W = W / sd.double()[None, :]
        layers.append((W.float().cpu().numpy(), b.float().cpu().numpy()))
    net = EnergyNet(layers, "silu", dev)
    e = torch.empty(len(gv), dtype=torch.float32, device=dev)
    call("amlp_mlp_energy", gv.data_ptr(), len(gv), ctypes.byref(net.struct), e.data_ptr(), stream)
    E_net = shape.en_min + (shape.en_max - shape.en_min) * e.double().cpu().numpy()
    Ecap = np.minimum(Ev, shape.en_max)
    rmse = float(np.sqrt(np.mean((E_net - Ecap) ** 2)))
    at_cut = (dv > 2.45) & (dv < 2.55)
    stats = dict(rmse=rmse, label_rms=float(np.sqrt(np.mean(Ecap ** 2))),
                 cutoff_mean=float(np.mean(E_net[at_cut])), cutoff_rms=float(np.sqrt(np.mean(E_net[at_cut] ** 2))),
                 cutoff_max=float(np.abs(E_net[at_cut]).max()))
    print(stats, flush=True)
    arrays = {}
    for k, (W, b) in enumerate(layers):
        arrays[f"W{k}"], arrays[f"b{k}"] = W, b
    np.savez(out_path, **arrays)
    with open(os.path.splitext(out_path)[0] + ".json", "w") as fh:
        json.dump(stats, fh, indent=1)


if __name__ == "__main__":
    name = sys.argv[1] if len(sys.argv) > 1 else "cyl24"
    main(name, sys.argv[2] if len(sys.argv) > 2 else os.path.join(HERE, f"model_{name}_soft.npz"))
