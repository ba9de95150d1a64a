"""Differentiation: the adjoint force/torque kernels and the weight gradient.

* 65,536 regular tetrahedra (16 points) at packing fraction 0.40, seed 2, net
  47->128->128->128->1 SiLU: forces and torques of the adjoint path on 256
  randomly chosen bodies against FP64 central differences of the summed pair
  energy (step 1e-4): relative error (norm over the 256 bodies) <= 1e-3, both
  for the exact product (``amlp_pair_energy_vjp``, no clip) and for the force
  path of the simulation (``System.compute_forces('adjoint')``) on the bodies
  none of whose pairs reach the +-100 clip. Against the reference's own
  forces and torques (FP32 forward differences, dx = dteta = 1e-5) the
  adjoint's deviation from the FP64 central differences is at most twice the
  reference's at the 50/90/99 % quantiles (plus 0.05).
  The net is Xavier-initialised with its output layer scaled by 0.05, so that
  pair forces stay mostly below the clip (a trained potential's range); the
  unscaled random net drives most pair forces past +-100.
* 4,096 random pairs (centre distance uniform in [0.8, 2.5], random
  orientations), synthetic energy labels normalised like the reference's
  training data: the MSE-loss weight gradient of ``amlp_mlp_loss_grad`` against
  torch FP64 autograd on the same descriptors (relative 1e-5), and the weight
  gradient through ``PairEnergy`` (descriptors recomputed on the GPU) against
  torch FP64 autograd on FP64 descriptors (relative 1e-4); position and
  orientation gradients through ``PairEnergy`` equal the exact FP64 forces and
  torques (relative 1e-3); a few Adam steps lower the loss.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from amlp import _lib  # noqa: E402
from amlp.autograd import (PairModel, mse_loss_grad, normalised_energies, pair_energies,  # noqa: E402
                           torque_from_quat_grad)
from amlp.configs import make_state, random_quaternions  # noqa: E402
from amlp.engine import EnergyNet, Hypers, System  # noqa: E402
from oracle import adjoint, nep  # noqa: E402
from oracle.shapes import SHAPES  # noqa: E402

DEV = torch.device("cuda:0")
WIDTHS = (128, 128, 128)


def _net(seed, out_scale=0.05):
    net = EnergyNet.xavier(47, WIDTHS, "silu", seed=seed, device="cpu")
    layers = list(net.layers)
    W, b = layers[-1]
    layers[-1] = (W * np.float32(out_scale), b)
    return EnergyNet(layers, "silu", DEV)


def _rel(got, want):
    return float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30))


# ----------------------------------------------------------------------------- 65,536 tetrahedra
@pytest.fixture(scope="module")
def tetra_system():
    st = make_state(65536, "tetra16", 0.40, seed=2)
    net = _net(seed=2)
    s = System(st, "tetra16", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    s.compute_forces("adjoint")
    torch.cuda.synchronize()
    assert _lib.device_error() == 0
    F, T = s.F.cpu().numpy().astype(np.float64), s.T.cpu().numpy().astype(np.float64)
    P = int(s.nf.item())
    pairs_dev = s.fpairs[:P].contiguous()
    pairs = pairs_dev.cpu().numpy().astype(np.int64)
    bodies = np.sort(np.random.default_rng(2024).choice(st.N, 256, replace=False))
    sub = pairs[np.isin(pairs[:, 0], bodies) | np.isin(pairs[:, 1], bodies)]
    shape = SHAPES["tetra16"]
    cdF, cdT = adjoint.central_difference_forces(st.pos, st.orient, sub, st.L, shape, (10, 8, 4), net.layers,
                                                 "silu", bodies, h=1e-4)
    return dict(st=st, s=s, net=net, F=F, T=T, pairs_dev=pairs_dev, sub=sub, bodies=bodies, cdF=cdF, cdT=cdT,
                shape=shape)


def test_tetra_pair_count_is_the_configuration(tetra_system):
    P = len(tetra_system["pairs_dev"])
    # about 110 partners per body within 2.5 at this density
    assert 5_000_000 < P < 10_000_000


def test_exact_product_vs_central_differences(tetra_system):
    ts = tetra_system
    s = ts["s"]
    model = PairModel("tetra16", Hypers(), s.net.dims, "silu", DEV)
    pos = s.pos.clone().requires_grad_()
    quat = s.quat.clone().requires_grad_()
    E = pair_energies(pos, quat, s.net.d_w, ts["pairs_dev"], s.L, model, clip=False)
    gp, gq = torch.autograd.grad(E.sum(), (pos, quat))
    b = torch.as_tensor(ts["bodies"], device=DEV)
    F = (-gp[b]).double().cpu().numpy()
    T = torque_from_quat_grad(s.quat[b].double(), gq[b].double()).cpu().numpy()
    assert _rel(F, ts["cdF"]) <= 1e-3, _rel(F, ts["cdF"])
    assert _rel(T, ts["cdT"]) <= 1e-3, _rel(T, ts["cdT"])
    ts["F_noclip"], ts["T_noclip"] = F, T


def test_force_path_vs_central_differences(tetra_system):
    ts = tetra_system
    if "F_noclip" not in ts:
        test_exact_product_vs_central_differences(ts)
    bodies = ts["bodies"]
    F, T = ts["F"][bodies], ts["T"][bodies]
    # bodies whose pairs all stay inside the clip: clipped and exact products agree
    same = (np.abs(F - ts["F_noclip"]).max(1) <= 1e-4 * (1 + np.abs(F).max(1))) & \
           (np.abs(T - ts["T_noclip"]).max(1) <= 1e-4 * (1 + np.abs(T).max(1)))
    assert same.sum() >= 200, same.sum()
    assert _rel(F[same], ts["cdF"][same]) <= 1e-3
    assert _rel(T[same], ts["cdT"][same]) <= 1e-3


def test_adjoint_vs_reference_forward_differences(tetra_system):
    """The reference's FP32 forward differences on the same bodies (all their
    pairs): the adjoint is closer to the FP64 truth at every quantile."""
    ts = tetra_system
    st, sub, bodies = ts["st"], ts["sub"], ts["bodies"]
    o = nep.pair_forces(st.pos, st.orient, sub, st.L, ts["shape"], (10, 8, 4), ts["net"].layers, "silu")
    refF, refT = o["forces"][bodies].astype(np.float64), o["torques"][bodies].astype(np.float64)
    for got, ref, cd in ((ts["F"][bodies], refF, ts["cdF"]), (ts["T"][bodies], refT, ts["cdT"])):
        e_gpu, e_ref = np.abs(got - cd), np.abs(ref - cd)
        for q in (0.5, 0.9, 0.99):
            assert np.quantile(e_gpu, q) <= 2 * np.quantile(e_ref, q) + 0.05, q


# ----------------------------------------------------------------------------- 4,096 random pairs
def _random_pairs(n_pairs=4096, seed=5):
    """Bodies 2k, 2k+1 form pair k: 2k on a lattice of spacing 8 (no other body
    within the cutoff), 2k+1 at a uniform distance in [0.8, 2.5] in a random
    direction; all orientations uniform random."""
    rng = np.random.default_rng(seed)
    m = int(np.ceil(n_pairs ** (1 / 3)))
    L = float(np.float32(8.0 * m))
    grid = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3)[:n_pairs]
    a = grid * 8.0 - L / 2 + 4.0
    d = rng.uniform(0.8, 2.5, n_pairs)
    u = rng.normal(size=(n_pairs, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pos = np.empty((2 * n_pairs, 3), np.float32)
    pos[0::2], pos[1::2] = a, a + d[:, None] * u
    quat = random_quaternions(rng, 2 * n_pairs)
    pairs = np.stack([np.arange(0, 2 * n_pairs, 2), np.arange(1, 2 * n_pairs, 2)], 1)
    # synthetic labels: a repulsive core and a shallow well in the centre distance, with noise
    E = 12.0 * np.exp(-4.0 * (d - 0.8)) - 3.0 * np.exp(-((d - 1.6) / 0.4) ** 2) + 0.2 * rng.normal(size=n_pairs)
    return pos, quat, pairs, L, E


def _fp64_net_grad(layers, g64, y64, act="silu"):
    params = []
    for W, b in layers:
        params += [torch.tensor(W, dtype=torch.float64, requires_grad=True),
                   torch.tensor(b, dtype=torch.float64, requires_grad=True)]
    h = g64
    for k in range(len(layers)):
        h = torch.nn.functional.linear(h, params[2 * k], params[2 * k + 1])
        if k < len(layers) - 1:
            h = torch.nn.functional.silu(h)
    loss = torch.mean((h[:, 0] - y64) ** 2)
    loss.backward()
    packed = torch.cat([torch.cat([params[2 * k].grad.reshape(-1), params[2 * k + 1].grad]) for k in range(len(layers))])
    return float(loss.detach()), packed.numpy()


@pytest.fixture(scope="module")
def pair_batch():
    pos, quat, pairs, L, E = _random_pairs()
    shape = SHAPES["tetra16"]
    net = _net(seed=7, out_scale=1.0)
    model = PairModel("tetra16", Hypers(), net.dims, "silu", DEV)
    y = normalised_energies(torch.tensor(E), shape["en_min"], shape["en_max"]).numpy()
    return dict(pos=pos, quat=quat, pairs=pairs, L=L, E=E, y=y, net=net, model=model, shape=shape)


def _dev(b):
    return (torch.tensor(b["pos"], device=DEV), torch.tensor(b["quat"], device=DEV),
            torch.tensor(b["pairs"].astype(np.int32), device=DEV).contiguous())


def test_loss_grad_kernel_vs_fp64_autograd_same_descriptors(pair_batch):
    b = pair_batch
    pos, quat, pairs = _dev(b)
    g = b["model"].descriptors(pos, quat, pairs, b["L"])
    y = torch.tensor(b["y"], dtype=torch.float32, device=DEV)
    loss, grad = mse_loss_grad(b["model"], b["net"].d_w, g, y)
    loss64, grad64 = _fp64_net_grad(b["net"].layers, g.double().cpu(), torch.tensor(b["y"], dtype=torch.float64))
    assert abs(float(loss.item()) - loss64) <= 1e-5 * abs(loss64)
    got = grad.cpu().numpy().astype(np.float64)
    assert _rel(got, grad64) <= 1e-5, _rel(got, grad64)


def test_weight_gradient_through_pair_energy_vs_fp64(pair_batch):
    b = pair_batch
    pos, quat, pairs = _dev(b)
    model = b["model"]
    w = b["net"].d_w.clone().requires_grad_()
    E = pair_energies(pos, quat, w, pairs, b["L"], model)
    y = torch.tensor(b["y"], dtype=torch.float32, device=DEV)
    loss = torch.mean(((E - model.en_min) / model.en_range - y) ** 2)
    loss.backward()
    # FP64 oracle: descriptors of the FP64 pair clouds, FP64 net
    shape = b["shape"]
    _, _, t = nep.min_image_filter(b["pos"], b["pairs"], b["L"], 1e30, np.float64)
    c1, _ = nep.pair_clouds(b["quat"], b["pairs"], t, shape["pts"], np.float64)
    g64 = adjoint.descriptor_torch(torch.tensor(c1), 10, 8, 4, float(shape["nep_cutoff"]))
    y64 = (torch.tensor(b["y"], dtype=torch.float64))
    loss64, grad64 = _fp64_net_grad(b["net"].layers, g64, y64)
    e64 = shape["en_min"] + (shape["en_max"] - shape["en_min"]) * adjoint.pair_energy_net(g64, b["net"].layers,
                                                                                           "silu").detach().numpy()
    assert np.abs(E.detach().cpu().numpy() - e64).max() <= 1e-4 * max(1.0, np.abs(e64).max())
    assert abs(float(loss) - loss64) <= 1e-4 * abs(loss64)
    got = w.grad.cpu().numpy().astype(np.float64)
    assert _rel(got, grad64) <= 1e-4, _rel(got, grad64)


def test_position_and_orientation_gradients_are_exact_forces(pair_batch):
    b = pair_batch
    pos, quat, pairs = _dev(b)
    pos.requires_grad_()
    quat.requires_grad_()
    E = pair_energies(pos, quat, b["net"].d_w, pairs, b["L"], b["model"], clip=False)
    gp, gq = torch.autograd.grad(E.sum(), (pos, quat))
    ref = adjoint.exact_pair_forces(b["pos"], b["quat"], b["pairs"], b["L"], b["shape"], (10, 8, 4),
                                    b["net"].layers, "silu", clip=False)
    F = -gp.double().cpu().numpy()
    T = torque_from_quat_grad(quat.detach().double(), gq.double()).cpu().numpy()
    assert _rel(F, ref["forces"]) <= 1e-3
    assert _rel(T, ref["torques"]) <= 1e-3


def test_clipped_product_is_the_force_path(pair_batch):
    """With clip and a unit upstream gradient the product equals the adjoint
    force kernel's output (same kernels)."""
    import gpu_helpers as gh
    b = pair_batch
    pos, quat, pairs = _dev(b)
    pos.requires_grad_()
    E = pair_energies(pos, quat, b["net"].d_w, pairs, b["L"], b["model"], clip=True)
    (gp,) = torch.autograd.grad(E.sum(), (pos,))
    F, T, pe = gh.fused_forces(b["pos"], b["quat"], b["L"], b["pairs"], b["shape"], (10, 8, 4), b["net"].layers,
                               "silu", method="amlp_forces_adjoint_wide")
    np.testing.assert_allclose(-gp.cpu().numpy(), F, rtol=1e-6, atol=1e-6)
    assert abs(float(E.sum()) - pe) <= 1e-5 * max(1.0, np.abs(E.detach().cpu().numpy()).sum())


def test_adam_steps_lower_the_loss(pair_batch):
    b = pair_batch
    model = b["model"]
    pos, quat, pairs = _dev(b)
    g = model.descriptors(pos, quat, pairs, b["L"])
    y = torch.tensor(b["y"], dtype=torch.float32, device=DEV)
    w = b["net"].d_w.clone()
    opt = torch.optim.Adam([w], lr=1e-3)
    losses = []
    for _ in range(30):
        loss, grad = mse_loss_grad(model, w, g, y)
        losses.append(float(loss.item()))
        w.grad = grad
        opt.step()
    assert losses[-1] < 0.5 * losses[0], losses[::10]
