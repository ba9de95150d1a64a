"""Displacement-triggered Verlet rebuilds (``nlist_policy="displacement"``).

* hot bodies (kT 8, 2,000 cubes): after every segment the filtered pair list
  is exactly the one a fresh Verlet list gives (no pair is ever missing), and
  the trajectory equals that of rebuilding every step, within the rounding of
  the float atomics (1e-4 of the scale after 30 steps of a gentle net);
* cold bodies (kT 0.01): fewer rebuilds in 300 steps than the fixed 100-step
  schedule's two, and the same trajectory;
* a rebuild that overflows the list's capacity is detected and the segment
  reruns with a larger list (pairs exact afterwards).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import gpu_helpers as gh  # noqa: E402
from amlp.configs import make_state  # noqa: E402
from amlp.engine import EnergyNet, Hypers, System  # noqa: E402
from oracle.shapes import SHAPES  # noqa: E402

DEV = torch.device("cuda:0")


def _net():
    net = EnergyNet.xavier(47, (64, 64), "tanh", seed=4, device="cpu")
    return EnergyNet([(W * np.float32(0.1), b) for W, b in net.layers], "tanh", DEV)


def _system(kT, policy, every=100, n=2000, seed=21):
    st = make_state(n, "cube26", 0.45, kT=kT, seed=seed)
    return System(st, "cube26", Hypers(), _net(), kT=kT, dt=0.005, device=DEV, nve=True, nlist_every=every,
                  nlist_policy=policy)


def _fresh_filtered(s):
    pos = s.pos.cpu().numpy()
    vp, _ = gh.nlist(pos, s.L, s.r_verlet)
    return gh.pair_filter(pos, s.L, float(s.shape.cutoff), vp)


def test_hot_system_never_misses_a_pair():
    s = _system(8.0, "displacement")
    for _ in range(6):
        s.run(50, "adjoint")
        s._gated_rebuild()  # the list and filter the next step starts from
        s.compute_forces("adjoint")
        torch.cuda.synchronize()
        np.testing.assert_array_equal(s.filtered_pairs().astype(np.int64), _fresh_filtered(s))
    assert s.rebuilds >= 3
    # the fixed schedule misses pairs at this temperature (why the policy exists)
    f = _system(8.0, "every", every=100)
    missing = 0
    for _ in range(3):
        f.run(99, "adjoint")
        f.compute_forces("adjoint")
        torch.cuda.synchronize()
        missing += len(_fresh_filtered(f)) - len(f.filtered_pairs())
        f.run(1, "adjoint")
    assert missing > 0


def test_same_trajectory_as_rebuilding_every_step():
    a = _system(8.0, "displacement")
    b = _system(8.0, "every", every=1)
    a.run(30, "adjoint")
    b.run(30, "adjoint")
    torch.cuda.synchronize()
    for x, y in ((a.pos, b.pos), (a.vel, b.vel), (a.quat, b.quat)):
        x, y = x.cpu().numpy(), y.cpu().numpy()
        assert np.abs(x - y).max() <= 1e-4 * max(1.0, np.abs(y).max())


def test_cold_system_does_not_rebuild():
    """Over 300 steps the float atomics' summation order alone lets two runs of
    the same system drift apart; the displacement policy's trajectory may differ
    from the fixed schedule's by no more than 10x that drift (plus 1e-5 of the scale)."""
    a = _system(0.01, "displacement")
    b = _system(0.01, "every", every=100)
    c = _system(0.01, "every", every=100)
    for s in (a, b, c):
        s.run(300, "adjoint")
    torch.cuda.synchronize()
    assert a.rebuilds < 2
    x, y, z = (s.pos.cpu().numpy() for s in (a, b, c))
    floor = np.abs(z - y).max()
    assert np.abs(x - y).max() <= 10 * floor + 1e-5 * max(1.0, np.abs(y).max())


def test_overflowing_rebuild_reruns_with_a_larger_list():
    s = _system(1.0, "displacement", n=1500, seed=5)
    nv = int(s.nv.item())
    s._alloc_pairs(nv)
    s.build_nlist()
    cap0 = s.cap
    # crowd 60 bodies around body 1000: the next list has more pairs than fit
    pos = s.pos.cpu().numpy()
    rng = np.random.default_rng(0)
    pos[:60] = pos[1000] + rng.uniform(-0.4, 0.4, (60, 3)).astype(np.float32)
    L = s.L
    pos = (pos + L / 2) % L - L / 2
    s.pos.copy_(torch.tensor(pos, device=DEV))
    s.run(1, "adjoint")
    torch.cuda.synchronize()
    assert s.cap > cap0
    assert int(s.nl_gate[2].item()) == 0
    s.compute_forces("adjoint")
    torch.cuda.synchronize()
    np.testing.assert_array_equal(s.filtered_pairs().astype(np.int64), _fresh_filtered(s))
    assert np.isfinite(s.pos.cpu().numpy()).all()
    assert SHAPES["cube26"]["cutoff"] == 2.5
