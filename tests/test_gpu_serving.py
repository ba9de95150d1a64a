"""Serving: many independent systems packed into multi-system launches.

* each system's result is the same alone (amlp.engine.System) and in the mix
  (amlp.serving.Server), within the rounding of the float atomics that sum
  forces: after one step positions, velocities and quaternions agree to 2e-6 of
  their scale (random Xavier nets, forces up to the +-100 clip); after 20 steps
  with a gentler net (weights x 0.05, so the dynamics do not amplify the
  rounding) positions and velocities agree to 1e-4;
* admission respects the HBM budget (first come, first served), every request
  completes.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from amlp.engine import EnergyNet, Hypers, System  # noqa: E402
from amlp.serving import Request, Server, request_stream, system_bytes  # noqa: E402
from amlp.shapes import get_shape  # noqa: E402
from amlp.configs import make_state  # noqa: E402

DEV = torch.device("cuda:0")


def _nets(scale=1.0):
    out = {}
    for k, name in enumerate(("cube26", "tetra16", "cyl24")):
        net = EnergyNet.xavier(47, (64, 64), "tanh", seed=k + 3, device="cpu")
        out[name] = EnergyNet([(W * scale, b) for W, b in net.layers], "tanh", DEV)
    return out


def _alone(req, net, steps):
    st = make_state(req.n, req.shape, req.phi, kT=req.kT, seed=req.seed)
    s = System(st, req.shape, Hypers(), net, kT=req.kT, dt=0.005, device=DEV, initial_ke_quirk=False)
    for _ in range(steps):
        s.step("adjoint")
    torch.cuda.synchronize()
    return s


def _mix():
    return [Request(0, 1500, "cube26", 0.40, 1.0, 0, 0.0, seed=11),
            Request(1, 800, "tetra16", 0.35, 0.7, 0, 0.0, seed=12),
            Request(2, 2500, "cyl24", 0.30, 1.5, 0, 0.0, seed=13),
            Request(3, 1200, "cube26", 0.30, 2.0, 0, 0.0, seed=14)]


@pytest.mark.parametrize("steps", [1, 20])
def test_each_result_same_alone_and_in_the_mix(steps):
    nets = _nets(scale=1.0 if steps == 1 else 0.05)
    reqs = _mix()
    for r in reqs:
        r.steps = steps
    srv = Server(nets, hbm_budget=8 << 30, segment=steps, device=DEV)
    stats = srv.run(reqs, keep_states=True)
    assert stats.summary()["requests"] == 4 and stats.max_active == 4
    for r in reqs:
        alone = _alone(r, nets[r.shape], steps)
        mixed = srv.results[r.rid]
        if steps == 1:
            for got, ref in ((mixed.pos, alone.pos), (mixed.vel, alone.vel), (mixed.orient, alone.quat),
                             (mixed.angmom, alone.angmom)):
                ref = ref.cpu().numpy()
                assert np.abs(got - ref).max() <= 2e-6 * max(1.0, np.abs(ref).max()), r.rid
        else:
            for got, ref in ((mixed.pos, alone.pos), (mixed.vel, alone.vel)):
                ref = ref.cpu().numpy()
                assert np.abs(got - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max()), r.rid


def test_admission_respects_budget():
    nets = _nets()
    reqs = [Request(k, 2000, "cube26", 0.35, 1.0, 10, 0.0, seed=20 + k) for k in range(4)]
    one = system_bytes(2000, get_shape("cube26"), 0.35)
    srv = Server(nets, hbm_budget=int(2.5 * one), segment=10, device=DEV)
    stats = srv.run(reqs)
    s = stats.summary()
    assert s["requests"] == 4 and stats.max_active == 2
    assert srv.used == 0


def test_stream_runs_and_reports():
    nets = _nets()
    reqs = request_stream(8, seed=5, steps=30, rate=200.0, n_range=(500, 5000))
    srv = Server(nets, hbm_budget=4 << 30, segment=10, device=DEV)
    s = srv.run(reqs).summary()
    assert s["requests"] == 8 and s["particle_steps"] == sum(r.n * 30 for r in reqs)
    assert s["segment_ms_p99"] >= s["segment_ms_p50"] > 0


def test_wide_nets_same_alone_and_in_the_mix():
    """Served systems whose nets are wider than the fused kernel takes (128 x 2
    SiLU, the precision workload's size) run on the multi-system wide path
    (amlp_multi_forces_adjoint_wide, harmonic-form descriptor passes); each
    result equals the system run alone through System.step within the rounding
    of the force atomics, after one step."""
    nets = {}
    for k, name in enumerate(("cube26", "tetra16", "cyl24")):
        net = EnergyNet.xavier(47, (128, 128), "silu", seed=k + 30, device="cpu")
        nets[name] = EnergyNet(net.layers, "silu", DEV)
    reqs = _mix()
    for r in reqs:
        r.steps = 1
    srv = Server(nets, hbm_budget=8 << 30, segment=1, device=DEV)
    srv.run(reqs, keep_states=True)
    assert all(b.adj_ws is not None for b in srv.buckets.values())  # the wide path
    for r in reqs:
        alone = _alone(r, nets[r.shape], 1)
        mixed = srv.results[r.rid]
        for got, ref in ((mixed.pos, alone.pos), (mixed.vel, alone.vel), (mixed.orient, alone.quat),
                         (mixed.angmom, alone.angmom)):
            ref = ref.cpu().numpy()
            assert np.abs(got - ref).max() <= 2e-6 * max(1.0, np.abs(ref).max()), r.rid
