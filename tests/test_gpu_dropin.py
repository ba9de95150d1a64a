"""The drop-in ``nep_simulator`` classes (``NVT``/``Sim``, ``DescriptorGenerator``,
``ForceEvaluator``, ``sim_input``) on the reference's own case: 200 ``th_v1``
bodies from ``init/th_init_N200.gsd``, ``model_th_C104`` (47 -> 150 x 3 -> 1
ReLU), hypers 10 8 4 4.5, kT 0.5, dt 0.005, driven through the reference's
builder calls (``sim_input.py:50-61``) from a GSD file and a ``.pth`` state
dict written here from the fixtures.

* ``generate_nep_descriptors`` returns the reference's filtered pairs (as a
  set: the Verlet list is in (i, j) order here, in cKDTree order there), P, and
  the reference's descriptor rows for them (5e-5 of their scale);
  ``evaluate_interactions`` gives forces and torques whose deviation from the
  FP64 finite differences is within twice the reference's own at the
  50/90/99 % quantiles (plus 0.05);
* one step through ``run``: thermostat variables equal the reference's (FP32,
  1e-6 relative), positions and velocities differ from the reference's by no
  more than the step-0 force differences can move them (dt^2 |dF| / m and
  dt |dF| / m);
* the command line writes frames 0, 100 and 200 for a 205-step run (frame 0 is
  the initial state, bit for bit), stores the thermostat state in each frame,
  and a run resumed from the last frame continues with that thermostat state;
* ``--method adjoint`` through the same command line runs the adjoint kernels.
"""
import os
import sys

import numpy as np
import pytest
import torch

from conftest import GOLDEN, PKG, load_case, load_model

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

NS = os.path.join(PKG, "nep_simulator")
if NS not in sys.path:
    sys.path.insert(0, NS)

from amlp.gsd import Frame, GsdFile, read_last_frame  # noqa: E402
from oracle import nep  # noqa: E402
from oracle.shapes import SHAPES  # noqa: E402

HYPERS = ["10", "8", "4", "4.5"]


def _write_init(path):
    z = np.load(os.path.join(GOLDEN, "init_th_init_N200.npz"))
    f = Frame()
    f.step, f.N, f.box, f.types = int(z["step"]), 200, z["box"], ["A", "B"]
    for k in ("position", "orientation", "velocity", "angmom", "moment_inertia", "body", "image"):
        f.particles[k] = z[k]
    with GsdFile(path, "w") as g:
        g.append(f)


def _state_dict(layers):
    names = ["layer_first"] + [f"layer_hidden.{k}" for k in range(len(layers) - 2)] + ["layer_last"]
    sd = {}
    for n, (W, b) in zip(names, layers):
        sd[n + ".weight"] = torch.tensor(W)
        sd[n + ".bias"] = torch.tensor(b)
    return sd


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("dropin")
    init = str(d / "th_init_N200.gsd")
    _write_init(init)
    pth = str(d / "model_th_C104.pth")
    torch.save(_state_dict(load_model("th_C104")), pth)
    net = [(np.asarray(W) * np.float32(0.2), np.asarray(b)) for W, b in _xavier_64()]
    pth64 = str(d / "model_tanh64.pth")
    torch.save(_state_dict(net), pth64)
    return dict(dir=d, init=init, pth=pth, pth64=pth64)


def _xavier_64():
    from amlp.engine import EnergyNet
    return EnergyNet.xavier(47, (64, 64), "tanh", seed=3, device="cpu").layers


def _builder(files, dump=None, out=None, **kw):
    from NVT import NVT
    sim = NVT()
    sim.setDevice(0)
    if "method" in kw:
        sim.setForceMethod(kw["method"])
    sim.initializeSystem(files["init"])
    sim.setNepDescriptors([float(h) for h in HYPERS])
    sim.setEvaluator(files["pth"])
    sim.setShape("th_v1")
    sim.setNeighborList()
    if dump:
        sim.setGsdDump(dump, out)
    sim.setkT(0.5)
    sim.setdt(0.005)
    return sim


def test_descriptors_and_forces_through_the_dropin_classes(files):
    c = load_case("th_C104")
    sim = _builder(files)
    sim.move_data_to_device()
    s = sim.system
    g, pp, P = sim.descriptor_generator.generate_nep_descriptors(s.pos, s.quat, sim.Nlist)
    torch.cuda.synchronize()
    assert int(P) == int(c["P0"])
    got = pp.cpu().numpy().astype(np.int64)
    want = c["pairs0"]
    key = lambda a: a[:, 0] * 1_000_000 + a[:, 1]  # noqa: E731
    assert np.array_equal(np.sort(key(got)), np.sort(key(want)))
    g = g.cpu().numpy().reshape(10, int(P), -1)
    pos_of = {int(k): n for n, k in enumerate(key(got))}
    idx = np.array([pos_of[int(k)] for k in key(want[: c["g0"].shape[1]])])
    ref = c["g0"]
    assert np.abs(g[:, idx] - ref).max() <= 5e-5 * max(1.0, np.abs(ref).max())
    F, T = sim.evaluator.evaluate_interactions(sim.descriptor_generator.g_all, pp, P)
    F, T = F.cpu().numpy(), T.cpu().numpy()
    shape = SHAPES["th_v1"]
    o64 = nep.pair_forces(c["pos0"], c["orient0"], c["pairs0"], c["L"], shape, (10, 8, 4), load_model("th_C104"),
                          "relu", dt=np.float64)
    for got_f, ref_f, exact in ((F, c["F0"], o64["forces"]), (T, c["T0"], o64["torques"])):
        e_gpu, e_ref = np.abs(got_f - exact), np.abs(ref_f - exact)
        for q in (0.5, 0.9, 0.99):
            assert np.quantile(e_gpu, q) <= 2 * np.quantile(e_ref, q) + 0.05, q
    files["F0"], files["T0"] = F, T


def test_one_step_matches_the_reference(files):
    c = load_case("th_C104")
    if "F0" not in files:
        test_descriptors_and_forces_through_the_dropin_classes(files)
    sim = _builder(files)
    sim.run(1)
    s = sim.system
    th = s.thermostat()
    got_th = np.array([th["xi"], th["eta"], th["xi_rot"], th["eta_rot"], th["thermo_fac"]], np.float64)
    np.testing.assert_allclose(got_th, c["thermo_s1"], rtol=1e-6, atol=1e-9)
    dF = np.abs(files["F0"] - c["F0"]).max()
    dt = 0.005
    pos = s.pos.cpu().numpy()
    vel = s.vel.cpu().numpy()
    assert np.abs(pos - c["pos_s1"]).max() <= 1.1 * dt * dt * dF + 1e-5
    assert np.abs(vel - c["vel_s1"]).max() <= 1.1 * dt * dF + 1e-5
    q = s.quat.cpu().numpy()
    assert np.abs(np.linalg.norm(q, axis=1) - 1).max() < 1e-5


def test_command_line_run_dumps_and_resume(files, monkeypatch):
    import sim_input
    c = load_case("th_C104")
    monkeypatch.chdir(files["dir"])
    args = ["--init", files["init"], "--out", "t205", "--ts", "205", "--dump", "100", "--kT", "0.5", "--dt", "0.005",
            "--hypers_nep", *HYPERS, "--model_path", files["pth"], "--gpu_id", "0", "--shape", "th_v1"]
    sim = sim_input.main(args)
    out = os.path.join(files["dir"], "out", "t205.gsd")
    with GsdFile(out) as g:
        steps = [g[i].step for i in range(len(g))]
        assert steps == list(c["long_frames_step"])
        np.testing.assert_array_equal(g[0].particles["position"], c["long_frames_pos"][0])
        for i in range(len(g)):
            assert "thermostat/integrator_vars" in g[i].log
        last = g[len(g) - 1]
    L = float(c["L"])
    assert np.isfinite(last.particles["position"]).all()
    assert np.abs(last.particles["position"]).max() <= L / 2 + 1e-4
    assert sim.timestep == 205
    # resume: the thermostat of the last frame is restored, not re-seeded
    from NVT import NVT
    r = NVT()
    r.setDevice(0)
    r.initializeSystem(out)
    r.setNepDescriptors([float(h) for h in HYPERS])
    r.setEvaluator(files["pth"])
    r.setShape("th_v1")
    r.setNeighborList()
    r.setkT(0.5)
    r.setdt(0.005)
    r.move_data_to_device()
    th = r.system.thermostat()
    want = last.log["thermostat/integrator_vars"]
    np.testing.assert_array_equal(np.array([th["xi"], th["eta"], th["xi_rot"], th["eta_rot"]], np.float32), want)
    r.run(3)
    assert np.isfinite(r.system.pos.cpu().numpy()).all()


def test_command_line_adjoint_method(files, monkeypatch):
    import sim_input
    from amlp.engine import EnergyNet, Hypers, System
    from amlp.configs import State
    monkeypatch.chdir(files["dir"])
    args = ["--init", files["init"], "--out", "adj", "--ts", "10", "--dump", "100", "--kT", "0.5", "--dt", "0.005",
            "--hypers_nep", *HYPERS, "--model_path", files["pth64"], "--gpu_id", "0", "--shape", "th_v1",
            "--method", "adjoint", "--activation", "tanh", "--nn_width", "64", "--nn_hidden", "1"]
    sim = sim_input.main(args)
    # the same run straight on the engine
    z = np.load(os.path.join(GOLDEN, "init_th_init_N200.npz"))
    st = State(pos=z["position"], orient=z["orientation"], vel=z["velocity"], angmom=z["angmom"],
               mass=np.ones(200, np.float32), moi=z["moment_inertia"][0], L=float(np.float32(z["box"][0])))
    net = EnergyNet.from_state_dict(torch.load(files["pth64"]), "tanh", "cuda:0")
    e = System(st, "th_v1", Hypers(10, 8, 4), net, kT=0.5, dt=0.005, device="cuda:0", initial_ke_quirk=True,
               moi=z["moment_inertia"][0])
    e.run(10, "adjoint")
    torch.cuda.synchronize()
    a, b = sim.system.pos.cpu().numpy(), e.pos.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-4, np.abs(a - b).max()
    assert read_last_frame(os.path.join(files["dir"], "out", "adj.gsd")).step == 0


def test_reference_model_on_the_tensor_core_adjoint(files):
    """The reference's own 150-wide model (model_th_C104, four ReLU layers)
    through the drop-in classes with the adjoint method runs on the tensor-core
    wide path; its forces are checked against FP64 in test_gpu_parity."""
    from amlp import _lib
    sim = _builder(files, method="adjoint")
    sim.run(5)
    torch.cuda.synchronize()
    assert sim.system.adj_ws is not None
    assert np.isfinite(sim.system.pos.cpu().numpy()).all()
    assert _lib.device_error() == 0
