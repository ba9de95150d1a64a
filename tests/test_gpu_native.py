"""The C ABI's own runtimes: the simulation handle (``amlp_sim``) and the
serving pool (``amlp_pool``), through ``amlp.native``.

* handle vs ``engine.System`` on the same state (cube26, 400 bodies): the
  Verlet list, filtered pairs and descriptors are identical (no atomics); the
  forces of both methods agree to float-atomics rounding (1e-5 of the scale);
  150 adjoint steps (a rebuild at step 100, graphs on both sides) end on the
  same trajectory within 1e-3 and the same thermostat within 1e-4;
* handle vs the FP64 oracle on the reference's descriptor layout (descriptors
  of the filtered pairs, 5e-5 of their scale);
* pool vs one handle per system: two systems (different sizes and kT) stepped
  20 steps in one pool match their handles within 1e-4; a system admitted
  later is pending until the next segment and then active; a capacity far too
  small for a system's Verlet list grows without changing the result; an
  evicted system returns its state and thermostat and the pool keeps stepping;
* errors: calls out of order, bad arguments and unknown modes return a status
  and leave a message in ``amlp_last_error`` / ``amlp_pool_last_error``.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from amlp import _lib  # noqa: E402
from amlp._lib import AmlpError, Nep, call  # noqa: E402
from amlp.configs import make_state  # noqa: E402
from amlp.engine import EnergyNet, Hypers, System  # noqa: E402
from amlp.native import NativePool, NativeSystem  # noqa: E402
from oracle import nep as onep  # noqa: E402
from oracle.shapes import SHAPES  # noqa: E402

DEV = torch.device("cuda:0")


def _net(act="tanh", widths=(64, 64), seed=4, scale=0.1):
    net = EnergyNet.xavier(47, widths, act, seed=seed, device="cpu")
    return EnergyNet([(W * np.float32(scale), b) for W, b in net.layers], act, DEV)


@pytest.fixture(scope="module")
def pair():
    st = make_state(400, "cube26", 0.30, kT=1.0, seed=7)
    net = _net()
    eng = System(st, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    nat = NativeSystem(st, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    return st, net, eng, nat


def test_descriptors_and_pairs_identical(pair):
    st, net, eng, nat = pair
    g, pairs, P = nat.descriptors(cap=200000)
    eng.filter_pairs()
    torch.cuda.synchronize()
    assert P == int(eng.nf.item()) > 0
    np.testing.assert_array_equal(pairs.cpu().numpy(), eng.filtered_pairs())
    g_e = torch.empty(10 * P, 47, dtype=torch.float32, device=DEV)
    call("amlp_descriptors", eng.pos.data_ptr(), eng.quat.data_ptr(), eng.L, eng.fpairs.data_ptr(), P,
         ctypes.byref(eng.nep), g_e.data_ptr(), torch.cuda.current_stream().cuda_stream)
    np.testing.assert_array_equal(g.cpu().numpy(), g_e.cpu().numpy())
    # the reference's descriptor rows (variant 0) from the FP64 oracle
    shape = SHAPES["cube26"]
    o = onep.pair_forces(st.pos, st.orient, pairs.cpu().numpy().astype(np.int64), st.L, shape, (10, 8, 4),
                         net.layers, "tanh", dt=np.float64, form="sh")
    ref = o["g_all"][:P]
    got = g.cpu().numpy()[:P]
    assert np.abs(got - ref).max() <= 5e-5 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("method", ["fd", "adjoint"])
def test_forces_match_engine(pair, method):
    st, net, eng, nat = pair
    F, T = nat.forces(method)
    eng.compute_forces(method)
    torch.cuda.synchronize()
    for a, b in ((F, eng.F), (T, eng.T)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-5 * max(1.0, np.abs(b).max())
    assert abs(nat.thermostat()["pe"] - eng.thermostat()["pe"]) <= 1e-6 * max(1.0, abs(eng.thermostat()["pe"]))


def test_run_matches_engine_across_a_rebuild():
    st = make_state(400, "cube26", 0.30, kT=1.0, seed=8)
    net = _net(seed=5)
    eng = System(st, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    nat = NativeSystem(st, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    eng.run(150, "adjoint")
    nat.run(150, "adjoint")
    torch.cuda.synchronize()
    assert nat.timestep == 150
    s = nat.state()
    for k, ref in (("pos", eng.pos), ("quat", eng.quat), ("vel", eng.vel), ("angmom", eng.angmom)):
        a, b = s[k].cpu().numpy(), ref.cpu().numpy()
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= 1e-3 * max(1.0, np.abs(b).max()), k
    ta, tb = nat.thermostat(), eng.thermostat()
    for k in ("xi", "eta", "xi_rot", "eta_rot"):
        assert abs(ta[k] - tb[k]) <= 1e-4 * max(1.0, abs(tb[k])), k
    nat.close()


def _pool_states():
    a = make_state(300, "cube26", 0.30, kT=1.0, seed=11)
    b = make_state(500, "cube26", 0.35, kT=0.5, seed=12)
    c = make_state(250, "cube26", 0.25, kT=1.5, seed=13)
    return a, b, c


def test_pool_matches_handles_and_admits_and_evicts():
    net = _net(seed=6)
    a, b, c = _pool_states()
    pool = NativePool("cube26", Hypers(), net, dt=0.005)
    ia = pool.admit(a, kT=1.0)
    ib = pool.admit(b, kT=0.5)
    assert pool.status(ia)["status"] == _lib.POOL_PENDING
    pool.step_segment(20)
    assert pool.status(ia)["status"] == _lib.POOL_ACTIVE and pool.status(ia)["steps_done"] == 20
    ref = {}
    for rid, st, kT in ((ia, a, 1.0), (ib, b, 0.5)):
        h = NativeSystem(st, "cube26", Hypers(), net, kT=kT, dt=0.005, device=DEV)
        h.run(20, "adjoint")
        ref[rid] = {k: v.cpu().numpy() for k, v in h.state().items()}
        ref[rid]["th"] = h.thermostat()
        h.close()
    ic = pool.admit(c, kT=1.5)
    assert len(pool) == 3
    pool.step_segment(10)
    assert pool.status(ic)["steps_done"] == 10 and pool.status(ia)["steps_done"] == 30
    out = pool.evict(ib)
    assert len(pool) == 2
    assert np.isfinite(out["pos"]).all() and np.isfinite(out["vel"]).all()
    pool.step_segment(5)
    assert pool.status(ia)["steps_done"] == 35
    # the first segment again in a fresh pool, with a Verlet capacity for b far
    # too small (it grows at the segment's first rebuild), against the handles
    pool2 = NativePool("cube26", Hypers(), net, dt=0.005)
    ja, jb = pool2.admit(a, kT=1.0), pool2.admit(b, kT=0.5, verlet_cap=512)
    pool2.step_segment(20)
    for rid, jid in ((ia, ja), (ib, jb)):
        got = pool2.evict(jid)
        for k in ("pos", "quat", "vel", "angmom"):
            assert np.abs(got[k] - ref[rid][k]).max() <= 1e-4 * max(1.0, np.abs(ref[rid][k]).max()), k
        for k in ("xi", "eta", "xi_rot", "eta_rot"):
            assert abs(got["thermostat"][k] - ref[rid]["th"][k]) <= 1e-4 * max(1.0, abs(ref[rid]["th"][k])), k
    assert len(pool2) == 0
    pool2.step_segment(5)  # an empty pool steps nothing
    pool.close()
    pool2.close()


def test_errors_are_statuses_with_messages():
    lib = _lib.lib
    cfg = _lib.SimConfig()
    cfg.n, cfg.nrad, cfg.nang, cfg.lmax, cfg.kT, cfg.dt = 100, 10, 8, 4, 1.0, 0.005
    h = ctypes.c_void_p()
    assert lib.amlp_create(ctypes.byref(cfg), ctypes.byref(h)) == 0
    s = torch.cuda.current_stream().cuda_stream
    assert lib.amlp_step(h, 10, 1, s) == 1  # no shape, model or state yet
    assert b"shape" in lib.amlp_last_error(h)
    pts = np.zeros((100, 3), np.float32)
    assert lib.amlp_set_shape(h, pts.ctypes.data, 100, -5.0, 15.0, 2.5, 2.5) == 1  # npts > AMLP_MAX_PTS
    net = _net(widths=(32,))
    bad = _lib.Mlp.from_buffer_copy(bytes(net.struct))
    bad.dims[0] = 40
    assert lib.amlp_set_model(h, ctypes.byref(bad), s) == 1
    assert b"descriptor" in lib.amlp_last_error(h)
    lib.amlp_destroy(h)
    st = make_state(200, "cube26", 0.30, seed=3)
    nat = NativeSystem(st, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    with pytest.raises(AmlpError, match="unknown mode"):
        nat._call("amlp_step", nat._h, 1, 7, s)
    with pytest.raises(AmlpError):
        nat.descriptors(cap=1)  # more filtered pairs than cap
    nat.close()
    pool = NativePool("cube26", Hypers(), net, dt=0.005)
    with pytest.raises(AmlpError, match="no such system"):
        pool._call("amlp_pool_evict", pool._h, 42, None, None, None, None, None)
    pool.close()
