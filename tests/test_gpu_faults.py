"""Bounded device-side waits, made to give up on purpose, without any fault.

Every wait of the library's kernels on tensor-core completion (an mbarrier) has
an iteration limit. When a wait runs out, the kernel raises bit 1 of
amlp_device_error, issues no further MMA, lets the one in flight finish (a
second wait at the normal limit), frees its tensor memory and returns; the
host raises AmlpDeviceError at its next check. The test hook
amlp_test_first_wait_limit(0) makes the first such wait of every CTA give up at
once, which runs exactly that path: nothing hangs, nothing faults, and the
next launch with the normal limit is clean.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from amlp import _lib  # noqa: E402
from amlp.configs import make_state  # noqa: E402
from amlp.engine import EnergyNet, Hypers, System  # noqa: E402
from oracle import adjoint  # noqa: E402
from oracle.shapes import SHAPES  # noqa: E402

DEV = torch.device("cuda:0")


def _system(seed):
    s = make_state(400, "cube26", 0.45, seed=seed)
    net = EnergyNet.xavier(47, (64, 64), "tanh", seed=seed + 1, device=DEV)
    return s, net, System(s, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=DEV)


def test_wait_that_gives_up_is_reported_and_the_next_launch_is_clean():
    _lib.device_error(clear=True)
    _, _, sysm = _system(3)
    _lib.call("amlp_test_first_wait_limit", 0)
    try:
        # one force pass: every CTA abandons its first tile, so no pair force is scattered
        sysm.compute_forces("adjoint")
        torch.cuda.synchronize()
        assert int(sysm.nf.item()) > 0
        assert float(sysm.F.abs().sum()) == 0.0 and float(sysm.T.abs().sum()) == 0.0
        assert _lib.device_error(clear=False) & 1
        # the host side raises at its next check (here: the end of run())
        with pytest.raises(_lib.AmlpDeviceError):
            sysm.run(2, "adjoint")
    finally:
        _lib.call("amlp_test_first_wait_limit", -1)
    assert _lib.device_error() == 0  # the raise cleared the flags

    # the next launches, at the normal limit, give the exact forces and raise nothing
    s, net, fresh = _system(5)
    fresh.compute_forces("adjoint")
    torch.cuda.synchronize()
    assert _lib.device_error() == 0
    fp = fresh.filtered_pairs().astype(np.int64)
    ex = adjoint.exact_pair_forces(s.pos, s.orient, fp, s.L, SHAPES["cube26"], (10, 8, 4), net.layers, "tanh")
    for got, want in ((fresh.F, ex["forces"]), (fresh.T, ex["torques"])):
        got = got.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-3
    fresh.run(3, "adjoint")  # and a graph-captured segment after it
    assert torch.isfinite(fresh.pos).all()


def test_simulation_handle_reports_the_wait_as_a_status():
    """The C ABI's simulation handle checks the flags at its synchronisations
    (the Verlet rebuilds) and returns AMLP_ERR_DEVICE_WAIT (7)."""
    from amlp._lib import AmlpError
    from amlp.native import NativeSystem
    s, net, _ = _system(7)
    _lib.device_error(clear=True)
    nat = NativeSystem(s, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    _lib.call("amlp_test_first_wait_limit", 0)
    try:
        with pytest.raises(AmlpError) as info:
            nat.run(150, "adjoint")  # a rebuild at step 100
        assert info.value.status == 7
    finally:
        _lib.call("amlp_test_first_wait_limit", -1)
        torch.cuda.synchronize()
        _lib.device_error(clear=True)
    nat.run(50, "adjoint")  # the flags cleared: the handle carries on
    torch.cuda.synchronize()
    assert _lib.device_error() == 0
    nat.close()
