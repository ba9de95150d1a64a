"""The domain-decomposed NVT run (amlp.domain.DomainSystem) on one GPU, its two
ranks emulated by two host threads that exchange halos, migrating bodies and
kinetic energies through in-process mailboxes. No kernel of one rank waits for
the other's: every wait is on the host, with a timeout.

* the forces and torques of the first step equal the single-domain forces of
  the same bodies (float atomics aside);
* after 150 steps (two Verlet rebuilds, one migration) every body is owned by
  exactly one rank, and the positions differ from the single-domain run by no
  more than 10x the drift between two identical single-domain runs (the float
  atomics' summation order) plus 1e-5 of the box.
"""
import threading

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from amlp.configs import make_state  # noqa: E402
from amlp.domain import DomainSystem  # noqa: E402
from amlp.engine import EnergyNet, Hypers, System  # noqa: E402
from amlp.shapes import get_shape  # noqa: E402

DEV = torch.device("cuda:0")
WORLD = 2


class _Hub:
    def __init__(self, world):
        self.world = world
        self.box = [None] * world
        self.barrier = threading.Barrier(world, timeout=120)

    def round(self, rank, item):
        self.barrier.wait()
        self.box[rank] = item
        self.barrier.wait()
        items = list(self.box)
        self.barrier.wait()
        return items


class LoopbackComm:
    """The Comm interface of amlp.domain for ranks that are threads of one process
    (a world x 1 x 1 grid: slabs along x)."""

    def __init__(self, hub, rank):
        self.hub, self.rank, self.world, self.device = hub, rank, hub.world, DEV
        self.dims = (hub.world, 1, 1)
        self.lower, self.upper = (rank - 1) % self.world, (rank + 1) % self.world

    def shift(self, to_lower, to_upper, axis=0, counts=None):
        if self.dims[axis] == 1:
            return to_lower[:0].clone(), to_upper[:0].clone()
        items = self.hub.round(self.rank, (to_lower.clone(), to_upper.clone()))
        return items[self.upper][0].clone(), items[self.lower][1].clone()

    def sum(self, t):
        items = self.hub.round(self.rank, t.clone())
        t.copy_(sum(items))
        return t


def _setup():
    s = make_state(4000, "cube26", 0.30, kT=1.0, seed=41)
    net = EnergyNet.xavier(47, (64, 64), "tanh", seed=42, device="cpu")
    net = EnergyNet([(W * np.float32(0.05) if k == 2 else W, b) for k, (W, b) in enumerate(net.layers)], "tanh", DEV)
    return s, net


def _run_domains(s, net, steps):
    hub = _Hub(WORLD)
    out, errors = [None] * WORLD, []

    def body(rank):
        try:
            torch.cuda.set_device(DEV)
            d = DomainSystem(LoopbackComm(hub, rank), s, get_shape("cube26"), Hypers(), net, kT=1.0, dt=0.005,
                             device=DEV)
            ids = d.owned["ids"].cpu().numpy()
            d.step()
            torch.cuda.synchronize()
            first = (ids, d.F.cpu().numpy(), d.T.cpu().numpy())
            d.run(steps - 1)
            torch.cuda.synchronize()
            out[rank] = (first, d.gather())
        except Exception as e:  # noqa: BLE001
            errors.append(e)
            hub.barrier.abort()

    th = [threading.Thread(target=body, args=(r,)) for r in range(WORLD)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    if errors:
        raise errors[0]
    return out


def _single(s, net, steps):
    a = System(s, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    F0 = T0 = None
    for k in range(steps):
        a.step("adjoint")
        if k == 0:
            torch.cuda.synchronize()
            F0, T0 = a.F.cpu().numpy(), a.T.cpu().numpy()
    torch.cuda.synchronize()
    return a, F0, T0


def test_two_domain_run_matches_single_domain():
    s, net = _setup()
    steps = 150
    dom = _run_domains(s, net, steps)
    a, F0, T0 = _single(s, net, steps)
    b, _, _ = _single(s, net, steps)
    for (ids, F, T), _ in dom:
        np.testing.assert_allclose(F, F0[ids], rtol=0, atol=1e-5 * max(1.0, np.abs(F0).max()))
        np.testing.assert_allclose(T, T0[ids], rtol=0, atol=1e-5 * max(1.0, np.abs(T0).max()))
    ids = np.concatenate([g["ids"] for _, g in dom])
    assert np.array_equal(np.sort(ids), np.arange(s.N))
    pos = np.empty((s.N, 3), np.float32)
    for _, g in dom:
        pos[g["ids"]] = g["pos"]
    ya, yb = a.pos.cpu().numpy(), b.pos.cpu().numpy()
    floor = np.abs(ya - yb).max()

    def dist(x, y):  # minimum image: a body may have crossed the periodic boundary in one run only
        d = x - y
        return np.abs(d - s.L * np.round(d / s.L)).max()

    assert dist(pos, ya) <= 10 * floor + 1e-5 * s.L
