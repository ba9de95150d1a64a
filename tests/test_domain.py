"""Spatial domain decomposition (amlp.domain) on two and three gloo ranks on the CPU.

Each rank owns the bodies of one slab of the box, receives the halo of its
neighbours by send/recv, and evaluates the forces of every pair with an owned
body over owned + halo bodies (the pairs across a boundary on both ranks, so no
forces travel back). The forces and torques each rank gets for its owned bodies
must be the single-domain forces of those bodies, and its share of the pair
energy must add up with the other rank's to the system's. Migration must hand
every body that left a slab to the rank that owns it now, each body on exactly
one rank. The force backend here is the oracle's FP64 exact derivative; the
library's kernels run the same decomposition in tests/test_gpu_domain.py.
"""
import os
import pickle
import socket

import numpy as np
import pytest
import torch

# (ranks, bodies, box): the reference's th_v1 init box of 33 with two slabs of 16.5, and a box of 48
# with three slabs of 16 (distinct lower and upper neighbours); each slab holds the halo of 7.75 twice
SETUPS = {2: (400, 33.0), 3: (1200, 48.0)}


def _state(world):
    from amlp.configs import make_state
    n, L = SETUPS[world]
    return make_state(n, "th_v1", 0.1, kT=0.5, seed=31, L=L)


def _layers():
    from conftest import load_model
    return load_model("th_C104")


def _forces(pos, quat, pairs_verlet, n_owned, L, shape, layers):
    from oracle import adjoint, nep
    vl = pairs_verlet[pairs_verlet[:, 0] < n_owned]
    _, pairs, _ = nep.min_image_filter(pos, vl, L, shape["cutoff"])
    ex = adjoint.exact_pair_forces(pos, quat, pairs, L, shape, (10, 8, 4), layers, "relu")
    own_pair = pairs[:, 1] < n_owned
    pe = ex["E"][own_pair].sum() + 0.5 * ex["E"][~own_pair].sum()
    return ex["forces"][:n_owned], ex["torques"][:n_owned], pe


def _worker(rank, world, port, outdir):
    import datetime
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for p in (here, os.path.dirname(here), os.path.join(os.path.dirname(here), "anisotropic-ml_b200")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from amlp.domain import Comm, Halo, Slab, migrate
    from oracle import nlist
    from oracle.shapes import SHAPES
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s = _state(world)
        shape = SHAPES["th_v1"]
        comm = Comm(dist, rank, world, "cpu")
        slab = Slab(s.L, world, rank)
        mine = np.nonzero(slab.owner(s.pos[:, 0]) == rank)[0]
        pos, quat = torch.tensor(s.pos[mine]), torch.tensor(s.orient[mine])
        halo = Halo(slab, shape["cutoff"] + 2.0)
        halo.choose(pos.numpy())
        ext_pos, ext_quat = halo.exchange(comm, pos, quat)
        vl = nlist.sorted_pairs(nlist.reference_pairs(ext_pos.numpy(), s.L, shape["cutoff"] + 2.0))
        F, T, pe = _forces(ext_pos.numpy(), ext_quat.numpy(), vl, len(mine), s.L, shape, _layers())
        pe_all = comm.sum(torch.tensor([pe], dtype=torch.float64)).item()
        # migration after every body moved by (3, 0.5, 0) (less than the skin along x)
        owned = {"pos": pos.clone(), "quat": quat.clone(), "vel": torch.tensor(s.vel[mine]),
                 "angmom": torch.tensor(s.angmom[mine]), "mass": torch.tensor(s.mass[mine]),
                 "ids": torch.tensor(mine, dtype=torch.long)}
        moved = owned["pos"] + torch.tensor([3.0, 0.5, 0.0])
        owned["pos"] = ((moved + s.L / 2) % s.L - s.L / 2).float()
        after = migrate(comm, slab, owned)
        with open(os.path.join(outdir, f"rank{rank}.pkl"), "wb") as fh:
            pickle.dump(dict(mine=mine, F=F, T=T, pe=pe, pe_all=pe_all, n_halo=int(ext_pos.shape[0]) - len(mine),
                             after={k: v.numpy() for k, v in after.items()}, lo=slab.lo, hi=slab.hi), fh)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.fixture(scope="module", params=sorted(SETUPS))
def ranks(request, tmp_path_factory):
    import torch.multiprocessing as mp
    world = request.param
    out = tmp_path_factory.mktemp(f"domain{world}")
    mp.start_processes(_worker, args=(world, _free_port(), str(out)), nprocs=world, start_method="spawn", join=True)
    res = []
    for r in range(world):
        with open(out / f"rank{r}.pkl", "rb") as fh:
            res.append(pickle.load(fh))
    return world, res


def test_domain_forces_equal_single_domain(ranks):
    from oracle import nlist
    from oracle.shapes import SHAPES
    world, ranks = ranks
    s = _state(world)
    shape = SHAPES["th_v1"]
    vl = nlist.sorted_pairs(nlist.reference_pairs(s.pos, s.L, shape["cutoff"] + 2.0))
    F, T, pe = _forces(s.pos, s.orient, vl, s.N, s.L, shape, _layers())
    owners = np.concatenate([r["mine"] for r in ranks])
    assert np.array_equal(np.sort(owners), np.arange(s.N))  # every body on exactly one rank
    for r in ranks:
        assert r["n_halo"] > 0
        np.testing.assert_allclose(r["F"], F[r["mine"]], rtol=0, atol=1e-9 * max(1.0, np.abs(F).max()))
        np.testing.assert_allclose(r["T"], T[r["mine"]], rtol=0, atol=1e-9 * max(1.0, np.abs(T).max()))
        assert abs(r["pe_all"] - pe) <= 1e-9 * max(1.0, abs(pe))
    assert abs(sum(r["pe"] for r in ranks) - pe) <= 1e-9 * max(1.0, abs(pe))


def test_migration_hands_every_body_to_its_new_owner(ranks):
    world, ranks = ranks
    s = _state(world)
    ids = np.concatenate([r["after"]["ids"] for r in ranks])
    assert np.array_equal(np.sort(ids), np.arange(s.N))
    for r in ranks:
        x = r["after"]["pos"][:, 0]
        assert np.all((x >= r["lo"]) & (x < r["hi"]))
        # the state travelled with the body
        np.testing.assert_array_equal(r["after"]["vel"], s.vel[r["after"]["ids"]])
        np.testing.assert_array_equal(r["after"]["quat"], s.orient[r["after"]["ids"]])
