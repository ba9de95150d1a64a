"""Spatial domain decomposition (amlp.domain) on two to eight gloo ranks on the CPU.

The box is cut into bricks: slabs along x for two and three ranks, a 2 x 2 x 1
and a 2 x 2 x 2 grid for four and eight. Each rank owns the bodies of its brick,
receives the halo of the others in one pass per cut axis (forwarding what the
earlier passes brought, so edge and corner neighbours arrive through the faces),
and evaluates the forces of every pair with an owned body over owned + halo
bodies (the pairs across a boundary on both ranks, so no forces travel back).
The forces and torques each rank gets for its owned bodies must be the
single-domain forces of those bodies, and its share of the pair energy must add
up with the other ranks' to the system's. Migration must hand every body that
left a brick, also across an edge or a corner, to the rank that owns it now,
each body on exactly one rank. The force backend here is the oracle's FP64
exact derivative; the library's kernels run the same decomposition in
tests/test_gpu_domain.py.
"""
import os
import pickle
import socket

import numpy as np
import pytest
import torch

# ranks -> (bodies, box, grid): the reference's th_v1 init box of 33 cut into two slabs of 16.5, a box
# of 48 into three slabs of 16, and the box of 33 into 2 x 2 x 1 and 2 x 2 x 2 bricks of 16.5; every
# cut axis holds the halo of 7.75 twice
SETUPS = {2: (400, 33.0, (2, 1, 1)), 3: (1200, 48.0, (3, 1, 1)), 4: (400, 33.0, (2, 2, 1)),
          8: (400, 33.0, (2, 2, 2))}


def _state(world):
    from amlp.configs import make_state
    n, L, _ = SETUPS[world]
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
    from amlp.domain import Brick, Comm, Halo, migrate
    from oracle import nlist
    from oracle.shapes import SHAPES
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        s = _state(world)
        shape = SHAPES["th_v1"]
        comm = Comm(dist, rank, world, "cpu", dims=SETUPS[world][2])
        brick = Brick(s.L, comm.dims, rank)
        mine = np.nonzero(brick.owner(s.pos) == rank)[0]
        pos, quat = torch.tensor(s.pos[mine]), torch.tensor(s.orient[mine])
        halo = Halo(brick, shape["cutoff"] + 2.0)
        ext_pos, ext_quat, ext_ids = halo.choose_and_exchange(comm, pos, quat, torch.tensor(mine, dtype=torch.long))
        vl = nlist.sorted_pairs(nlist.reference_pairs(ext_pos.numpy(), s.L, shape["cutoff"] + 2.0))
        F, T, pe = _forces(ext_pos.numpy(), ext_quat.numpy(), vl, len(mine), s.L, shape, _layers())
        pe_all = comm.sum(torch.tensor([pe], dtype=torch.float64)).item()
        # the halo copies arrive once each, with their global indices
        halo_ids = ext_ids[len(mine):].numpy()
        assert len(np.unique(halo_ids)) == len(halo_ids) and not np.isin(halo_ids, mine).any()
        # between rebuilds the same rows travel with the counts known, without a count exchange
        again_pos, again_quat = halo.exchange(comm, pos, quat)
        assert torch.equal(again_pos, ext_pos) and torch.equal(again_quat, ext_quat)
        # migration after every body moved by (3, 3, 3) (less than the skin along each axis): bodies
        # leave through faces, edges and corners
        owned = {"pos": pos.clone(), "quat": quat.clone(), "vel": torch.tensor(s.vel[mine]),
                 "angmom": torch.tensor(s.angmom[mine]), "mass": torch.tensor(s.mass[mine]),
                 "ids": torch.tensor(mine, dtype=torch.long)}
        moved = owned["pos"] + torch.tensor([3.0, 3.0, 3.0])
        owned["pos"] = ((moved + s.L / 2) % s.L - s.L / 2).float()
        after = migrate(comm, brick, owned)
        with open(os.path.join(outdir, f"rank{rank}.pkl"), "wb") as fh:
            pickle.dump(dict(mine=mine, F=F, T=T, pe=pe, pe_all=pe_all, n_halo=int(ext_pos.shape[0]) - len(mine),
                             after={k: v.numpy() for k, v in after.items()},
                             lo=[brick.lo(a) for a in range(3)], hi=[brick.hi(a) for a in range(3)]), fh)
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
        for a in range(3):
            x = r["after"]["pos"][:, a]
            assert np.all((x >= r["lo"][a]) & (x < r["hi"][a]))
        # the state travelled with the body
        np.testing.assert_array_equal(r["after"]["vel"], s.vel[r["after"]["ids"]])
        np.testing.assert_array_equal(r["after"]["quat"], s.orient[r["after"]["ids"]])


def test_brick_dims_prefers_cubes_that_hold_the_halo():
    from amlp.domain import brick_dims
    assert brick_dims(8, 33.0, 7.75) == (2, 2, 2)
    assert brick_dims(4, 33.0, 7.75) == (2, 2, 1)
    assert brick_dims(2, 33.0, 7.75) == (2, 1, 1)
    assert brick_dims(8, 200.0, 7.75) == (2, 2, 2)
    assert brick_dims(6, 66.0, 7.75) == (3, 2, 1)
    with pytest.raises(ValueError):
        brick_dims(4, 20.0, 7.75)  # bricks of 10 < two halos: no grid of four fits
