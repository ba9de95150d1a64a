"""Host-side tests that need no GPU: the C-ABI library loads and exports every
declared symbol, argument validation, GSD I/O, shape tables, seeded configs,
the exact-derivative oracle."""
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, REPO


@pytest.fixture(scope="module")
def lib():
    from amlp import build
    build.build()
    from amlp import _lib
    return _lib


def _declared():
    text = open(os.path.join(REPO, "include", "amlp.h")).read()
    decl = r"^(?:amlp_status|int|void|long long|const char \*)\s*\*?(amlp_[a-z0-9_]+)\s*\("
    return sorted(set(re.findall(decl, text, flags=re.M)))


def test_header_symbols_exported(lib):
    names = _declared()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib.lib, n), f"{n} declared in include/amlp.h but not exported"
    assert set(names) <= set(lib.exported_symbols()), "a declared entry point has no ctypes signature"


def test_status_strings(lib):
    assert lib.lib.amlp_version() >= 1
    assert lib.status_string(0) == "ok"
    assert "workspace" in lib.status_string(3)


def test_argument_validation_without_gpu(lib):
    import ctypes
    # invalid sizes are rejected before any CUDA call
    assert lib.call_status("amlp_nlist_build", None, 0, 10.0, 4.5, None, 0, None, None, 0, None) == 1
    assert lib.call_status("amlp_nlist_build", None, 10, -1.0, 4.5, None, 0, None, None, 0, None) == 1
    sz = ctypes.c_size_t()
    assert lib.call_status("amlp_nlist_workspace_bytes", 1000, 14.9, 4.5, ctypes.byref(sz)) == 0 and sz.value > 0
    assert lib.call_status("amlp_nvt_workspace_bytes", 0, ctypes.byref(sz)) == 1
    n = lib.Nep()
    n.nrad, n.nang, n.lmax, n.npts = 3, 3, 3, 4  # no compiled kernel for these hypers
    n.d_pts, n.cutoff, n.nep_cutoff = 1, 2.5, 2.5
    assert lib.call_status("amlp_descriptors", 1, 1, 10.0, 1, 1, ctypes.byref(n), 1, None) == 2
    with pytest.raises(lib.AmlpError):
        lib.call("amlp_nvt_workspace_bytes", -5, ctypes.byref(sz))
    # simulation handles and the pool: null and out-of-range arguments, no CUDA call
    h = ctypes.c_void_p()
    assert lib.call_status("amlp_create", None, ctypes.byref(h)) == 1 and not h.value
    cfg = lib.SimConfig()
    cfg.n, cfg.nrad, cfg.nang, cfg.lmax, cfg.dt = 0, 10, 8, 4, 0.005
    assert lib.call_status("amlp_create", ctypes.byref(cfg), ctypes.byref(h)) == 1 and not h.value
    assert lib.call_status("amlp_step", None, 1, 0, None) == 1
    assert lib.lib.amlp_last_error(None) == b"null handle"
    assert lib.lib.amlp_timestep(None) == -1
    lib.lib.amlp_destroy(None)
    assert lib.call_status("amlp_pool_create", None, ctypes.byref(h)) == 1
    pc = lib.PoolConfig()
    assert lib.call_status("amlp_pool_create", ctypes.byref(pc), ctypes.byref(h)) == 1 and not h.value
    assert lib.lib.amlp_pool_size(None) == 0
    assert lib.call_status("amlp_pool_step_segment", None, 1, None) == 1
    lib.lib.amlp_pool_destroy(None)


def test_gsd_reads_hoomd_file_and_roundtrips(tmp_path):
    from amlp.gsd import Frame, GsdFile, read_last_frame
    z = np.load(os.path.join(GOLDEN, "init_th_init_N200.npz"))
    f = Frame()
    f.step, f.N, f.box, f.types = 100, 200, z["box"], ["Re", "Os"]
    for k in ("position", "orientation", "velocity", "angmom", "moment_inertia", "body", "image"):
        f.particles[k] = z[k]
    p = str(tmp_path / "a.gsd")
    with GsdFile(p, "w") as g:
        g.append(f)
        f.step = 200
        f.particles["position"] = z["position"] + 1
        f.log["thermostat/integrator_vars"] = np.arange(4, dtype=np.float32)
        g.append(f)
    with GsdFile(p, "a") as g:  # append a third frame to an existing file
        for k in range(40):     # grow the index past its first allocation
            f.step = 300 + k
            g.append(f)
    r = read_last_frame(p)
    assert r.step == 339 and r.N == 200 and r.types == ["Re", "Os"]
    np.testing.assert_array_equal(r.particles["position"], z["position"] + 1)
    np.testing.assert_array_equal(r.get("mass"), np.ones(200, np.float32))  # schema default
    np.testing.assert_array_equal(r.log["thermostat/integrator_vars"], np.arange(4, dtype=np.float32))
    with GsdFile(p) as g:
        assert len(g) == 42
        np.testing.assert_array_equal(g[0].particles["position"], z["position"])


def test_gsd_rejects_corrupt(tmp_path):
    from amlp.gsd import GsdError, GsdFile
    p = tmp_path / "bad.gsd"
    p.write_bytes(b"not a gsd file" * 30)
    with pytest.raises(GsdError):
        GsdFile(str(p))


def test_reference_init_file_reader():
    from oracle.ref_kernels import REF_ROOT
    ref = os.path.join(REF_ROOT, "nep_simulator", "init", "th_init_N200.gsd")
    if not os.path.exists(ref):
        pytest.skip("reference checkout not present")
    from amlp.gsd import read_last_frame
    f = read_last_frame(ref)
    z = np.load(os.path.join(GOLDEN, "init_th_init_N200.npz"))
    assert f.N == 200 and f.step == int(z["step"])
    np.testing.assert_array_equal(f.particles["position"], z["position"])


def test_shapes_match_oracle_tables():
    from amlp.shapes import SHAPES
    from oracle.shapes import SHAPES as OS
    assert set(SHAPES) == set(OS)
    for k, s in SHAPES.items():
        np.testing.assert_array_equal(s.pts, OS[k]["pts"])
        assert (s.en_min, s.en_max, s.cutoff, s.nep_cutoff) == (OS[k]["en_min"], OS[k]["en_max"], OS[k]["cutoff"],
                                                                OS[k]["nep_cutoff"])
    assert SHAPES["cube26"].npts == 26 and SHAPES["tetra16"].npts == 16 and SHAPES["cyl24"].npts == 24


def test_unknown_shape_raises():
    from amlp.shapes import get_shape
    with pytest.raises(KeyError):
        get_shape("dodecahedron")


def test_configs_seeded_and_physical():
    from amlp.configs import make_state, quat_mul
    a = make_state(1000, "cube26", 0.30, kT=1.0, seed=0)
    b = make_state(1000, "cube26", 0.30, kT=1.0, seed=0)
    np.testing.assert_array_equal(a.pos, b.pos)
    assert abs(a.L ** 3 - 1000 / 0.30) / (1000 / 0.30) < 1e-5
    assert np.all(np.abs(a.pos) <= a.L / 2)
    np.testing.assert_allclose(np.linalg.norm(a.orient, axis=1), 1, atol=1e-6)
    # rotational KE as the reference computes it: s = 1/2 conj(q) p, KE = sum s_k^2 / (2 I_k)
    conj = a.orient.astype(np.float64) * np.array([1, -1, -1, -1])
    s = 0.5 * quat_mul(conj, a.angmom.astype(np.float64))
    ke_r = 0.5 * np.sum(s[:, 1:] ** 2 / a.moi.astype(np.float64), axis=1).mean()
    assert abs(ke_r - 1.5) < 0.2 and np.abs(s[:, 0]).max() < 1e-5
    assert abs(0.5 * np.sum(a.vel.astype(np.float64) ** 2, axis=1).mean() - 1.5) < 0.2


def test_exact_forces_oracle_matches_fp64_differences():
    from amlp.configs import make_state
    from amlp.engine import EnergyNet
    from oracle import adjoint, nep, nlist
    from oracle.shapes import SHAPES
    s = make_state(120, "tetra16", 0.40, seed=2)
    shape = SHAPES["tetra16"]
    vp = nlist.sorted_pairs(nlist.reference_pairs(s.pos, s.L, 4.5))
    _, pairs, _ = nep.min_image_filter(s.pos, vp, s.L, 2.5)
    pairs = pairs[:150]
    net = EnergyNet.xavier(47, (32, 32), "silu", seed=4, device="cpu")
    a = adjoint.exact_pair_forces(s.pos, s.orient, pairs, s.L, shape, (10, 8, 4), net.layers, "silu", clip=False)
    o = nep.pair_forces(s.pos, s.orient, pairs, s.L, shape, (10, 8, 4), net.layers, "silu", dt=np.float64, form="sh")
    e = o["e_all"].reshape(10, -1)
    rng = shape["en_max"] - shape["en_min"]
    for k, base in (("F_pair", 1), ("T_i", 4), ("T_j", 7)):
        fd = np.stack([-(e[base + c] - e[0]) / 1e-5 for c in range(3)], 1) * rng
        scale = max(1.0, np.abs(fd).max())
        assert np.abs(fd - a[k]).max() <= 2e-3 * scale, k  # forward-difference truncation O(dx)


def test_central_differences_oracle_matches_exact_derivative():
    """FP64 central differences (step 1e-4) of the summed pair energy of a body
    agree with the exact derivative (autograd) to the O(h^2) truncation."""
    from amlp.configs import make_state
    from amlp.engine import EnergyNet
    from oracle import adjoint, nep, nlist
    from oracle.shapes import SHAPES
    s = make_state(200, "tetra16", 0.40, seed=2)
    shape = SHAPES["tetra16"]
    vp = nlist.sorted_pairs(nlist.reference_pairs(s.pos, s.L, 4.5))
    _, pairs, _ = nep.min_image_filter(s.pos, vp, s.L, 2.5)
    bodies = np.array([3, 77, 150])
    sub = pairs[np.isin(pairs[:, 0], bodies) | np.isin(pairs[:, 1], bodies)]
    net = EnergyNet.xavier(47, (32, 32), "silu", seed=4, device="cpu")
    F, T = adjoint.central_difference_forces(s.pos, s.orient, sub, s.L, shape, (10, 8, 4), net.layers, "silu",
                                             bodies, h=1e-4)
    a = adjoint.exact_pair_forces(s.pos, s.orient, sub, s.L, shape, (10, 8, 4), net.layers, "silu", clip=False)
    for got, want in ((F, a["forces"][bodies]), (T, a["torques"][bodies])):
        assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())


def test_oracle_workload_is_the_products():
    """bench.py's reference arm builds its state and net with oracle.workload (it
    imports nothing of the product): the arrays must be the product's, bit for bit."""
    from amlp.configs import make_state
    from amlp.engine import EnergyNet
    from oracle import workload
    for args in ((1000, "cube26", 0.30, 1.0, 0), (4096, "tetra16", 0.40, 0.7, 2), (3000, "cyl24", 0.35, 1.3, 3)):
        a, b = workload.make_state(*args), make_state(*args[:3], kT=args[3], seed=args[4])
        assert a.L == b.L
        for k in ("pos", "orient", "vel", "angmom", "mass", "moi"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), k
    for (Wa, ba), (Wb, bb) in zip(workload.xavier_layers(47, (64, 64), 1),
                                  EnergyNet.xavier(47, (64, 64), "tanh", seed=1, device="cpu").layers):
        assert np.array_equal(Wa, Wb) and np.array_equal(ba, bb)
