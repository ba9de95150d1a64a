"""Parity of every CUDA entry point with the oracle (and through the oracle, with
the reference's own run). All calls go through the C ABI of libamlp.

Tolerances:
* Verlet list and pair filter: bit-exact (same pairs, same order);
* descriptors: |g_gpu - g_fp64| <= 5e-5 * max(1, |g|) -- the GPU evaluates the
  angular sum in FP32 through the addition theorem, or directly like the
  reference for clouds of at most 12 points and the (10, 10, 10) hypers;
* net energies: relative 1e-5 against torch FP32 on the same descriptors; on
  the GPU's own descriptors, the deviation from FP64 may not exceed twice the
  reference's own FP32 deviation from FP64 (plus 1e-6 of the energy scale);
* finite-difference forces: the reference's own FP32 forward differences
  (dx = dteta = 1e-5) carry rounding noise of up to tens of force units per
  pair (see test_fd_noise_floor_of_the_reference), so they are compared as a
  distribution: the GPU's deviation from FP64 finite differences may not exceed
  the reference's own deviation by more than a factor 2 at the 50/90/99 %
  quantiles; the pair-energy sum must agree to 1e-5 relative;
* integrator: positions/velocities/quaternions relative 2e-6 against the FP32
  oracle given the same forces.
"""
import numpy as np
import pytest
import torch

from conftest import case_model, case_shape, load_case

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import gpu_helpers as gh  # noqa: E402
from amlp.configs import make_state  # noqa: E402
from oracle import nep, nlist  # noqa: E402
from oracle.shapes import SHAPES  # noqa: E402

CASES = ["th_C104", "th_C100", "cube_C104", "cube_R64"]


def _hyp(c):
    return tuple(int(h) for h in c["hypers"][:3])


# ----------------------------------------------------------------------------- Verlet list
def _nlist_cases():
    rng = np.random.default_rng(5)
    out = []
    for name in CASES:
        c = load_case(name)
        out.append((f"golden-{name}", c["pos0"], float(c["L"]), case_shape(c)["cutoff"] + 2.0))
    L = np.float32(20.0)
    out.append(("uniform-3000", (rng.random((3000, 3)) * L - L / 2).astype(np.float32), float(L), 4.5))
    s = make_state(4096, "cube26", 0.45, seed=1)
    out.append(("cube26-4096-phi045", s.pos, s.L, 4.5))
    s = make_state(2000, "cyl24", 0.35, seed=3)
    out.append(("cyl24-2000", s.pos, s.L, 4.5))
    # dense: more than a warp's shared buffer (1,024) of neighbours j > i for many bodies
    s = make_state(8000, "tetra16", 0.40, seed=2)
    out.append(("tetra16-8000-phi040-dense", s.pos, s.L, 4.5))
    L = np.float32(8.0)
    out.append(("small-box-brute-force", (rng.random((60, 3)) * L - L / 2).astype(np.float32), float(L), 4.5))
    out.append(("one-body", np.zeros((1, 3), np.float32), 10.0, 4.5))
    L = np.float32(30.0)
    out.append(("sparse-empty", np.array([[-10, -10, -10], [0, 0, 0], [10, 10, 10]], np.float32), float(L), 2.0))
    # bodies on the box faces and pairs at exactly r along an axis
    edge = np.array([[-15, 0, 0], [14.5, 0, 0], [0, -15, 0], [0, 14.99, 0], [0, 0, 4.5], [0, 0, 0],
                     [4.5, 0, 0], [-4.5, 0, 0], [0, 0, -15]], np.float32)
    out.append(("faces-and-exact-r", edge, 30.0, 4.5))
    return out


@pytest.mark.parametrize("case", _nlist_cases(), ids=lambda c: c[0])
def test_nlist_bit_exact_vs_ckdtree(case):
    _, pos, L, r = case
    got, k = gh.nlist(pos, L, r)
    ref = nlist.sorted_pairs(nlist.reference_pairs(pos, L, r))
    assert k == len(ref)
    assert np.array_equal(got, ref), "GPU Verlet list differs from cKDTree.query_pairs"


def test_nlist_capacity_reports_count():
    s = make_state(1000, "cube26", 0.45, seed=0)
    full, k = gh.nlist(s.pos, s.L, 4.5)
    part, k2 = gh.nlist(s.pos, s.L, 4.5, cap=100)
    assert k2 == k and np.array_equal(part, full[:100])
    # a capacity that cuts through a body with more than 1,024 neighbours j > i
    s = make_state(8000, "tetra16", 0.40, seed=2)
    full, k = gh.nlist(s.pos, s.L, 4.5)
    counts = np.bincount(full[:, 0], minlength=8000)
    big = int(np.argmax(counts > 1024))
    assert counts[big] > 1024
    cut = int(counts[:big].sum()) + 500
    part, k2 = gh.nlist(s.pos, s.L, 4.5, cap=cut)
    assert k2 == k and np.array_equal(part, full[:cut])


# ----------------------------------------------------------------------------- pair filter
@pytest.mark.parametrize("name", CASES)
def test_filter_bit_exact(name):
    c = load_case(name)
    shape = case_shape(c)
    vp, _ = gh.nlist(c["pos0"], c["L"], shape["cutoff"] + 2.0)
    got = gh.pair_filter(c["pos0"], c["L"], shape["cutoff"], vp)
    _, ref, _ = nep.min_image_filter(c["pos0"], vp, c["L"], shape["cutoff"])
    assert np.array_equal(got, ref)
    assert np.array_equal(got, nlist.sorted_pairs(c["pairs0"]))  # the reference's own filtered pairs


def test_filter_random_cube26():
    s = make_state(3000, "cube26", 0.45, seed=4)
    vp, _ = gh.nlist(s.pos, s.L, 4.5)
    got = gh.pair_filter(s.pos, s.L, 2.5, vp)
    _, ref, _ = nep.min_image_filter(s.pos, vp, s.L, 2.5)
    assert np.array_equal(got, ref)


# ----------------------------------------------------------------------------- descriptors
def _check_desc(g, g64):
    scale = np.maximum(1.0, np.abs(g64))
    err = np.abs(g - g64) / scale
    assert err.max() <= 5e-5, f"max scaled descriptor error {err.max():.3g}"


@pytest.mark.parametrize("name", CASES)
def test_descriptors_vs_reference_and_fp64(name):
    c = load_case(name)
    shape, hyp = case_shape(c), _hyp(c)
    pairs = c["pairs0"]
    P = len(pairs)
    g = gh.descriptors(c["pos0"], c["orient0"], c["L"], pairs, shape, hyp)
    _, _, t = nep.min_image_filter(c["pos0"], pairs, c["L"], shape["cutoff"], np.float64)
    c1, c2 = nep.pair_clouds(c["orient0"], pairs, t, shape["pts"], np.float64)
    g64 = nep.descriptor(nep.fd_variants(c1, c2, 1e-5, 1e-5, np.float64), hyp, shape["nep_cutoff"], np.float64)
    _check_desc(g, g64)
    head = g.reshape(10, P, -1)[:, :c["g0"].shape[1]]
    _check_desc(head, c["g0"].astype(np.float64))


@pytest.mark.parametrize("shape_name,phi,seed", [("cube26", 0.45, 1), ("tetra16", 0.40, 2), ("cyl24", 0.35, 3)])
def test_descriptors_new_shapes(shape_name, phi, seed):
    s = make_state(160, shape_name, phi, seed=seed)
    shape = SHAPES[shape_name]
    vp = nlist.sorted_pairs(nlist.reference_pairs(s.pos, s.L, 4.5))
    _, pairs, t = nep.min_image_filter(s.pos, vp, s.L, shape["cutoff"])
    pairs = pairs[:200]
    g = gh.descriptors(s.pos, s.orient, s.L, pairs, shape, (10, 8, 4))
    _, _, t = nep.min_image_filter(s.pos, pairs, s.L, shape["cutoff"], np.float64)
    c1, c2 = nep.pair_clouds(s.orient, pairs, t, shape["pts"], np.float64)
    g64 = nep.descriptor(nep.fd_variants(c1, c2, 1e-5, 1e-5, np.float64), (10, 8, 4), shape["nep_cutoff"],
                         np.float64, form="sh")
    _check_desc(g, g64)


@pytest.mark.parametrize("shape_name,hyp,ld", [("th_v1", (10, 8, 4), 52), ("cube_v2", (10, 8, 4), 47),
                                               ("pbp_v3", (10, 8, 4), 48), ("th_v1", (10, 10, 10), 132),
                                               ("cube_v2", (10, 10, 10), 121)])
def test_pair_descriptors_vs_fp64(shape_name, hyp, ld):
    """amlp_pair_descriptors, the forward of the adjoint path: the direct form for
    (10, 10, 10) and for (10, 8, 4) clouds of up to 12 points (th_v1, cube_v2), the
    harmonic form for pbp_v3's 14; row strides with and without 16-byte rows and
    zero padding past D."""
    s = make_state(300, shape_name, 0.1, seed=5, L={"pbp_v3": 32.0}.get(shape_name, 24.0))  # ~20 neighbours each
    shape = SHAPES[shape_name]
    vp = nlist.sorted_pairs(nlist.reference_pairs(s.pos, s.L, shape["cutoff"] + 2.0))
    _, pairs, _ = nep.min_image_filter(s.pos, vp, s.L, shape["cutoff"])
    assert 1000 < len(pairs) < 10000
    D = (hyp[0] + 1) + (hyp[1] + 1) * hyp[2]
    g = gh.pair_descriptors(s.pos, s.orient, s.L, pairs, shape, hyp, ld=ld)
    _, _, t = nep.min_image_filter(s.pos, pairs, s.L, shape["cutoff"], np.float64)
    c1, _ = nep.pair_clouds(s.orient, pairs, t, shape["pts"], np.float64)
    g64 = nep.descriptor(c1, hyp, shape["nep_cutoff"], np.float64)
    _check_desc(g[:, :D], g64)
    if ld > D:
        assert np.all(g[:, D:] == 0.0)


@pytest.mark.parametrize("shape_name,hyp", [("cube_v2", (10, 10, 10)), ("pbp_v3", (10, 10, 10)),
                                            ("pbp_v3", (10, 8, 4))])
def test_descriptors_both_forms(shape_name, hyp):
    """amlp_descriptors (g_all of the ten finite-difference variants) in both of
    its forms: the direct form for cube_v2's 12-point clouds, the harmonic passes
    for pbp_v3's 14 points, with (10, 10, 10) because the direct form's
    per-thread clouds would not fit the shared memory beside its 121-row tile."""
    s = make_state(300, shape_name, 0.1, seed=6, L={"pbp_v3": 32.0}.get(shape_name, 24.0))
    shape = SHAPES[shape_name]
    vp = nlist.sorted_pairs(nlist.reference_pairs(s.pos, s.L, shape["cutoff"] + 2.0))
    _, pairs, _ = nep.min_image_filter(s.pos, vp, s.L, shape["cutoff"])
    pairs = pairs[:400]
    g = gh.descriptors(s.pos, s.orient, s.L, pairs, shape, hyp)
    _, _, t = nep.min_image_filter(s.pos, pairs, s.L, shape["cutoff"], np.float64)
    c1, c2 = nep.pair_clouds(s.orient, pairs, t, shape["pts"], np.float64)
    g64 = nep.descriptor(nep.fd_variants(c1, c2, 1e-5, 1e-5, np.float64), hyp, shape["nep_cutoff"], np.float64)
    _check_desc(g, g64)


# ----------------------------------------------------------------------------- net energies
@pytest.mark.parametrize("widths,act", [((64, 64), "tanh"), ((128, 128, 128), "silu"), ((150, 150, 150, 150), "relu"),
                                        ((160, 160), "relu"), ((100, 37), "tanh")])
def test_mlp_energy_vs_torch(widths, act):
    """amlp_mlp_energy against FP32 torch on 3001 rows (a partial last tile): the
    160-wide layers' register tiling (150 padded, and 160 with no padding column),
    the narrower layers' columns (64, 100 and 37 wide) and the one-output layer."""
    from amlp.engine import EnergyNet
    rng = np.random.default_rng(0)
    g = rng.standard_normal((3001, 47)).astype(np.float32)
    net = EnergyNet.xavier(47, widths, act, seed=3, device="cpu")
    ref = nep.mlp_forward(net.layers, act, g).reshape(-1)
    got = gh.mlp_energy(net.layers, act, g)
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5 * np.abs(ref).max())


@pytest.mark.parametrize("name", CASES)
def test_mlp_energy_golden(name):
    c = load_case(name)
    layers = case_model(c)
    shape, hyp = case_shape(c), _hyp(c)
    pairs = c["pairs0"]
    g = gh.descriptors(c["pos0"], c["orient0"], c["L"], pairs, shape, hyp)
    e = gh.mlp_energy(layers, "relu", g)
    e64 = _fd64(c, shape, hyp, layers)["e_all"]
    ref_err = np.abs(c["e0"] - e64).max()
    gpu_err = np.abs(e - e64).max()
    assert gpu_err <= 2 * ref_err + 1e-6 * np.abs(e64).max(), (gpu_err, ref_err)
    rel = np.abs(e - c["e0"]) / np.maximum(np.abs(c["e0"]), 1e-3)
    assert np.median(rel) <= 1e-5  # typical agreement with the reference's energies


# ----------------------------------------------------------------------------- forces
@pytest.mark.parametrize("name", CASES)
def test_fd_scatter_matches_reference(name):
    """Same energies in -> the reference's forces out (only the atomic summation order differs)."""
    c = load_case(name)
    shape = case_shape(c)
    N = len(c["pos0"])
    F, T, pe = gh.fd_scatter(c["e0"], c["pairs0"], N, shape)
    tol = 1e-5 * max(1.0, np.abs(c["F0"]).max())
    np.testing.assert_allclose(F, c["F0"], rtol=0, atol=tol)
    np.testing.assert_allclose(T, c["T0"], rtol=0, atol=1e-5 * max(1.0, np.abs(c["T0"]).max()))
    P = len(c["pairs0"])
    en_min32 = np.float64(np.float32(shape["en_min"]))
    rng32 = np.float64(np.float32(np.float32(shape["en_max"]) - np.float32(shape["en_min"])))
    pe_ref = np.sum(en_min32 + rng32 * c["e0"][:P].astype(np.float64))  # FP32 constants, FP64 sum
    assert abs(pe - pe_ref) <= 1e-9 * max(1.0, abs(pe_ref)) * P


def _fd64(c, shape, hyp, layers, act="relu"):
    pairs = c["pairs0"]
    return nep.pair_forces(c["pos0"], c["orient0"], pairs, c["L"], shape, hyp, layers, act, dt=np.float64)


def test_fd_noise_floor_of_the_reference():
    """Documents the size of the reference's FP32 finite-difference noise."""
    c = load_case("th_C104")
    shape, hyp, layers = case_shape(c), _hyp(c), case_model(c)
    o64 = _fd64(c, shape, hyp, layers)
    P = len(c["pairs0"])
    rng = shape["en_max"] - shape["en_min"]
    f32 = np.clip(c["Fgrad0"] * np.float32(rng), -100, 100)
    err = np.abs(f32 - o64["F_pair"])
    assert np.quantile(err, 0.99) > 0.1  # the noise is real and large
    assert P == o64["P"]


def test_fused_fd_kernel_on_the_reference_run():
    """The benched plain kernel (amlp_forces_fd: descriptors of the 10 variants,
    FP32 net, differences, clip and scatter in one kernel) on the fixture that the
    reference's own DescriptorGenerator + ForceEvaluator made with a
    47 -> 64 -> 64 -> 1 ReLU net (cube_R64: 400 cube_v2 bodies, 2,780 pairs).

    * every one of the 10 P per-variant energies (net outputs) within relative
      1e-5 of the reference's, as a maximum;
    * per-body energies (half the energy of each pair a body belongs to) within
      1e-5 of the body's summed pair-energy magnitudes, and the pair-energy sum
      likewise;
    * the kernel's forces and torques are the reference's forward differences,
      clip and scatter of its own energies (to float-atomic order);
    * against FP64 finite differences the forces and torques deviate no more
      than twice the reference's own FP32 deviation (+0.05) at the 50/90/99 %
      quantiles (relative 1e-5 per force is below the FP32 finite-difference
      noise of any implementation: an energy ulp over dx = 1e-5 is 0.06 force
      units here)."""
    c = load_case("cube_R64")
    shape, hyp, layers = case_shape(c), _hyp(c), case_model(c)
    pairs = c["pairs0"]
    P, N = len(pairs), len(c["pos0"])
    F, T, pe, e = gh.fused_forces(c["pos0"], c["orient0"], c["L"], pairs, shape, hyp, layers, "relu",
                                  method="amlp_forces_fd_energies")
    e_ref = c["e0"].astype(np.float64)
    assert e.shape == e_ref.shape and np.isfinite(e).all()
    rel = np.abs(e - e_ref) / np.maximum(np.abs(e_ref), 1e-2 * np.abs(e_ref).max())
    assert rel.max() <= 1e-5, f"max per-variant energy error {rel.max():.3g}"
    en_min32 = np.float64(np.float32(shape["en_min"]))
    rng32 = np.float64(np.float32(np.float32(shape["en_max"]) - np.float32(shape["en_min"])))
    Eg, Er = en_min32 + rng32 * e[:P].astype(np.float64), en_min32 + rng32 * e_ref[:P]
    body = lambda E: 0.5 * (np.bincount(pairs[:, 0], E, N) + np.bincount(pairs[:, 1], E, N))  # noqa: E731
    mag = body(np.abs(Er))
    has = mag > 0
    assert (np.abs(body(Eg) - body(Er))[has] / mag[has]).max() <= 1e-5
    assert abs(pe - Er.sum()) <= 1e-5 * np.abs(Er).sum()
    # the kernel's differences, clip and scatter are the reference's, applied to its own energies
    Fp, Ti, Tj = nep.fd_forces(e, P, 1e-5, 1e-5, shape["en_min"], shape["en_max"])
    Fo, To = nep.scatter(pairs, Fp, Ti, Tj, N)
    np.testing.assert_allclose(F, Fo, rtol=0, atol=1e-5 * max(1.0, np.abs(Fo).max()))
    np.testing.assert_allclose(T, To, rtol=0, atol=1e-5 * max(1.0, np.abs(To).max()))
    o64 = _fd64(c, shape, hyp, layers)
    for got, ref, want in ((F, c["F0"], o64["forces"]), (T, c["T0"], o64["torques"])):
        ref_err, gpu_err = np.abs(ref - want), np.abs(got - want)
        for q in (0.5, 0.9, 0.99):
            assert np.quantile(gpu_err, q) <= 2 * np.quantile(ref_err, q) + 0.05, q


def _split_forces(c, shape, hyp, layers, act="relu"):
    pairs = c["pairs0"]
    g = gh.descriptors(c["pos0"], c["orient0"], c["L"], pairs, shape, hyp)
    e = gh.mlp_energy(layers, act, g)
    return gh.fd_scatter(e, pairs, len(c["pos0"]), shape) + (e,)


@pytest.mark.parametrize("name", CASES)
def test_split_fd_forces_statistical(name):
    c = load_case(name)
    shape, hyp, layers = case_shape(c), _hyp(c), case_model(c)
    F, T, pe, e = _split_forces(c, shape, hyp, layers)
    o64 = _fd64(c, shape, hyp, layers)
    ref_err = np.abs(c["F0"] - o64["forces"])
    gpu_err = np.abs(F - o64["forces"])
    for q in (0.5, 0.9, 0.99):
        assert np.quantile(gpu_err, q) <= 2 * np.quantile(ref_err, q) + 0.05, q
    ref_err_t = np.abs(c["T0"] - o64["torques"])
    gpu_err_t = np.abs(T - o64["torques"])
    for q in (0.5, 0.9, 0.99):
        assert np.quantile(gpu_err_t, q) <= 2 * np.quantile(ref_err_t, q) + 0.05, q
    P = len(c["pairs0"])
    rng = shape["en_max"] - shape["en_min"]
    pe64 = np.sum(shape["en_min"] + rng * o64["e_all"][:P])
    pe_ref = np.sum(shape["en_min"] + rng * c["e0"][:P].astype(np.float64))
    assert abs(pe - pe64) <= 2 * abs(pe_ref - pe64) + 1e-6 * rng * P


@pytest.mark.parametrize("act,widths", [("tanh", (64, 64)), ("relu", (64, 32))])
def test_fused_equals_split_statistically(act, widths):
    from amlp.engine import EnergyNet
    s = make_state(500, "cube26", 0.45, seed=11)
    shape = SHAPES["cube26"]
    vp, _ = gh.nlist(s.pos, s.L, 4.5)
    pairs = gh.pair_filter(s.pos, s.L, 2.5, vp)
    net = EnergyNet.xavier(47, widths, act, seed=5, device="cpu")
    c = dict(pos0=s.pos, orient0=s.orient, L=s.L, pairs0=pairs)
    Fs, Ts, pes, e = _split_forces(c, shape, (10, 8, 4), net.layers, act)
    Ff, Tf, pef = gh.fused_forces(s.pos, s.orient, s.L, pairs, shape, (10, 8, 4), net.layers, act)
    assert abs(pef - pes) <= 1e-5 * max(1.0, abs(pes))
    o64 = nep.pair_forces(s.pos, s.orient, pairs, s.L, shape, (10, 8, 4), net.layers, act, dt=np.float64, form="sh")
    es = np.abs(Fs - o64["forces"])
    ef = np.abs(Ff - o64["forces"])
    for q in (0.5, 0.9, 0.99):
        assert np.quantile(ef, q) <= 2 * np.quantile(es, q) + 0.05


# ----------------------------------------------------------------------------- integrator
@pytest.mark.parametrize("name", ["th_C104", "cube_C104"])
def test_integrator_vs_oracle(name):
    """Step two + step one on the GPU with the reference's forces of step 0, against the FP32 oracle."""
    import ctypes
    from amlp._lib import Nvt, Thermostat, call, size_query
    c = load_case(name)
    N = len(c["pos0"])
    st = nep.NVTState(c["pos0"], c["vel0"], c["orient0"], c["angmom0"], c["mass"], c["moi"], c["L"],
                      float(c["kT"]), float(c["dt"]))
    dev = gh.DEV
    pos, vel, q, p = gh.t32(c["pos0"]), gh.t32(c["vel0"]), gh.t32(c["orient0"]), gh.t32(c["angmom0"])
    mass = gh.t32(c["mass"])
    F, T = gh.t32(c["F0"]), gh.t32(c["T0"])
    accel = torch.zeros(N, 3, device=dev)
    dp = torch.zeros(N, 4, device=dev)
    prm = Nvt()
    prm.dt, prm.tau, prm.kT = float(c["dt"]), float(np.float32(100 * c["dt"])), float(c["kT"])
    prm.n_dof, prm.rn_dof = float((N - 1) * 3), float(3 * N)
    for k in range(3):
        prm.moi[k] = float(c["moi"][k])
    prm.box, prm.nve = float(c["L"]), 0
    th = Thermostat()
    th.xi, th.eta, th.xi_rot, th.eta_rot, th.thermo_fac = (-0.0317711, 0.108609, 0.00814227, -0.014238, 1.00011)
    th_t = torch.frombuffer(bytearray(bytes(th)), dtype=torch.uint8).to(dev)
    ws = torch.empty(size_query("amlp_nvt_workspace_bytes", N), dtype=torch.uint8, device=dev)
    s = gh.stream()
    call("amlp_nvt_init", vel.data_ptr(), q.data_ptr(), p.data_ptr(), mass.data_ptr(), N, ctypes.byref(prm), 1,
         th_t.data_ptr(), ws.data_ptr(), ws.numel(), s)
    call("amlp_nvt_step_two", vel.data_ptr(), accel.data_ptr(), F.data_ptr(), mass.data_ptr(), q.data_ptr(),
         T.data_ptr(), p.data_ptr(), dp.data_ptr(), N, ctypes.byref(prm), th_t.data_ptr(), s)
    call("amlp_nvt_step_one", pos.data_ptr(), vel.data_ptr(), accel.data_ptr(), q.data_ptr(), p.data_ptr(),
         dp.data_ptr(), mass.data_ptr(), N, ctypes.byref(prm), th_t.data_ptr(), ws.data_ptr(), ws.numel(), s)
    st.step_two(c["F0"], c["T0"])
    st.step_one()
    # same forces as the reference -> the reference's state after one step
    for got, ref, ref_run in ((pos, st.pos, c["pos_s1"]), (vel, st.vel, c["vel_s1"]), (q, st.orient, c["orient_s1"]),
                              (p, st.angmom, c["angmom_s1"])):
        g = got.cpu().numpy()
        np.testing.assert_allclose(g, ref, rtol=2e-6, atol=2e-6 * np.abs(ref).max())
        np.testing.assert_allclose(g, ref_run, rtol=2e-6, atol=2e-6 * np.abs(ref_run).max())
    thr = Thermostat.from_buffer_copy(bytes(th_t.cpu().numpy().tobytes()))
    np.testing.assert_allclose([thr.xi, thr.eta, thr.xi_rot, thr.eta_rot, thr.thermo_fac], c["thermo_s1"], rtol=1e-5)
    np.testing.assert_allclose([thr.ke_t, thr.ke_r], [st.ke_t, st.ke_r], rtol=1e-5)


def test_integrator_large_n_no_fixed_grid():
    """N far above the reference's fixed grids (N <= 1706): every body moves."""
    from amlp.engine import EnergyNet, Hypers, System
    s = make_state(20000, "tetra16", 0.2, seed=9)
    net = EnergyNet.xavier(47, (64, 64), "tanh", seed=1, device=gh.DEV)
    sys_ = System(s, "tetra16", Hypers(), net, kT=1.0, dt=0.005, device=gh.DEV)
    p0 = sys_.pos.clone()
    sys_.step("fd")
    torch.cuda.synchronize()
    moved = (sys_.pos - p0).abs().sum(dim=1) > 0
    assert bool(moved.all())


# ----------------------------------------------------------------------------- system
def test_system_run_graph_rebuilds_and_matches_eager():
    from amlp.engine import EnergyNet, Hypers, System
    s = make_state(1000, "cube26", 0.30, seed=0)
    net = EnergyNet.xavier(47, (64, 64), "tanh", seed=0, device=gh.DEV)
    a = System(s, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=gh.DEV)
    b = System(s, "cube26", Hypers(), net, kT=1.0, dt=0.005, device=gh.DEV)
    a.run(1, graph=True)
    b.step()
    torch.cuda.synchronize()
    # one step: only the order of the float atomics differs
    assert torch.allclose(a.pos, b.pos, atol=1e-5) and torch.allclose(a.vel, b.vel, atol=1e-3)
    a.run(205, graph=True)  # crosses two Verlet rebuilds
    torch.cuda.synchronize()
    pos = a.pos.cpu().numpy()
    ref = nlist.sorted_pairs(nlist.reference_pairs(pos, a.L, a.r_verlet))
    a.build_nlist()
    assert np.array_equal(a.verlet_pairs().astype(np.int64), ref)
    assert np.isfinite(a.conserved_quantity())


# ----------------------------------------------------------------------------- adjoint
def _adjoint_case(shape_name, n, phi, seed, widths, act, pair_limit=None, method="amlp_forces_adjoint",
                  relu_margin=None):
    from amlp.engine import EnergyNet
    from oracle import adjoint
    s = make_state(n, shape_name, phi, seed=seed)
    shape = SHAPES[shape_name]
    vp, _ = gh.nlist(s.pos, s.L, shape["cutoff"] + 2.0)
    pairs = gh.pair_filter(s.pos, s.L, shape["cutoff"], vp)
    if pair_limit:
        pairs = pairs[:pair_limit]
    net = EnergyNet.xavier(47, widths, act, seed=seed + 10, device="cpu")
    if relu_margin is not None:
        # keep the pairs whose every hidden pre-activation is clear of the ReLU kink
        m = adjoint.relu_margin(s.pos, s.orient, pairs, s.L, shape, (10, 8, 4), net.layers)
        pairs = pairs[m > relu_margin]
    F, T, pe = gh.fused_forces(s.pos, s.orient, s.L, pairs, shape, (10, 8, 4), net.layers, act, method=method)
    from amlp import _lib
    assert _lib.device_error() == 0
    ref = adjoint.exact_pair_forces(s.pos, s.orient, pairs, s.L, shape, (10, 8, 4), net.layers, act)
    return F, T, pe, ref


@pytest.mark.parametrize("shape_name,phi,widths,act", [("cube26", 0.45, (64, 64), "tanh"),
                                                       ("tetra16", 0.40, (64, 64, 64), "silu"),
                                                       ("cyl24", 0.35, (48, 32), "silu")])
def test_adjoint_forces_vs_fp64_exact(shape_name, phi, widths, act):
    """Adjoint kernel (FP32 descriptor, split-bf16 tensor-core net) against the
    FP64 exact derivative: relative error <= 1e-3 (norm over all bodies)."""
    F, T, pe, ref = _adjoint_case(shape_name, 600, phi, 7, widths, act)
    for got, want in ((F, ref["forces"]), (T, ref["torques"])):
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= 1e-3, err
    pe_ref = ref["E"].sum()
    # pair energies through the bf16x3 net: 1e-4 of the summed magnitudes
    assert abs(pe - pe_ref) <= 1e-4 * max(1.0, np.abs(ref["E"]).sum())


def test_adjoint_partial_tile_and_single_pair():
    F, T, pe, ref = _adjoint_case("cube26", 300, 0.45, 3, (64, 64), "tanh", pair_limit=1)
    np.testing.assert_allclose(F, ref["forces"], atol=2e-3 * max(1.0, np.abs(ref["forces"]).max()))
    F, T, pe, ref = _adjoint_case("cube26", 300, 0.45, 3, (64, 64), "tanh", pair_limit=200)
    assert np.linalg.norm(F - ref["forces"]) / np.linalg.norm(ref["forces"]) <= 1e-3


@pytest.mark.parametrize("shape_name,phi,widths,act", [("tetra16", 0.40, (128, 128, 128), "silu"),
                                                       ("cyl24", 0.35, (128, 128), "silu"),
                                                       ("cube26", 0.45, (64, 64), "tanh")])
def test_adjoint_wide_nets_vs_fp64_exact(shape_name, phi, widths, act):
    """The three-kernel path for nets up to 128 wide (the differentiation and
    precision configurations' nets), same 1e-3 bar."""
    F, T, pe, ref = _adjoint_case(shape_name, 500, phi, 9, widths, act, method="amlp_forces_adjoint_wide")
    for got, want in ((F, ref["forces"]), (T, ref["torques"])):
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= 1e-3, err
    assert abs(pe - ref["E"].sum()) <= 1e-4 * max(1.0, np.abs(ref["E"]).sum())


@pytest.mark.parametrize("method", ["amlp_forces_adjoint", "amlp_forces_adjoint_wide", "amlp_forces_fd"])
def test_force_scatter_takes_pairs_in_any_order(method):
    """The fused kernels sum the i side of a warp's pairs over runs of equal i
    when the list is sorted (as amlp_pair_filter writes it); any other order,
    e.g. the reference's own cKDTree order, must give the same forces."""
    from amlp.engine import EnergyNet
    s = make_state(600, "cube26", 0.45, seed=13)
    shape = SHAPES["cube26"]
    vp, _ = gh.nlist(s.pos, s.L, 4.5)
    pairs = gh.pair_filter(s.pos, s.L, 2.5, vp)
    shuffled = pairs[np.random.default_rng(1).permutation(len(pairs))]
    net = EnergyNet.xavier(47, (64, 64), "tanh", seed=2, device="cpu")
    a = gh.fused_forces(s.pos, s.orient, s.L, pairs, shape, (10, 8, 4), net.layers, "tanh", method=method)
    b = gh.fused_forces(s.pos, s.orient, s.L, shuffled, shape, (10, 8, 4), net.layers, "tanh", method=method)
    for x, y in zip(a[:2], b[:2]):
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-5 * max(1.0, np.abs(x).max()))
    assert abs(a[2] - b[2]) <= 1e-9 * max(1.0, abs(a[2]))


@pytest.mark.parametrize("name", ["th_C104", "th_C100", "cube_C104"])
def test_adjoint_reference_models_vs_fp64_exact(name):
    """The reference's own trained models (TheEnergyNet(150, 3, D): four 150-wide
    ReLU layers, Sim.py:60, ForceEvaluator.py:6-26; D = 47 for the C104 models,
    121 for C100 with its direct-form descriptor passes) on the tensor-core adjoint
    path (amlp_forces_adjoint_wide) against the FP64 exact derivative of the same
    pair energy: relative 1e-3 on forces and torques (norm over bodies)."""
    from amlp import _lib
    from oracle import adjoint
    c = load_case(name)
    shape, hyp, layers = case_shape(c), _hyp(c), case_model(c)
    assert [W.shape[0] for W, _ in layers[:-1]] == [150] * 4
    pairs = c["pairs0"]
    F, T, pe = gh.fused_forces(c["pos0"], c["orient0"], c["L"], pairs, shape, hyp, layers, "relu",
                               method="amlp_forces_adjoint_wide")
    assert _lib.device_error() == 0
    ref = adjoint.exact_pair_forces(c["pos0"], c["orient0"], pairs, c["L"], shape, hyp, layers, "relu")
    for got, want in ((F, ref["forces"]), (T, ref["torques"])):
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= 1e-3, err
    assert abs(pe - ref["E"].sum()) <= 1e-4 * max(1.0, np.abs(ref["E"]).sum())


@pytest.mark.parametrize("widths,act", [((150, 150, 150, 150), "relu"), ((150, 150, 150), "silu"),
                                        ((128, 128, 128, 128), "tanh"), ((160, 96), "relu")])
def test_adjoint_wide_nets_to_160_and_four_layers(widths, act):
    """k_mlp_grad at the widths and depths beyond the fused kernel: up to 160 wide
    and four hidden layers; ReLU derivatives kept as bits, smooth ones in TMEM.

    A random ReLU net's forces jump where a hidden pre-activation crosses zero:
    flipping the kinks of the pairs within 1e-5 (relative) of one moves these
    forces by about 1 %, so the ReLU cases keep the pairs whose every
    pre-activation is more than 1e-3 of its layer's mean |z| from zero (about
    two thirds of them); there the FP32 path and the FP64 oracle take the same
    branch of every ReLU."""
    margin = 1e-3 if act == "relu" else None
    F, T, pe, ref = _adjoint_case("cube26", 500, 0.45, 17, widths, act, method="amlp_forces_adjoint_wide",
                                  relu_margin=margin)
    for got, want in ((F, ref["forces"]), (T, ref["torques"])):
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= 1e-3, err
    assert abs(pe - ref["E"].sum()) <= 1e-4 * max(1.0, np.abs(ref["E"]).sum())


@pytest.mark.parametrize("shape_name,hyp", [("th_v1", (10, 8, 4)), ("cube26", (10, 8, 4))])
def test_stage_timing_of_the_wide_path(shape_name, hyp):
    """amlp_stage_timing / amlp_stage_times: three positive stage times whose sum
    stays within the whole call's event time, and the same forces with the
    events on as without them."""
    import ctypes
    from amlp import _lib
    from amlp.engine import EnergyNet
    L = {"th_v1": 24.0}.get(shape_name)
    s = make_state(400, shape_name, 0.1 if L else 0.45, seed=3, L=L)
    shape = SHAPES[shape_name]
    vp, _ = gh.nlist(s.pos, s.L, shape["cutoff"] + 2.0)
    pairs = gh.pair_filter(s.pos, s.L, shape["cutoff"], vp)
    net = EnergyNet.xavier(47, (150, 150), "relu", seed=4, device="cpu")
    ref = gh.fused_forces(s.pos, s.orient, s.L, pairs, shape, hyp, net.layers, "relu",
                          method="amlp_forces_adjoint_wide")
    _lib.call("amlp_stage_timing", 1)
    try:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        got = gh.fused_forces(s.pos, s.orient, s.L, pairs, shape, hyp, net.layers, "relu",
                              method="amlp_forces_adjoint_wide")
        e1.record()
        torch.cuda.synchronize()
        ms = (ctypes.c_float * 3)()
        _lib.call("amlp_stage_times", ms)
    finally:
        _lib.call("amlp_stage_timing", 0)
    assert all(m > 0.0 for m in ms)
    assert sum(ms) <= e0.elapsed_time(e1)
    for a, b in zip(got[:2], ref[:2]):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-5 * max(1.0, np.abs(b).max()))


def test_direct_form_large_clouds_and_empty_lists():
    """The direct-form passes at large clouds (cube26 with the hypers (10, 10,
    10): 52 points, 52 KB of shared memory per block, above the default 48 KB),
    against the FP64 descriptor and exact derivative; and an empty pair list,
    which leaves the forces zero. Each thread sums the 1,326 point pairs of a
    52-point cloud in one FP32 register, and the Legendre terms cancel, so the
    descriptor is checked against each row's largest entry (1e-5 of it) rather
    than entry by entry (the reference's C100 shapes, 8 to 14 points, meet the
    entry-wise bar in test_pair_descriptors_vs_fp64)."""
    from amlp.engine import EnergyNet
    from oracle import adjoint
    s = make_state(200, "cube26", 0.45, seed=21)
    shape = SHAPES["cube26"]
    vp, _ = gh.nlist(s.pos, s.L, shape["cutoff"] + 2.0)
    pairs = gh.pair_filter(s.pos, s.L, shape["cutoff"], vp)[:300]
    hyp = (10, 10, 10)
    g = gh.pair_descriptors(s.pos, s.orient, s.L, pairs, shape, hyp, ld=124)
    _, _, t = nep.min_image_filter(s.pos, pairs, s.L, shape["cutoff"], np.float64)
    c1, _ = nep.pair_clouds(s.orient, pairs, t, shape["pts"], np.float64)
    g64 = nep.descriptor(c1, hyp, shape["nep_cutoff"], np.float64)
    row_scale = np.abs(g64).max(axis=1, keepdims=True)
    assert (np.abs(g[:, :121] - g64) / row_scale).max() <= 1e-5
    assert np.all(g[:, 121:] == 0.0)
    net = EnergyNet.xavier(121, (64, 64), "tanh", seed=22, device="cpu")
    F, T, pe = gh.fused_forces(s.pos, s.orient, s.L, pairs, shape, hyp, net.layers, "tanh",
                               method="amlp_forces_adjoint_wide")
    ref = adjoint.exact_pair_forces(s.pos, s.orient, pairs, s.L, shape, hyp, net.layers, "tanh")
    for got, want in ((F, ref["forces"]), (T, ref["torques"])):
        assert np.linalg.norm(got - want) / np.linalg.norm(want) <= 1e-3
    F0, T0, pe0 = gh.fused_forces(s.pos, s.orient, s.L, pairs[:0], shape, hyp, net.layers, "tanh",
                                  method="amlp_forces_adjoint_wide")
    assert not F0.any() and not T0.any() and pe0 == 0.0
