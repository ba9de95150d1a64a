"""Pins the oracle against the golden fixtures produced by the reference's own
classes (``tests/golden/make_golden.py``). The oracle's FP32 path follows the
reference's operation order, so the comparisons are bitwise."""
import numpy as np
import pytest

from conftest import case_model, case_shape, load_case
from oracle import nep, nlist
from oracle.sim import OracleSim

CASES = ["th_C104", "th_C100", "cube_C104", "cube_R64"]


def _sim(c, steps_dt=np.float32):
    return OracleSim(c["pos0"], c["vel0"], c["orient0"], c["angmom0"], c["mass"], c["moi"], c["L"],
                     case_shape(c), tuple(int(h) for h in c["hypers"][:3]), case_model(c), "relu",
                     float(c["kT"]), float(c["dt"]), dt=steps_dt)


@pytest.mark.parametrize("name", CASES)
def test_nlist_is_reference_call(name):
    c = load_case(name)
    shape = case_shape(c)
    p = nlist.sorted_pairs(nlist.reference_pairs(c["pos0"], c["L"], shape["cutoff"] + 2.0))
    assert np.array_equal(p, c["nlist0"])
    bf = nlist.sorted_pairs(nlist.brute_force_pairs(c["pos0"], c["L"], shape["cutoff"] + 2.0))
    assert np.array_equal(bf, c["nlist0"])


@pytest.mark.parametrize("name", CASES)
def test_step0_bitwise(name):
    c = load_case(name)
    s = _sim(c)
    F, T = s.forces()
    o = s.last
    P = int(c["P0"])
    assert o["P"] == P
    assert np.array_equal(o["pairs"], c["pairs0"])
    g = o["g_all"].reshape(10, P, -1)[:, :c["g0"].shape[1]]
    assert np.array_equal(g, c["g0"])
    assert np.array_equal(o["e_all"], c["e0"])
    en_range = case_shape(c)["en_max"] - case_shape(c)["en_min"]
    assert np.array_equal(F, c["F0"]) and np.array_equal(T, c["T0"])
    # unclipped gradients match the reference's too
    e = o["e_all"].reshape(10, P)
    np.testing.assert_array_equal(-(e[1] - e[0]) / np.float32(1e-5), c["Fgrad0"][:, 0])
    assert en_range > 0


@pytest.mark.parametrize("name", CASES)
def test_steps_bitwise(name):
    c = load_case(name)
    s = _sim(c)
    steps = sorted(int(k.split("_s")[1]) for k in c if k.startswith("pos_s"))
    for k in steps:
        s.run(k - s.timestep)
        st = s.state
        for key, arr in (("pos", st.pos), ("vel", st.vel), ("orient", st.orient), ("angmom", st.angmom)):
            np.testing.assert_array_equal(arr, c[f"{key}_s{k}"], err_msg=f"{key} after {k} steps")
        th = np.array(list(st.th.var) + [st.th.thermo_fac], np.float32)
        np.testing.assert_array_equal(th, c[f"thermo_s{k}"])


def test_long_run_with_rebuilds_bitwise():
    c = load_case("th_C104")
    s = _sim(c)
    frames = []
    s.run(int(c["long_steps"]), on_dump=lambda t, st: frames.append((t, st.pos.copy())), dump=int(c["long_dump"]))
    np.testing.assert_array_equal(s.state.pos, c["pos_long"])
    np.testing.assert_array_equal(s.state.angmom, c["angmom_long"])
    assert [t for t, _ in frames] == list(c["long_frames_step"])
    for (t, p), q in zip(frames, c["long_frames_pos"]):
        np.testing.assert_array_equal(p, q)


def test_sh_form_equals_direct_fp64():
    c = load_case("cube_C104")
    s = _sim(c, np.float64)
    st = s.state
    a = nep.pair_forces(st.pos, st.orient, s.nlist, st.L, s.shape, s.hypers, s.layers, "relu", dt=np.float64)
    b = nep.pair_forces(st.pos, st.orient, s.nlist, st.L, s.shape, s.hypers, s.layers, "relu", dt=np.float64,
                        form="sh")
    np.testing.assert_allclose(b["g_all"], a["g_all"], rtol=0, atol=1e-10 * np.abs(a["g_all"]).max())


def test_sh_addition_theorem_lmax10():
    rng = np.random.default_rng(0)
    u = rng.standard_normal((50, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    Y = nep.sh_scaled(u, 10)
    cos = u @ u.T
    k = 0
    from scipy.special import eval_legendre
    for l in range(1, 11):
        blk = Y[:, k:k + 2 * l + 1]
        np.testing.assert_allclose(blk @ blk.T, eval_legendre(l, cos), atol=1e-11)
        k += 2 * l + 1
