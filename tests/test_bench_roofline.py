"""The benchmark's roofline arithmetic on the CPU: the algorithmic FLOP counts of
both descriptor forms, and the per-stage roofline of the wide force pass (each
stage against its own peak, the slowest stage on the line)."""
import pytest

import bench


def test_descriptor_flops_of_both_forms():
    # harmonic form, (10, 8, 4): 573 Nd + 432
    assert bench.descriptor_flops(52) == 573 * 52 + 432
    # direct form, per unordered point pair (dot 5 + Legendre 4 (lmax - 1) + (nang+1) products
    # + 2 (nang+1) lmax) and per point (42 + 2 (nang+1) + (nrad+1))
    assert bench.descriptor_flops(8, (10, 10, 10), direct=True) == 272 * 28 + 75 * 8
    assert bench.descriptor_flops(8, (10, 8, 4), direct=True) == 98 * 28 + 71 * 8
    # the wide path takes the direct form for (10, 10, 10) and for clouds of up to 12 points
    assert bench.uses_direct_form(8) and bench.uses_direct_form(12) and not bench.uses_direct_form(14)
    assert bench.uses_direct_form(52, (10, 10, 10))


@pytest.mark.parametrize("stage_ms,dominant", [((0.1, 0.94, 0.26), "k_mlp_grad"),
                                               ((0.5, 0.2, 0.9), "k_desc_direct_bwd")])
def test_wide_roofline_takes_the_slowest_stage(monkeypatch, stage_ms, dominant):
    monkeypatch.setattr(bench, "SHAPE", "th_v1")
    monkeypatch.setattr(bench, "HYPERS", (10, 8, 4))
    monkeypatch.setattr(bench, "WIDTHS", (150, 150, 150, 150))
    P = 695382
    base = {"bound": "fp32", "kernel": "k_forces_adjoint", "peak_nominal": 74.4, "frac_of_nominal": 0.0}
    r = {"P": P, "stage_ms": list(stage_ms)}
    out = bench.wide_roofline(base, r, 47, 72.5, 1627.5)
    assert out["kernel"] == dominant
    names = [s["kernel"] for s in out["stages"]]
    assert names == ["k_desc_direct_fwd", "k_mlp_grad", "k_desc_direct_bwd"]
    fd1 = bench.descriptor_flops(8, (10, 8, 4), direct=True)
    fl_tc = bench.algorithmic_flops_per_pair("adjoint", nd=8, D=47, widths=(150,) * 4)[1]
    want = [(fd1, 72.5), (fl_tc, 1627.5), (2 * fd1, 72.5)]
    for st, ms, (fl, peak) in zip(out["stages"], stage_ms, want):
        assert st["achieved"] == pytest.approx(fl * P / (ms / 1e3) / 1e12)
        assert st["frac"] == pytest.approx(st["achieved"] / peak)
    assert out["stages"][1]["bound"] == "tensor"
    assert out["stages"][1]["frac_executed"] == pytest.approx(3 * out["stages"][1]["frac"])
    assert out["bound"] == ("tensor" if dominant == "k_mlp_grad" else "fp32")
    assert "peak_nominal" not in out
