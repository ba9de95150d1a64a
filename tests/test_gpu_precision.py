"""Precision of the tensor-core path against the FP64 oracle on the precision
workload: 262,144 twisted cylinders (cyl24) at packing fraction 0.35, seed 3
(about 3 M filtered pairs), net 47->128->128->1 SiLU (the soft-repulsion fit of
``golden/make_soft_potential.py``).

The force pass (``System.compute_forces('adjoint')``: FP32 descriptors, net on
the tensor cores as bf16x3 splits with FP32 accumulation, FP64 energy sum) is
compared on 256 random bodies (all of their pairs) with the FP64 exact
derivative, clipped per pair as the force path does:
* forces and torques: relative error (norm over the bodies) <= 1e-3;
* pair energies: the same kernel run on the sampled bodies' pairs alone sums
  their energies to within 1e-4 of the summed magnitudes; per pair, the FP32
  net of ``PairEnergy`` is within 1e-4 of the energy range.
With ``AMLP_REPORT_DIR`` set, the measured errors are written to
``precision_cyl24.json`` there.
"""
import json
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

import gpu_helpers as gh  # noqa: E402
from amlp import _lib  # noqa: E402
from amlp.autograd import PairModel, pair_energies  # noqa: E402
from amlp.configs import make_state  # noqa: E402
from amlp.engine import EnergyNet, Hypers, System  # noqa: E402
from oracle import adjoint  # noqa: E402
from oracle.shapes import SHAPES  # noqa: E402

DEV = torch.device("cuda:0")
MODEL = os.path.join(GOLDEN, "model_cyl24_soft.npz")


def _layers():
    z = np.load(MODEL)
    return [(z[f"W{k}"], z[f"b{k}"]) for k in range(len(z.files) // 2)]


@pytest.fixture(scope="module")
def cyl_case():
    if not os.path.exists(MODEL):
        pytest.skip("model_cyl24_soft.npz not generated")
    st = make_state(262144, "cyl24", 0.35, seed=3)
    layers = _layers()
    net = EnergyNet(layers, "silu", DEV)
    s = System(st, "cyl24", Hypers(), net, kT=1.0, dt=0.005, device=DEV)
    s.compute_forces("adjoint")
    torch.cuda.synchronize()
    assert _lib.device_error() == 0
    P = int(s.nf.item())
    pairs = s.fpairs[:P].cpu().numpy().astype(np.int64)
    bodies = np.sort(np.random.default_rng(33).choice(st.N, 256, replace=False))
    sub = pairs[np.isin(pairs[:, 0], bodies) | np.isin(pairs[:, 1], bodies)]
    shape = SHAPES["cyl24"]
    ref = adjoint.exact_pair_forces(st.pos, st.orient, sub, st.L, shape, (10, 8, 4), layers, "silu", clip=True)
    return dict(st=st, s=s, layers=layers, P=P, bodies=bodies, sub=sub, ref=ref, shape=shape,
                F=s.F.cpu().numpy().astype(np.float64), T=s.T.cpu().numpy().astype(np.float64))


def _report(key, values):
    d = os.environ.get("AMLP_REPORT_DIR")
    if not d:
        return
    path = os.path.join(d, "precision_cyl24.json")
    data = json.load(open(path)) if os.path.exists(path) else {}
    data[key] = values
    with open(path, "w") as fh:
        json.dump(data, fh, indent=1)


def _rel(got, want):
    return float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30))


def test_pairs_per_step(cyl_case):
    assert 2_500_000 < cyl_case["P"] < 3_500_000


def test_forces_torques_vs_fp64(cyl_case):
    c = cyl_case
    b = c["bodies"]
    F, T = c["F"][b], c["T"][b]
    Fr, Tr = c["ref"]["forces"][b], c["ref"]["torques"][b]
    errs = {"force_rel_norm": _rel(F, Fr), "torque_rel_norm": _rel(T, Tr),
            "force_max_abs": float(np.abs(F - Fr).max()), "torque_max_abs": float(np.abs(T - Tr).max()),
            "force_rms": float(np.sqrt(np.mean(Fr ** 2))), "torque_rms": float(np.sqrt(np.mean(Tr ** 2))),
            "bodies": int(len(b)), "pairs": int(len(c["sub"])), "filtered_pairs_total": int(c["P"])}
    _report("forces_torques", errs)
    assert errs["force_rel_norm"] <= 1e-3, errs
    assert errs["torque_rel_norm"] <= 1e-3, errs


def test_pair_energies_vs_fp64(cyl_case):
    c = cyl_case
    st, sub, shape = c["st"], c["sub"], c["shape"]
    E64 = c["ref"]["E"]
    # the tensor-core force kernel on the sampled pairs alone: its FP64 energy sum
    _, _, pe = gh.fused_forces(st.pos, st.orient, st.L, sub, shape, (10, 8, 4), c["layers"], "silu",
                               method="amlp_forces_adjoint_wide")
    # per pair: the FP32 net behind PairEnergy
    model = PairModel("cyl24", Hypers(), [47, 128, 128, 1], "silu", DEV)
    net = EnergyNet(c["layers"], "silu", DEV)
    E = pair_energies(torch.tensor(st.pos, device=DEV), torch.tensor(st.orient, device=DEV), net.d_w,
                      torch.tensor(sub.astype(np.int32), device=DEV), st.L, model).cpu().numpy()
    rng = shape["en_max"] - shape["en_min"]
    errs = {"tensor_core_sum_rel": float(abs(pe - E64.sum()) / np.abs(E64).sum()),
            "tensor_core_sum_abs": float(abs(pe - E64.sum())), "sum_fp64": float(E64.sum()),
            "fp32_pair_max_abs": float(np.abs(E - E64).max()), "fp32_pair_rms": float(np.sqrt(np.mean((E - E64) ** 2))),
            "pair_energy_rms": float(np.sqrt(np.mean(E64 ** 2))), "pairs": int(len(sub))}
    _report("energies", errs)
    assert errs["tensor_core_sum_rel"] <= 1e-4, errs
    assert errs["fp32_pair_max_abs"] <= 1e-4 * rng, errs
