"""Benchmark: particle-steps/s of the NVT step of 131,072 rigid cubes on B200.

Workload (one "step" = one full time step: pair filter, force pass, both NVT
halves; the Verlet list is rebuilt at the first timed step and every 100 steps
after it, so every timed window holds ceil(K / 100) rebuilds -- for K < 100
more than the amortised 1/100 share):
131,072 cube26 bodies at packing fraction 0.45, jittered lattice, random unit
quaternions, seed 1, NEP hypers (10, 8, 4), FFNN 47 -> 64 -> 64 -> 1 tanh with
seeded Xavier weights, dt 0.005, kT 1.0 (synthetic; no dataset involved).

Arms:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--method both|fd|adjoint]
      "value" is the tuned method (exact adjoint forces, net on the tensor
      cores); with "both" the plain FP32 finite-difference drop-in is measured
      in the same run under "plain"
  python bench.py --impl reference ...   the reference's step on the host
      cores through the oracle (bit-identical to the reference's own classes),
      on a process pool; each timed step covers a random sample of the bodies
      (their pair filter and force pass) and both NVT halves of all bodies, and
      "value" counts the sampled bodies only. The arm imports nothing of the
      product package (oracle.workload generates the same state and net).

With --gpus N > 1 (launched by torch.distributed.run) every rank runs an
independent replica on its own GPU (weak scaling, no data-path collective);
time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "anisotropic-ml_b200"))

N_BODIES = 131072
PHI = 0.45
SEED = 1
WIDTHS = (64, 64)
ACT = "tanh"
DT = 0.005
KT = 1.0
METRIC = "particle-steps/s"
WORKLOAD = "nvt-step-131072-cube26-phi0.45-mlp47x64x64x1-tanh"
SHAPE = "cube26"
NET = "xavier"
IS_BENCHMARK = True  # the default workload (serving leg, CPU baseline and ncu traffic belong to it)

# The other configurations, measured with --workload (the default is the cube workload above): the
# small 1,000-cube system (packing fraction 0.30, seed 0),
# 65,536 regular tetrahedra of 16 points (differentiation workload) and 262,144 twisted cylinders
# (precision workload), both with the soft-repulsion nets trained by
# tests/golden/make_soft_potential.py (random nets make the dynamics blow up at these sizes). The
# last two have 128-wide nets, so their tuned path is the wide adjoint and the fused plain kernel
# (widths <= 64) does not apply.
WORKLOADS = {
    "cube26": dict(n=131072, shape="cube26", phi=0.45, seed=1, widths=(64, 64), act="tanh", net="xavier"),
    "cube1000": dict(n=1000, shape="cube26", phi=0.30, seed=0, widths=(64, 64), act="tanh", net="xavier"),
    "tetra16": dict(n=65536, shape="tetra16", phi=0.40, seed=2, widths=(128, 128, 128), act="silu", net="trained"),
    "cyl24": dict(n=262144, shape="cyl24", phi=0.35, seed=3, widths=(128, 128), act="silu", net="trained"),
    # the reference's own trained models (TheEnergyNet(150, 3, D), ReLU) on its th_v1 tetrahedra, at the
    # number density of its init files (200 bodies in a box of 33) and its temperature kT 0.5
    "th_C104": dict(n=262144, shape="th_v1", L=33.0 * (262144 / 200) ** (1 / 3), seed=4, widths=(150,) * 4,
                    act="relu", net="model_th_C104", hypers=(10, 8, 4), kT=0.5),
    "th_C100": dict(n=262144, shape="th_v1", L=33.0 * (262144 / 200) ** (1 / 3), seed=4, widths=(150,) * 4,
                    act="relu", net="model_th_C100", hypers=(10, 10, 10), kT=0.5),
}
HYPERS = (10, 8, 4)
BOX = None  # explicit box edge (workloads at a given number density instead of a packing fraction)

# kernels launched by each libamlp entry point (for the gpu_launches count)
LAUNCHES = {"amlp_nlist_build": 11, "amlp_pair_filter": 2, "amlp_forces_fd": 1, "amlp_forces_adjoint": 1,
            "amlp_nvt_step_two": 2, "amlp_nvt_step_one": 1}


# DRAM bytes (read + written) per filtered pair of one force launch, from an ncu capture of
# dram__bytes_read.sum + dram__bytes_write.sum at 32,768 cube26 bodies (436,636 pairs; the kernels'
# profiles give the command). The traffic grows with the pairs (a capture at 131,072 bodies gave the
# same bytes per pair), so the roofline's traffic is this figure times the launch's pairs.
DRAM_BYTES_PER_PAIR = {"adjoint": 5.340928e6 / 436636, "fd": 5.318912e6 / 436636}
# The wide path (nets wider than 64) stores each pair's descriptor row, harmonic sums and dE/dg in
# HBM between its three launches: the sum over k_adj_desc forward, k_mlp_grad and k_adj_desc backward
# captured at 32,768 cyl24 bodies (381,342 pairs). The per-pair rows do not depend on the shape or the
# net, so the figure serves every wide workload.
DRAM_BYTES_PER_PAIR["adjoint_wide"] = (4.141824e6 + 350.520064e6 + 79.480064e6 + 26.586624e6 + 409.184e6
                                       + 5.303552e6) / 381342
# Per stage of the wide path, keyed by (kernel, D): ncu dram__bytes_read.sum + dram__bytes_write.sum per
# pair at 32,768 th_v1 bodies (87,256 pairs; the profiles give the commands). The descriptor rows
# depend on D, not on the net or the shape.
STAGE_DRAM_BYTES_PER_PAIR = {
    # the harmonic-form passes (clouds of more than 12 points), 32,768 cyl24 bodies, 381,342 pairs
    ("k_adj_desc (forward)", 47): (4.141824e6 + 350.520064e6) / 381342,
    ("k_adj_desc (backward)", 47): (409.184e6 + 5.303552e6) / 381342,
    ("k_mlp_grad", 47): 18.56128e6 / 87256,
    ("k_mlp_grad", 121): (46.54e6 + 0.39e6) / 87257,
    ("k_desc_direct_fwd", 47): 1.64e6 / 87256,
    ("k_desc_direct_bwd", 47): 19.54e6 / 87256,
    ("k_desc_direct_fwd", 121): (2.888960e6 + 1.725440e6) / 87257,
    ("k_desc_direct_bwd", 121): (47.458304e6 + 0.022528e6) / 87257,
}


def uses_direct_form(nd: int, hypers=(10, 8, 4)) -> bool:
    """Whether the adjoint wide path runs the direct-form descriptor kernels: the
    hypers (10, 10, 10), and (10, 8, 4) clouds of at most 12 points (the
    library's own choice, kDirectMaxNd47)."""
    return tuple(hypers) != (10, 8, 4) or nd <= 12


def descriptor_flops(nd: int, hypers=(10, 8, 4), direct: bool = False) -> float:
    """Algorithmic FLOPs of one descriptor evaluation of an Nd-point cloud.
    Spherical-harmonic form (the plain path, and the adjoint path for (10, 8, 4)
    and larger clouds): per point the 2 (nang+1) K contraction over K = lmax
    (lmax + 2) harmonics plus their recurrences and the radial basis, 573 Nd + 432
    for (10, 8, 4) and 3,050 Nd + 250 for (10, 10, 10). Direct form: the sum over
    point pairs is symmetric, so per unordered pair a < b the dot product (5), the
    Legendre recurrences (4 (lmax - 1)), the (nang+1) products f_n(a) f_n(b) and
    the (nang+1) lmax multiply-adds, 272 FLOPs for (10, 10, 10) and 98 for
    (10, 8, 4); per point the radial basis (42), its diagonal term (2 (nang+1))
    and the radial sums (nrad+1)."""
    nrad, nang, lmax = (int(h) for h in hypers[:3])
    if direct:
        per_pair = 5 + 4 * (lmax - 1) + (nang + 1) + 2 * (nang + 1) * lmax
        per_point = 42 + 2 * (nang + 1) + (nrad + 1)
        return per_pair * nd * (nd - 1) / 2.0 + per_point * nd
    if tuple(hypers) == (10, 8, 4):
        return 573.0 * nd + 432.0
    return 3050.0 * nd + 250.0


def algorithmic_flops_per_pair(method: str, nd: int = 52, D: int = 47, widths=WIDTHS, hypers=(10, 8, 4)):
    """Algorithmic FLOPs per filtered pair as (FP32 SIMT part, tensor-core part):
    descriptor F_d per cloud evaluation (descriptor_flops), net F_n = 2 (sum of
    layer in x out). The plain methods evaluate 10 clouds and 10 nets per pair,
    all in FP32 SIMT; the adjoint one cloud + its backward (3 F_d, FP32 SIMT) and
    the net forward + backward (2 F_n) on the tensor cores."""
    dims = [D] + list(widths) + [1]
    fn = 2.0 * sum(dims[k] * dims[k + 1] for k in range(len(dims) - 1))
    if method in ("fd", "fd_split"):
        return 10.0 * (descriptor_flops(nd, hypers) + fn), 0.0
    wide = max(widths) > 64 or tuple(hypers) != (10, 8, 4)
    return 3.0 * descriptor_flops(nd, hypers, direct=wide and uses_direct_form(nd, hypers)), 2.0 * fn


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, gpu: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measure_fp32_peak(dev) -> float:
    """FP32 TFLOP/s of the library's multiply-add probe (amlp_fp32_fma_probe):
    best of three ~0.1 s launches, CUDA events on the launching stream."""
    import ctypes
    import torch
    from amlp import _lib
    out = torch.zeros(1, device=dev)
    stream = torch.cuda.current_stream()
    flops = ctypes.c_double(0.0)
    best = 0.0
    _lib.call("amlp_fp32_fma_probe", out.data_ptr(), 20000, ctypes.byref(flops), stream.cuda_stream)  # warm-up
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.call("amlp_fp32_fma_probe", out.data_ptr(), 1500000, ctypes.byref(flops), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        best = max(best, flops.value / (e0.elapsed_time(e1) / 1e3) / 1e12)
    return best


def measured_peaks() -> dict:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return {"hbm_gbs": d.get("hbm_gbs"), "bf16_tflops": d.get("bf16_tflops"),
                "sm_max_mhz": d.get("sm_max_mhz", 1965.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0, "source": "fallback"}


# ----------------------------------------------------------------------------- reference arm / CPU baseline
def common_config(world: int) -> dict:
    """The workload's description, the same in both arms."""
    return {"workload": WORKLOAD, "bodies": N_BODIES, "shape": SHAPE, "phi": PHI, "seed": SEED,
            "net": f"47x{'x'.join(str(w) for w in WIDTHS)}x1 {ACT} ({NET})", "dt": DT, "kT": KT,
            "nlist_every": 100, "parallelism": "replicas" if world > 1 else "single",
            "l2": "GPU arm: flushed between timed steps (256 MB write); CPU arm: not applicable"}


def _oracle_layers():
    """The workload's net from the oracle side (numpy only)."""
    import numpy as np
    from oracle import workload
    if NET == "trained":
        z = np.load(os.path.join(REPO, "tests", "golden", f"model_{SHAPE}_soft.npz"))
        return [(z[f"W{k}"], z[f"b{k}"]) for k in range(len(z.files) // 2)]
    layers = workload.xavier_layers(47, WIDTHS, SEED)
    if NET == "xavier_out0.05":
        W, b = layers[-1]
        layers[-1] = (W * np.float32(0.05), b)
    return layers


class CpuRun:
    """The reference's step on the host cores (oracle.workload.CpuStep): timed
    steps on random samples of `bodies_per_step` bodies, sized at set-up so that
    a step takes about `target_s` seconds."""

    def __init__(self, n, shape, phi, seed, target_s=2.0, workers=None):
        import numpy as np
        from oracle import workload
        self.np = np
        state = workload.make_state(n, shape, phi, kT=KT, seed=seed)
        self.n = n
        self.step = workload.CpuStep(state, shape, (10, 8, 4), _oracle_layers(), ACT, KT, DT, workers=workers)
        self.rng = np.random.default_rng(0)
        self.bodies = n
        if target_s is not None and n > 256:
            self.step.step(self._sample(256))  # the workers' first call loads their libraries
            t = self.step.step(self._sample(256))
            self.bodies = int(min(n, max(64, 256 * target_s / max(t, 1e-3))))

    def _sample(self, k):
        return None if k >= self.n else self.np.sort(self.rng.choice(self.n, size=k, replace=False))

    def timed(self, steps):
        times, pairs = [], 0
        for _ in range(steps):
            times.append(self.step.step(self._sample(self.bodies)))
            pairs += self.step.pairs_last
        return times, pairs

    def describe(self, pairs_per_step):
        full = self.bodies >= self.n
        what = "all bodies" if full else f"a random sample of {self.bodies} of the {self.n} bodies"
        return (f"each step: {what} (pair filter of the Verlet pairs they own, force pass of the "
                f"{pairs_per_step:.0f} filtered pairs on average: 10 FP32 finite-difference clouds, direct "
                f"descriptors, torch-CPU net, differences, clip, scatter) and both NVT halves of all {self.n} "
                f"bodies; the oracle's FP32 path (bit-identical to the reference's classes) on "
                f"{self.step.workers} worker processes; value counts the {'' if full else 'sampled '}bodies; "
                f"the Verlet rebuild (one cKDTree call, {self.step.t_nlist:.2f} s for all bodies, every 100 steps) "
                f"is outside the timed steps")

    def close(self):
        self.step.close()


def cpu_step_sample(steps: int = 5):
    """cpu_baseline leg of the GPU arm: a bounded run of the reference's step on the host cores."""
    run = CpuRun(N_BODIES, SHAPE, PHI, SEED)
    try:
        run.timed(1)
        times, pairs = run.timed(steps)
        t = statistics.mean(times)
        return {"value": run.bodies / t, "unit": "particle-steps/s", "cores": run.step.workers, "kind": "port",
                "sample": run.describe(pairs / steps), "bodies_per_step": run.bodies,
                "s_per_step": t, "extrapolated_s_per_full_step": t * N_BODIES / run.bodies}
    finally:
        run.close()


def _product_library_mapped() -> bool:
    try:
        with open("/proc/self/maps") as fh:
            return "libamlp.so" in fh.read()
    except OSError:
        return False


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    if SHAPE != "cube26":
        print(json.dumps({"impl": "reference", "unavailable": "the CPU arm is timed on the cube26 benchmark workload"}))
        return
    run = CpuRun(N_BODIES, SHAPE, PHI, SEED)
    try:
        run.timed(args.warmup)
        times, pairs = run.timed(args.steps)
    finally:
        run.close()
    per_step = statistics.mean(times)
    value = run.bodies / per_step
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded lattice, Xavier weights)",
            "config": common_config(world),
            "method": "fd (the reference's finite differences)",
            "sample": {"bodies_per_step": run.bodies, "bodies_total": N_BODIES,
                       "filtered_pairs_per_step": pairs / args.steps, "measured_s_per_step": per_step,
                       "timed_s": sum(times), "extrapolated_s_per_full_step": per_step * N_BODIES / run.bodies},
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": run.step.workers, "kind": "port",
                             "sample": run.describe(pairs / args.steps)},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    assert not _product_library_mapped(), "the reference arm must not load libamlp.so"
    if WORKLOAD.startswith("nvt-step-131072-cube26"):
        # the small configuration (1,000 cubes, packing fraction 0.30, seed 0) run in full: every body, every pair
        small = CpuRun(1000, "cube26", 0.30, 0, target_s=None)
        try:
            small.timed(2)
            st, sp = small.timed(10)
        finally:
            small.close()
        line["full_run_1000_cubes"] = {"value": 1000 * len(st) / sum(st), "unit": "particle-steps/s", "steps": len(st),
                                       "ms_per_step": statistics.mean(st) * 1e3, "filtered_pairs_per_step": sp / len(st),
                                       "sample": "none: all 1,000 bodies and all their pairs every step"}
    print(json.dumps(line))


# ----------------------------------------------------------------------------- ranks
def max_over_ranks(x: float, dist, device) -> float:
    """The largest of every rank's x (one process per GPU, replicas): the slowest
    replica's device time is the job's time. x itself without a process group."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, n_bodies: int, steps: int, job_ms: float) -> float:
    """Particle-steps/s of the whole job: every rank steps its own replica of
    n_bodies, and job_ms is the time over ranks (max_over_ranks)."""
    return world * n_bodies * steps / (job_ms / 1e3)


# ----------------------------------------------------------------------------- GPU arm
def _measure(system, method: str, steps: int, warmup: int, dist, dev):
    """Device time of `steps` full steps (L2 flushed between steps, outside the
    events) and of the force kernel inside them. Returns a dict."""
    import ctypes
    import torch
    from amlp import _lib
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2
    launches = [0]
    entry = "amlp_forces_" + ("fd" if method == "fd" else "adjoint")
    wide = method == "adjoint" and system.adj_ws is not None  # beyond the fused kernel: the wide adjoint
    if wide:
        entry = "amlp_forces_adjoint_wide"

    # Verlet rebuilds: every nlist_every steps counted from the first timed step, so that
    # the timed window starts with one (warm-up steps follow the engine's own schedule)
    origin = [None]
    rebuilds = [0]

    def one_step(ev_force=None):
        t = system.timestep
        due = (t - origin[0]) % system.nlist_every == 0 if origin[0] is not None else \
            (t % system.nlist_every == 0 and t > 0)
        if due:
            system.build_nlist(check=False)
            launches[0] += LAUNCHES["amlp_nlist_build"]
            rebuilds[0] += 1
        system.F.zero_()
        system.T.zero_()
        system.th[_lib.Thermostat.pe.offset:_lib.Thermostat.pe.offset + 8].zero_()
        system.filter_pairs()
        if ev_force is not None:
            ev_force[0].record(stream)
        args = [system.pos.data_ptr(), system.quat.data_ptr(), system.L, system.fpairs.data_ptr(),
                system.nf.data_ptr(), system.cap, ctypes.byref(system.nep), ctypes.byref(system.net.struct),
                system.F.data_ptr(), system.T.data_ptr(), system._pe_ptr()]
        if wide:
            args += [system.adj_ws.data_ptr(), system.adj_ws.numel()]
        if method == "fd_split":  # the reference's data flow: g_all and e_all in HBM, one pair-count read
            system._forces_split()
        else:
            _lib.call(entry, *args, stream.cuda_stream)
        if ev_force is not None:
            ev_force[1].record(stream)
        system.integrate_step_two()
        system.integrate_step_one()
        system.timestep += 1
        launches[0] += (LAUNCHES["amlp_pair_filter"] + (4 if wide else 3 if method == "fd_split" else 1) +
                        LAUNCHES["amlp_nvt_step_two"] + LAUNCHES["amlp_nvt_step_one"])

    for _ in range(warmup):
        one_step()
    torch.cuda.synchronize()
    P, NV = int(system.nf.item()), int(system.nv.item())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches[0] = 0
    rebuilds[0] = 0
    origin[0] = system.timestep
    start = (system.timestep, system.snapshot_tensors())  # the end-to-end leg starts from the same state
    step_ms, force_ms, stage_ms = [], [], []
    if wide:  # events between the three kernels of the wide force pass, on the launching stream
        _lib.call("amlp_stage_timing", 1)
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        one_step((f0, f1))
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        force_ms.append(f0.elapsed_time(f1))
        if wide:
            st3 = (ctypes.c_float * 3)()
            _lib.call("amlp_stage_times", st3)
            stage_ms.append(list(st3))
    if wide:
        _lib.call("amlp_stage_timing", 0)
    total = max_over_ranks(sum(step_ms), dist, dev)
    assert _lib.device_error() == 0, "a bounded device wait gave up"
    finite = bool(torch.isfinite(system.pos).all() and torch.isfinite(system.vel).all())
    return {"total_ms": total, "force_ms": statistics.mean(force_ms), "force_share": sum(force_ms) / sum(step_ms),
            "P": P, "NV": NV, "launches": launches[0], "P_end": int(system.nf.item()), "finite": finite,
            "rebuilds": rebuilds[0], "start": start,
            "stage_ms": [statistics.mean(col) for col in zip(*stage_ms)] if stage_ms else None}


def _e2e(system, method, steps, dist, dev, start):
    """Same metric through the public API with host buffers: every step copies the
    state in from pinned host memory, runs System.step and reads the state back.
    It starts from the state that began the device-timed window (`start`), with a
    Verlet rebuild at its first step like that window: a system that relaxes from
    its initial lattice loses pairs step by step, so a later start would time less
    work."""
    import numpy as np
    import torch
    stream = torch.cuda.current_stream()
    t0, snap = start
    system.restore_tensors(snap)
    system.timestep = t0 + (-t0) % system.nlist_every if t0 > 0 else system.nlist_every  # step() rebuilds first
    host = {k: torch.from_numpy(np.ascontiguousarray(getattr(system, k).cpu().numpy())).pin_memory()
            for k in ("pos", "quat", "vel", "angmom")}
    nbytes = sum(t.numel() * t.element_size() for t in host.values())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        for k in host:
            getattr(system, k).copy_(host[k], non_blocking=True)
        system.step(method)
        for k in host:
            host[k].copy_(getattr(system, k), non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    return ms, nbytes


def run_serving(dev, n_requests: int = 48, steps: int = 300, rate: float = 8.0, seq_requests: int = 0) -> dict:
    """Mixed request stream served by continuous batching, and the same requests
    run one after another with the plain FP32 method for the same number of
    steps each (all of them, or the first `seq_requests` of the stream)."""
    import torch
    from amlp.configs import make_state
    from amlp.engine import EnergyNet, Hypers, System
    from amlp.serving import Server, request_stream
    nets = {name: EnergyNet.xavier(47, WIDTHS, ACT, seed=SEED + k, device=dev)
            for k, name in enumerate(("cube26", "tetra16", "cyl24"))}
    reqs = request_stream(n_requests, seed=SEED, steps=steps, rate=rate)
    srv = Server(nets, hbm_budget=24 << 30, segment=100, device=dev)
    stats = srv.run(reqs).summary()
    seq_reqs = reqs[:seq_requests] if 0 < seq_requests < len(reqs) else reqs
    seq_steps = steps  # the same steps per request as served
    body_steps, ms = 0, 0.0
    for r in seq_reqs:
        st = make_state(r.n, r.shape, r.phi, kT=r.kT, seed=r.seed)
        sysm = System(st, r.shape, Hypers(), nets[r.shape], kT=r.kT, dt=DT, device=dev)
        sysm.run(3, method="fd")  # warm-up: graph capture (the timed steps replay the same graph size)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sysm.run(seq_steps, method="fd")
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        body_steps += r.n * seq_steps
        del sysm
    seq_rate = body_steps / (ms / 1e3)
    return {"value": stats["particle_steps_per_s"], "unit": "particle-steps/s",
            "value_server_clock": stats["particle_steps_per_s_server_clock"],
            "segment_ms_p50": stats["segment_ms_p50"], "segment_ms_p99": stats["segment_ms_p99"],
            "segment_wall_ms_p50": stats["segment_wall_ms_p50"], "segment_wall_ms_p99": stats["segment_wall_ms_p99"],
            "segment_ms_note": "per 100-step segment: device time of the graph replay; wall: Verlet lists + replay",
            "clock": ("admissions and request latencies on the server's clock: the device time of the segments "
                      "plus jumps over idle gaps, so the seeded stream is served the same way every run; "
                      "value is over the wall time (host work included), value_server_clock over the server's "
                      "clock"),
            "request_latency_s_p50": stats["request_latency_s_p50"],
            "request_latency_s_p99": stats["request_latency_s_p99"],
            "max_concurrent": stats["max_concurrent"], "requests": stats["requests"],
            "graphs_captured": stats["graphs_captured"], "wall_s": stats["wall_s"],
            "stream": f"{n_requests} requests, {steps} steps each, Poisson arrivals at {rate}/s, N log-uniform "
                      f"[500, 50000], shape uniform {{cube26, tetra16, cyl24}}, phi U[0.25, 0.45], kT U[0.5, 2.0], "
                      f"seed {SEED}; adjoint forces, bf16x3 tensor-core net, 100-step segments, 24 GiB budget",
            "sequential_plain": {"value": seq_rate, "unit": "particle-steps/s",
                                 "sample": (f"{'all ' if len(seq_reqs) == len(reqs) else 'the first '}"
                                            f"{len(seq_reqs)} requests x {seq_steps} steps, one after "
                                            f"another, plain FP32 finite differences, CUDA graphs")},
            "served_over_sequential_plain": stats["particle_steps_per_s"] / seq_rate}


def wide_roofline(roof: dict, r: dict, D: int, fp32_peak: float, bf16_peak: float) -> dict:
    """Roofline of the wide adjoint force pass from its three stages, each timed
    with CUDA events on the launching stream inside the timed window
    (amlp_stage_timing): the descriptor forward (one evaluation, FP32), the net
    forward and backward on the tensor cores (2 F_n per pair, algorithmic: one
    product per multiply-add, executed as three bf16 products), the descriptor
    backward (two evaluations' worth, FP32). The line's roofline is the stage
    that takes the most time; all three are listed."""
    from amlp.shapes import get_shape
    nd = get_shape(SHAPE).nd
    direct = uses_direct_form(nd, HYPERS)
    fd1 = descriptor_flops(nd, HYPERS, direct=direct)
    _, tc_pair = algorithmic_flops_per_pair("adjoint", nd=nd, D=D, widths=WIDTHS, hypers=HYPERS)
    names = (["k_desc_direct_fwd", "k_mlp_grad", "k_desc_direct_bwd"] if direct else
             ["k_adj_desc (forward)", "k_mlp_grad", "k_adj_desc (backward)"])
    P = r["P"]
    stages = []
    for name, ms, (fl, bound) in zip(names, r["stage_ms"], ((fd1, "fp32"), (tc_pair, "tensor"), (2 * fd1, "fp32"))):
        ach = fl * P / (ms / 1e3) / 1e12
        peak = bf16_peak if bound == "tensor" else fp32_peak
        tb = STAGE_DRAM_BYTES_PER_PAIR.get((name, D))
        st = {"kernel": name, "ms": ms, "bound": bound, "flops_per_pair": fl, "achieved": ach, "peak": peak,
              "frac": ach / peak, "traffic": tb * P if tb else None}
        if bound == "tensor":
            st["executed_tflops"] = 3.0 * ach
            st["frac_executed"] = 3.0 * ach / peak
        stages.append(st)
    dom = max(stages, key=lambda x: x["ms"])
    out = dict(roof)
    out.update({"bound": dom["bound"], "kernel": dom["kernel"], "achieved": dom["achieved"], "peak": dom["peak"],
                "frac": dom["frac"], "traffic": dom["traffic"], "stages": stages,
                "work": ("the stage that takes the most time; tensor stages count one product per multiply-add "
                         "against the measured bf16 peak (executed as three: frac_executed)")})
    out.pop("peak_nominal", None)
    out.pop("frac_of_nominal", None)
    return out


def make_net(dev):
    """The workload's net: seeded Xavier weights, the same with the output layer scaled by 0.05, or the
    shape's trained soft-repulsion net."""
    import numpy as np
    from amlp.engine import EnergyNet
    if NET == "trained" or NET.startswith("model_"):
        name = NET if NET.startswith("model_") else f"model_{SHAPE}_soft"
        z = np.load(os.path.join(REPO, "tests", "golden", f"{name}.npz"))
        return EnergyNet([(z[f"W{k}"], z[f"b{k}"]) for k in range(len(z.files) // 2)], ACT, dev)
    net = EnergyNet.xavier(47, WIDTHS, ACT, seed=SEED, device="cpu")
    layers = list(net.layers)
    if NET == "xavier_out0.05":
        W, b = layers[-1]
        layers[-1] = (W * np.float32(0.05), b)
    return EnergyNet(layers, ACT, dev)


def run_gpu(args, rank: int, world: int, local_rank: int) -> None:
    import torch
    from amlp.configs import make_state
    from amlp.engine import EnergyNet, Hypers, System

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    state = make_state(N_BODIES, SHAPE, PHI if PHI else 0.1, kT=KT, seed=SEED, L=BOX)
    net = make_net(dev)
    methods = ["adjoint", "fd"] if args.method == "both" else [args.method]
    if max(WIDTHS) > 64 or HYPERS != (10, 8, 4):
        # the fused plain kernel takes widths up to 64 and D = 47: the plain arm is the reference's
        # own data flow (descriptors, net, differences as three kernels), where one is asked for
        methods = ["adjoint", "fd_split"] if args.method == "both" and NET.startswith("model_") else ["adjoint"]
    peaks = measured_peaks()
    clk_mhz = peaks["sm_max_mhz"] or 1965.0
    fp32_nominal = 148 * 128 * 2 * clk_mhz * 1e6 / 1e12
    fp32_peak = measure_fp32_peak(dev)  # the denominator: measured here, not the nominal figure
    results = {}
    clocks = ClockSampler(local_rank)
    for m in methods:
        system = System(state, SHAPE, Hypers(*HYPERS), net, kT=KT, dt=DT, device=dev)
        r = _measure(system, m, args.steps, args.warmup, dist, dev)
        e2e_steps = max(3, min(args.steps, 20))
        r["e2e_ms"], r["e2e_bytes"] = _e2e(system, m, e2e_steps, dist, dev, r.pop("start"))
        r["e2e_steps"] = e2e_steps
        results[m] = r
        del system
        torch.cuda.empty_cache()
    clk = clocks.stop()

    def summary(m):
        r = results[m]
        from amlp.shapes import get_shape
        D = (HYPERS[0] + 1) + (HYPERS[1] + 1) * HYPERS[2]
        fl_pair, tc_pair = algorithmic_flops_per_pair(m, nd=get_shape(SHAPE).nd, D=D, widths=WIDTHS, hypers=HYPERS)
        achieved = fl_pair * r["P"] / (r["force_ms"] / 1e3) / 1e12
        tensor = None
        if tc_pair:
            tc_alg = tc_pair * r["P"] / (r["force_ms"] / 1e3) / 1e12
            tensor = {"algorithmic_tflops": tc_alg, "executed_tflops": 3.0 * tc_alg,
                      "peak": peaks["bf16_tflops"], "frac_executed": 3.0 * tc_alg / peaks["bf16_tflops"],
                      "note": "net on the tensor cores as three bf16 products per multiply-add (bf16x3)"}
        wide = m == "adjoint" and (max(WIDTHS) > 64 or HYPERS != (10, 8, 4))
        kernel = {"fd": "k_forces_fd", "fd_split": "k_descriptors + k_mlp + k_fd_scatter"}.get(m, "k_forces_adjoint")
        traffic = DRAM_BYTES_PER_PAIR.get(m)
        roof = {"bound": "fp32", "kernel": kernel, "achieved": achieved, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                "peak_nominal": fp32_nominal, "frac_of_nominal": achieved / fp32_nominal,
                "traffic": traffic * r["P"] if traffic else None,
                "traffic_unit": "bytes per launch (ncu, scaled by pairs from 32,768 bodies)",
                "flops_per_pair": fl_pair, "tensor_flops_per_pair": tc_pair, "tensor": tensor,
                "pairs_per_launch": r["P"], "launch_ms": r["force_ms"], "force_share_of_step": r["force_share"],
                "peak_source": (f"measured FP32 FMA throughput of amlp_fp32_fma_probe in this run (best of 3, "
                                f"CUDA events); nominal 148 SM x 128 lanes x 2 x {clk_mhz:.0f} MHz beside it; "
                                f"HBM {peaks['hbm_gbs']} GB/s, bf16 {peaks['bf16_tflops']} TFLOP/s "
                                f"{peaks['source']}"),
                "work": ("achieved counts the FP32 SIMT work only (descriptor forward and backward); "
                         "the net's tensor-core work is reported under 'tensor'") if tc_pair else
                        "achieved counts all the work (descriptors and net, FP32 SIMT)"}
        if wide and r.get("stage_ms"):
            roof = wide_roofline(roof, r, D, fp32_peak, peaks["bf16_tflops"])
        return {"value": job_throughput(world, N_BODIES, args.steps, r["total_ms"]), "ms_per_step": r["total_ms"] / args.steps,
                "roofline": roof,
                "e2e": {"value": job_throughput(world, N_BODIES, r["e2e_steps"], r["e2e_ms"]), "unit": "particle-steps/s",
                        "h2d_bytes_per_step": r["e2e_bytes"], "d2h_bytes_per_step": r["e2e_bytes"],
                        "steps": r["e2e_steps"]},
                "gpu_launches": r["launches"]}

    head = methods[0]
    hs = summary(head)
    line = {"metric": METRIC, "value": hs["value"], "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": hs["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded lattice, " + ("Xavier weights)" if NET != "trained" else
                                                                 "net fitted to a soft repulsion, committed fixture)"),
            "config": common_config(world),
            "run": {"method": head, "verlet_pairs": results[head]["NV"], "filtered_pairs": results[head]["P"],
                    "filtered_pairs_last_step": results[head]["P_end"], "state_finite": results[head]["finite"],
                    "nlist_rebuilds_in_window": results[head]["rebuilds"],
                    "nlist_schedule": "rebuild at the first timed step and every 100 steps after it",
                    "precision": ("FP32 descriptors; net on tensor cores as bf16x3 splits with FP32 accumulation"
                                  if head == "adjoint" else "FP32 throughout")},
            "roofline": hs["roofline"], "e2e": hs["e2e"], "gpu_launches": hs["gpu_launches"], "clocks": clk}
    if len(methods) > 1:
        ps = summary(methods[1])
        line["plain"] = {"method": methods[1], "value": ps["value"], "ms_per_step": ps["ms_per_step"],
                         "roofline": ps["roofline"], "e2e": ps["e2e"]}
        line["tuned_over_plain"] = hs["value"] / ps["value"]
        line["gpu_launches"] += ps["gpu_launches"]
    if rank == 0 and world == 1 and not args.no_serving and IS_BENCHMARK:
        line["serving"] = run_serving(dev, args.serving_requests, args.serving_steps, args.serving_rate,
                                      args.serving_seq_requests)
    if rank == 0 and not args.no_cpu_baseline and world == 1 and SHAPE == "cube26":
        line["cpu_baseline"] = cpu_step_sample()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------------------------- NVE energy drift
DRIFT_MODEL = os.path.join(REPO, "tests", "golden", "model_cyl24_soft.npz")


def run_drift(args, local_rank: int) -> None:
    """Energy conservation of the precision workload: 262,144 twisted cylinders
    (cyl24) at packing fraction 0.35, seed 3, net 47 -> 128 -> 128 -> 1 SiLU
    fitted to a soft point-point repulsion that vanishes inside the pair cutoff
    (a random net's energy jumps at the cutoff would swamp the integrator's
    drift). The lattice start is first equilibrated under the NVT thermostat at
    kT 1.0 (``--drift-equil`` steps, dt 0.005); from that state each run
    integrates NVE and reads H = KE_t + KE_r + PE (FP64) every 100 steps.
    Runs: the tensor-core adjoint forces at dt 0.005 (``--drift-steps``) and at
    dt 0.0025 (``--drift-half-steps``, to separate time-step error from the
    rest), and the plain FP32 finite differences at dt 0.005
    (``--drift-fd-steps``). Prints one JSON line per run."""
    import numpy as np
    import torch
    from amlp.configs import make_state
    from amlp.engine import EnergyNet, Hypers, System
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    z = np.load(args.drift_model)
    layers = [(z[f"W{k}"], z[f"b{k}"]) for k in range(len(z.files) // 2)]
    net = EnergyNet(layers, "silu", dev)
    n = 262144
    state = make_state(n, "cyl24", 0.35, kT=1.0, seed=3)
    equil = {"steps": args.drift_equil}
    if args.drift_equil > 0:
        s = System(state, "cyl24", Hypers(), net, kT=1.0, dt=0.005, device=dev)
        s.run(args.drift_equil, "adjoint")
        th = s.thermostat()
        equil.update(ke_per_body=(th["ke_t"] + th["ke_r"]) / n, pe_per_body=th["pe"] / n)
        state = s.state()
        del s
        torch.cuda.empty_cache()
    for method, dt, steps in (("adjoint", 0.005, args.drift_steps), ("adjoint", 0.0025, args.drift_half_steps),
                              ("fd_split", 0.005, args.drift_fd_steps)):
        if steps <= 0:
            continue
        s = System(state, "cyl24", Hypers(), net, kT=1.0, dt=dt, device=dev, nve=True)
        H, t_H = [], []
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.run(1, method)  # first force pass: H at t = 0
        torch.cuda.synchronize()
        H.append(s.conserved_quantity())
        t_H.append(0)
        th = s.thermostat()
        ke0, pe0 = th["ke_t"] + th["ke_r"], th["pe"]
        ev0.record()
        while s.timestep < steps + 1:
            s.run(min(100, steps + 1 - s.timestep), method)
            H.append(s.conserved_quantity())
            t_H.append(s.timestep - 1)
        ev1.record()
        torch.cuda.synchronize()
        H = np.asarray(H)
        time_units = np.asarray(t_H, np.float64) * dt
        slope = float(np.polyfit(time_units, H, 1)[0]) if len(H) > 2 else float("nan")
        th = s.thermostat()
        line = {"metric": "nve_energy_drift", "method": method, "dt": dt, "steps": steps,
                "workload": "nve-262144-cyl24-phi0.35-mlp47x128x128x1-silu", "bodies": n,
                "filtered_pairs": int(s.nf.item()), "equilibration": equil,
                "H0": float(H[0]), "H_end": float(H[-1]), "ke0": ke0, "pe0": pe0,
                "ke_end": th["ke_t"] + th["ke_r"], "pe_end": th["pe"],
                "drift_per_body": float((H[-1] - H[0]) / n),
                "slope_per_time_unit_per_body": slope / n,
                "max_abs_dev_per_body": float(np.abs(H - H[0]).max() / n),
                "rel_drift_vs_ke0": float((H[-1] - H[0]) / ke0),
                "ms_per_step": ev0.elapsed_time(ev1) / steps,
                "precision": ("FP32 descriptors, net on tensor cores as bf16x3 splits, FP32 accumulation; "
                              "FP64 kinetic-energy and pair-energy sums" if method == "adjoint" else
                              "FP32 finite differences (dx = dteta = 1e-5), the reference's method"),
                "H_per_body_samples": [float(h / n) for h in H[:: max(1, len(H) // 20)]]}
        print(json.dumps(line), flush=True)
        del s
        torch.cuda.empty_cache()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--method", choices=["both", "fd", "adjoint"], default="both")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=48,
                    help="requests of the served stream (the full stream of the serving configuration is 512)")
    ap.add_argument("--serving-steps", type=int, default=300,
                    help="NVT steps per request (2000 in the full serving configuration)")
    ap.add_argument("--serving-rate", type=float, default=8.0, help="Poisson arrival rate, requests per second")
    ap.add_argument("--serving-seq-requests", type=int, default=0,
                    help="requests of the stream run one after another with the plain method (0: all)")
    ap.add_argument("--serving-only", action="store_true",
                    help="only the serving leg (one JSON line with its results)")
    ap.add_argument("--bodies", type=int, default=N_BODIES,
                    help="system size (the benchmark workload is 131072; smaller sizes are for profiling)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="cube26",
                    help="cube26 is the benchmark; tetra16 and cyl24 are the differentiation and precision workloads")
    ap.add_argument("--drift", action="store_true",
                    help="NVE energy drift of the 262,144-cylinder precision workload instead of the benchmark")
    ap.add_argument("--drift-steps", type=int, default=10000)
    ap.add_argument("--drift-half-steps", type=int, default=0,
                    help="also run the adjoint forces at dt 0.0025 for this many NVE steps")
    ap.add_argument("--drift-fd-steps", type=int, default=0,
                    help="also run the plain finite-difference forces for this many NVE steps")
    ap.add_argument("--drift-equil", type=int, default=2000, help="NVT steps before the NVE runs")
    ap.add_argument("--drift-model", default=DRIFT_MODEL)
    args = ap.parse_args()
    if args.workload != "cube26":
        w = WORKLOADS[args.workload]
        g = globals()
        g.update(N_BODIES=w["n"], SHAPE=w["shape"], PHI=w.get("phi"), SEED=w["seed"], WIDTHS=w["widths"],
                 ACT=w["act"], NET=w["net"], IS_BENCHMARK=False, HYPERS=w.get("hypers", (10, 8, 4)),
                 BOX=w.get("L"), KT=w.get("kT", 1.0))
        D = (HYPERS[0] + 1) + (HYPERS[1] + 1) * HYPERS[2]
        dens = f"phi{w['phi']:.2f}" if w.get("phi") else f"L{w['L']:.1f}"
        g["WORKLOAD"] = (f"nvt-step-{w['n']}-{w['shape']}-{dens}-mlp{D}x" +
                         "x".join(str(x) for x in w["widths"]) + f"x1-{w['act']}" +
                         (f"-{w['net']}" if w["net"].startswith("model_") else ""))
        if args.bodies == 131072:
            args.bodies = w["n"]
    if args.drift:
        run_drift(args, int(os.environ.get("LOCAL_RANK", 0)))
        return
    if args.bodies != N_BODIES:
        globals()["WORKLOAD"] = WORKLOAD.replace(str(N_BODIES), str(args.bodies))
        if BOX:  # the same number density
            globals()["BOX"] = BOX * (args.bodies / N_BODIES) ** (1.0 / 3.0)
        globals()["N_BODIES"] = args.bodies
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.serving_only:
        import torch
        dev = torch.device("cuda", local_rank)
        torch.cuda.set_device(dev)
        print(json.dumps({"metric": "served particle-steps/s", "serving": run_serving(
            dev, args.serving_requests, args.serving_steps, args.serving_rate, args.serving_seq_requests)}))
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
