"""Benchmark: particle-steps/s of the NVT step of 131,072 rigid cubes on B200.

Workload (one "step" = one full time step: pair filter, force pass, both NVT
halves; the Verlet list is rebuilt every 100 steps inside the timed region):
131,072 cube26 bodies at packing fraction 0.45, jittered lattice, random unit
quaternions, seed 1, NEP hypers (10, 8, 4), FFNN 47 -> 64 -> 64 -> 1 tanh with
seeded Xavier weights, dt 0.005, kT 1.0 (synthetic; no dataset involved).

Arms:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--method fd|adjoint]
  python bench.py --impl reference ...   CPU restatement of the reference's
      step (the oracle, bit-identical to the reference's own classes) on the
      host cores, timed on a bounded sample of the same workload.

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

# kernels launched by each libamlp entry point (for the gpu_launches count)
LAUNCHES = {"amlp_nlist_build": 11, "amlp_pair_filter": 2, "amlp_forces_fd": 1, "amlp_forces_adjoint": 1,
            "amlp_nvt_step_two": 2, "amlp_nvt_step_one": 1}


def algorithmic_flops_per_pair(method: str, nd: int = 52, D: int = 47, widths=WIDTHS) -> float:
    """Algorithmic FLOPs per filtered pair: descriptor F_d = 573 Nd + 432 per
    cloud evaluation (spherical-harmonic form), net F_n = 2 (sum of layer
    in x out); the plain method evaluates 10 clouds and 10 nets per pair, the
    adjoint one cloud + its backward (2 F_d) and the net forward + backward (2 F_n)."""
    dims = [D] + list(widths) + [1]
    fn = 2.0 * sum(dims[k] * dims[k + 1] for k in range(len(dims) - 1))
    fd = 573.0 * nd + 432.0
    if method == "fd":
        return 10.0 * (fd + fn)
    return 3.0 * fd + 2.0 * fn


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
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if "Active" in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks() -> dict:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return {"hbm_gbs": d.get("hbm_gbs"), "bf16_tflops": d.get("bf16_tflops"),
                "sm_max_mhz": d.get("sm_max_mhz", 1965.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0, "source": "fallback"}


# ----------------------------------------------------------------------------- reference arm / CPU baseline
def cpu_step_sample(state, budget_s: float = 15.0, pairs_sample: int = 1500):
    """Seconds per full step of the CPU oracle on this workload, estimated from a
    bounded sample: the force pass on `pairs_sample` filtered pairs scaled to all
    pairs, plus the integrator on all bodies and 1/100 of a cKDTree rebuild."""
    import numpy as np
    import torch
    from amlp.engine import EnergyNet
    from oracle import nep, nlist
    from oracle.shapes import SHAPES
    torch.set_num_threads(os.cpu_count() or 1)
    shape = SHAPES["cube26"]
    net = EnergyNet.xavier(47, WIDTHS, ACT, seed=SEED, device="cpu")
    t0 = time.perf_counter()
    vp = nlist.reference_pairs(state.pos, state.L, shape["cutoff"] + 2.0)
    t_nl = time.perf_counter() - t0
    keep, pairs, _ = nep.min_image_filter(state.pos, vp, state.L, shape["cutoff"])
    P = len(pairs)
    rng = np.random.default_rng(0)
    sel = np.sort(rng.choice(P, size=min(pairs_sample, P), replace=False))
    t0 = time.perf_counter()
    o = nep.pair_forces(state.pos, state.orient, pairs[sel], state.L, shape, (10, 8, 4), net.layers, ACT)
    t_f = (time.perf_counter() - t0) * P / len(sel)
    st = nep.NVTState(state.pos, state.vel, state.orient, state.angmom, state.mass, state.moi, state.L, KT, DT)
    t0 = time.perf_counter()
    st.step_two(o["forces"], o["torques"])
    st.step_one()
    t_i = time.perf_counter() - t0
    step = t_f + t_i + t_nl / 100.0
    sample = (f"force pass on {len(sel)} of {P} filtered pairs (scaled by {P / len(sel):.0f}x), integrator on "
              f"all {state.N} bodies, cKDTree rebuild/100; oracle FP32 path (numpy + torch CPU, "
              f"{torch.get_num_threads()} threads)")
    return step, sample, P


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    from amlp.configs import make_state
    state = make_state(N_BODIES, "cube26", PHI, kT=KT, seed=SEED)
    times = []
    sample = ""
    for _ in range(args.warmup + args.steps):
        t, sample, P = cpu_step_sample(state)
        times.append(t)
    per_step = statistics.mean(times[args.warmup:])
    value = N_BODIES / per_step
    cores = os.cpu_count() or 1
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "bodies": N_BODIES, "filtered_pairs": P, "parallelism": "replicas"},
            "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ----------------------------------------------------------------------------- GPU arm
def run_gpu(args, rank: int, world: int, local_rank: int) -> None:
    import numpy as np
    import torch
    from amlp import _lib
    from amlp.configs import make_state
    from amlp.engine import EnergyNet, Hypers, System

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    state = make_state(N_BODIES, "cube26", PHI, kT=KT, seed=SEED)
    net = EnergyNet.xavier(47, WIDTHS, ACT, seed=SEED, device=dev)
    system = System(state, "cube26", Hypers(), net, kT=KT, dt=DT, device=dev)
    method = args.method
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def one_step(ev_force=None):
        if system.timestep % system.nlist_every == 0 and system.timestep > 0:
            system.build_nlist(check=False)
            launches[0] += LAUNCHES["amlp_nlist_build"]
        system.F.zero_()
        system.T.zero_()
        system.th[_lib.Thermostat.pe.offset:_lib.Thermostat.pe.offset + 8].zero_()
        system.filter_pairs()
        if ev_force is not None:
            ev_force[0].record(stream)
        import ctypes
        _lib.call("amlp_forces_" + ("fd" if method == "fd" else "adjoint"), system.pos.data_ptr(),
                  system.quat.data_ptr(), system.L, system.fpairs.data_ptr(), system.nf.data_ptr(), system.cap,
                  ctypes.byref(system.nep), ctypes.byref(system.net.struct), system.F.data_ptr(),
                  system.T.data_ptr(), system._pe_ptr(), stream.cuda_stream)
        if ev_force is not None:
            ev_force[1].record(stream)
        system.integrate_step_two()
        system.integrate_step_one()
        system.timestep += 1
        launches[0] += LAUNCHES["amlp_pair_filter"] + 1 + LAUNCHES["amlp_nvt_step_two"] + LAUNCHES["amlp_nvt_step_one"]

    launches = [0]
    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    P = int(system.nf.item())
    NV = int(system.nv.item())
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches[0] = 0
    clocks = ClockSampler(local_rank)
    step_ms, force_ms = [], []
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between timed steps, outside the events
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        one_step((f0, f1))
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        force_ms.append(f0.elapsed_time(f1))
    torch.cuda.synchronize()
    clk = clocks.stop()
    total_ms = sum(step_ms)
    if dist:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
        total_ms = float(t.item())
    value = world * N_BODIES * args.steps / (total_ms / 1e3)

    # end to end through the public API with host buffers: every step copies the
    # state in from pinned host memory, runs the step and reads the state back
    host = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in
            (("pos", system.pos.cpu().numpy()), ("quat", system.quat.cpu().numpy()),
             ("vel", system.vel.cpu().numpy()), ("angmom", system.angmom.cpu().numpy()))}
    dev_t = {"pos": system.pos, "quat": system.quat, "vel": system.vel, "angmom": system.angmom}
    nbytes = sum(t.numel() * t.element_size() for t in host.values())
    e2e_steps = max(3, min(args.steps, 20))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        for k in host:
            dev_t[k].copy_(host[k], non_blocking=True)
        system.step(method)
        for k in host:
            host[k].copy_(dev_t[k], non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * N_BODIES * e2e_steps / (e2e_ms / 1e3)

    peaks = measured_peaks()
    fl_pair = algorithmic_flops_per_pair(method)
    f_avg = statistics.mean(force_ms) / 1e3
    achieved_tf = fl_pair * P / f_avg / 1e12
    clk_mhz = peaks["sm_max_mhz"] or 1965.0
    fp32_peak = 148 * 128 * 2 * clk_mhz * 1e6 / 1e12
    line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded lattice, Xavier weights)",
            "config": {"workload": WORKLOAD, "method": method, "bodies": N_BODIES, "verlet_pairs": NV,
                       "filtered_pairs": P, "nlist_every": 100, "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": {"bound": "fp32", "kernel": "k_forces_" + ("fd" if method == "fd" else "adjoint"),
                         "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved_tf / fp32_peak,
                         "traffic": None, "flops_per_pair": fl_pair, "pairs_per_launch": P,
                         "launch_ms": f_avg * 1e3, "force_share_of_step": sum(force_ms) / sum(step_ms),
                         "peak_source": f"FP32 SIMT: 148 SM x 128 lanes x 2 x {clk_mhz:.0f} MHz "
                                        f"(no measured FP32 peak; HBM {peaks['hbm_gbs']} GB/s {peaks['source']})"},
            "e2e": {"value": e2e_value, "unit": "particle-steps/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": nbytes, "steps": e2e_steps},
            "gpu_launches": launches[0], "clocks": clk}
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        t_cpu, sample, _ = cpu_step_sample(state)
        line["cpu_baseline"] = {"value": N_BODIES / t_cpu, "unit": "particle-steps/s", "cores": os.cpu_count() or 1,
                                "kind": "port", "sample": sample}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--method", choices=["fd", "adjoint"], default="fd")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
