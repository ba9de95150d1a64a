"""Generate the golden fixtures in this directory by running the reference's own
``NVT``/``Sim``/``DescriptorGenerator``/``ForceEvaluator`` classes on the CPU.

Runs only where the reference checkout is present (``AMLP_REFERENCE_ROOT``,
else a ``reference`` directory beside this repository). The reference imports CuPy and gsd, which are not
installed; ``oracle.ref_cupy_shim`` supplies numpy-backed stand-ins and runs
the reference's CUDA kernel strings compiled for the host
(``oracle/ref_kernels.py``). The reference's sequence of builder calls is the
one of ``nep_simulator/sim_input.py:50-61``.

Cases (one ``case_<name>.npz`` each, weights in ``model_<model>.npz``):

* ``th_C104``  -- ``init/th_init_N200.gsd``, hypers 10 8 4 4.5, ``model_th_C104``,
  shape ``th_v1``, kT 0.5, dt 0.005 (``runner.sh:4`` with the C104 model);
  step-0 intermediates, state after 1 and 3 steps, and a 205-step run with
  dumps every 100 steps (two neighbour-list rebuilds);
* ``th_C100``  -- same init with hypers 10 10 10 4.5 and ``model_th_C100``
  (``runner.sh:4``); step-0 intermediates and state after 1 step;
* ``cube_C104`` -- 200 ``cube_v2`` bodies on a seeded lattice (L = 26; the
  cube init file of ``runner.sh:2`` is not in the reference checkout) with
  ``model_nep_C104``; step-0 intermediates and state after 3 steps;
* ``cube_R64`` -- 400 ``cube_v2`` bodies on a seeded lattice (L = 30) with a
  seeded 47 -> 64 -> 64 -> 1 ReLU net (``model_cube_R64``, torch's default
  initialisation under ``torch.manual_seed(64)``), the width of the fused
  finite-difference kernel. ``Sim.setEvaluator`` fixes the net at 150 x 3
  (``Sim.py:60``); this case drives the same ``ForceEvaluator`` with
  ``setNN_dimensions(64, 1)`` (``ForceEvaluator.py:38-40``) and keeps all 10 P
  per-variant energies of step 0 (``e0``) besides the usual intermediates.

Usage: ``python tests/golden/make_golden.py``.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "anisotropic-ml_b200"))

G0_PAIRS = 32  # descriptor rows kept for the first pairs only (file size)


def _layers(sd):
    names = ["layer_first"] + [f"layer_hidden.{k}" for k in range(len(sd) // 2 - 2)] + ["layer_last"]
    return names


def save_model(model_path, name):
    import torch
    sd = torch.load(model_path, map_location="cpu")
    arrs = {}
    for k, nm in enumerate(_layers(sd)):
        arrs[f"W{k}"] = sd[nm + ".weight"].numpy().astype(np.float32)
        arrs[f"b{k}"] = sd[nm + ".bias"].numpy().astype(np.float32)
    np.savez(os.path.join(HERE, f"model_{name}.npz"), **arrs)


def _snapshot(sim):
    return dict(pos=np.array(sim.central_pos), vel=np.array(sim.velocities),
                orient=np.array(sim.orientations), angmom=np.array(sim.angmom),
                thermo=np.array([float(np.asarray(v)) for v in (sim.integrator_vars0, sim.integrator_vars1,
                                                                sim.integrator_vars2, sim.integrator_vars3,
                                                                sim.m_exp_thermo_fac)], np.float32))


def save_seeded_relu_net(path, name, D, width, depth, seed):
    """TheEnergyNet(width, depth, D) of the reference (ForceEvaluator.py:6-26) with
    torch's default initialisation under ``torch.manual_seed(seed)``, saved as a
    state dict (.pth) for ``read_model`` and as ``model_<name>.npz``."""
    import torch
    from ForceEvaluator import TheEnergyNet  # reference module, loaded by the shim's source finder
    torch.manual_seed(seed)
    net = TheEnergyNet(width, depth, D)
    torch.save(net.state_dict(), path)
    save_model(path, name)


def run_case(root, name, init_gsd, hypers, model, shape, kT, dt, steps_list, long_run=None, model_path=None,
             nn_dims=None):
    from ForceEvaluator import ForceEvaluator
    from NVT import NVT  # reference module, loaded by the shim's source finder

    model_path = model_path or os.path.join(root, "models", model + ".pth")
    if nn_dims is not None:
        # Sim.setEvaluator calls setNN_dimensions(150, 3) (Sim.py:60); the net of this case is nn_dims
        orig_dims = ForceEvaluator.setNN_dimensions
        ForceEvaluator.setNN_dimensions = lambda self, w, d: orig_dims(self, *nn_dims)
    try:
        _run_case(name, init_gsd, hypers, model, model_path, shape, kT, dt, steps_list, long_run, NVT)
    finally:
        if nn_dims is not None:
            ForceEvaluator.setNN_dimensions = orig_dims


def _run_case(name, init_gsd, hypers, model, model_path, shape, kT, dt, steps_list, long_run, NVT):
    def build(dump, fn):
        sim = NVT()
        sim.setDevice(0)
        sim.initializeSystem(init_gsd)
        sim.setNepDescriptors(list(hypers))
        sim.setEvaluator(model_path)
        sim.setShape(shape)
        sim.setNeighborList()
        sim.setGsdDump(dump, fn)
        sim.setkT(kT)
        sim.setdt(dt)
        return sim

    tmp = tempfile.mkdtemp()
    sim = build(10 ** 9, os.path.join(tmp, "a.gsd"))
    out = dict(hypers=np.asarray(hypers, np.float32), kT=np.float32(kT), dt=np.float32(dt),
               shape=np.bytes_(shape), model=np.bytes_(model))
    out.update({k + "0": v for k, v in _snapshot(sim).items() if k != "thermo"})
    out["mass"] = np.array(sim.mass, np.float32)
    out["moi"] = np.array(sim.moi, np.float32)
    out["L"] = np.float32(sim.Lx)
    nl = np.array(sim.Nlist)
    out["nlist0"] = nl[np.lexsort((nl[:, 1], nl[:, 0]))]
    cap = {}
    dg, ev = sim.descriptor_generator, sim.evaluator
    g_orig, e_orig, eg_orig = dg.generate_nep_descriptors, ev.evaluate_interactions, ev.evaluate_gradients

    def g_rec(*a):
        r = g_orig(*a)
        if "g" not in cap:
            P = int(r[2])
            g = np.array(r[0]).reshape(10, P, -1)
            cap["g"] = g[:, :G0_PAIRS].copy()
            cap["pairs"] = np.array(r[1].numpy())
            cap["P"] = P
        return r

    def eg_rec(g_all, P):
        import torch
        eg_orig(g_all, P)
        if "e" not in cap:
            with torch.no_grad():
                cap["e"] = ev.energy_net(torch.from_dlpack(g_all)).numpy().reshape(-1).copy()
            cap["F_pair"] = ev.gradient_dx.numpy().copy()
            cap["Ti"] = ev.gradient_dtetax.numpy().copy()
            cap["Tj"] = ev.gradient_dtetax2.numpy().copy()

    def e_rec(*a):
        r = e_orig(*a)
        if "F" not in cap:
            cap["F"], cap["T"] = np.array(r[0]), np.array(r[1])
        return r

    dg.generate_nep_descriptors, ev.evaluate_interactions, ev.evaluate_gradients = g_rec, e_rec, eg_rec
    done = 0
    for k in steps_list:
        sim.run(k - done) if done == 0 else _continue(sim, k - done)
        done = k
        for kk, v in _snapshot(sim).items():
            out[f"{kk}_s{k}"] = v
    out.update(g0=cap["g"], pairs0=cap["pairs"], P0=np.int64(cap["P"]), e0=cap["e"], Fgrad0=cap["F_pair"],
               Tigrad0=cap["Ti"], Tjgrad0=cap["Tj"], F0=cap["F"], T0=cap["T"])
    if long_run:
        nsteps, dump = long_run
        sim2 = build(dump, os.path.join(tmp, "long.gsd"))
        sim2.run(nsteps)
        for kk, v in _snapshot(sim2).items():
            out[f"{kk}_long"] = v
        out["long_steps"] = np.int64(nsteps)
        out["long_dump"] = np.int64(dump)
        from amlp.gsd import GsdFile
        with GsdFile(os.path.join(tmp, "long.gsd")) as g:
            out["long_frames_step"] = np.array([g[i].step for i in range(len(g))], np.int64)
            out["long_frames_pos"] = np.stack([g[i].particles["position"] for i in range(len(g))])
    np.savez(os.path.join(HERE, f"case_{name}.npz"), **out)
    print(name, "P0 =", cap["P"], "pairs in Verlet list:", len(nl))


def _continue(sim, nsteps):
    """Steps of ``Sim.run`` (``Sim.py:218-234``) without its one-time set-up."""
    end = sim.timestep + nsteps
    while sim.timestep < end:
        if sim.timestep % sim.Nlist_freq == 0 and sim.timestep > 0:
            sim.refreshNList()
        sim.step()


def cube_init(path, n=200, L=26.0, m=6, shuffle=False):
    from amlp.gsd import Frame, GsdFile
    rng = np.random.default_rng(7)
    g = np.arange(m)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    sites = sites[rng.permutation(len(sites))[:n]] if shuffle else sites[:n]
    pos = ((sites + 0.5) * (L / m) - L / 2 + rng.uniform(-0.3, 0.3, (n, 3))).astype(np.float32)
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    f = Frame()
    f.N, f.box, f.types = n, np.array([L, L, L, 0, 0, 0], np.float32), ["A"]
    f.particles.update(position=pos, orientation=q.astype(np.float32),
                       velocity=(rng.standard_normal((n, 3)) * np.sqrt(0.5)).astype(np.float32),
                       angmom=(rng.standard_normal((n, 4)) * 0.5).astype(np.float32),
                       moment_inertia=np.full((n, 3), 1.5, np.float32))
    with GsdFile(path, "w") as gf:
        gf.append(f)


def make_r64(root):
    tmp = tempfile.mkdtemp()
    mpath = os.path.join(tmp, "model_cube_R64.pth")
    save_seeded_relu_net(mpath, "cube_R64", 47, 64, 1, seed=64)
    cpath = os.path.join(tmp, "cube_init_400.gsd")
    cube_init(cpath, n=400, L=30.0, m=8, shuffle=True)
    run_case(root, "cube_R64", cpath, (10, 8, 4, 4.5), "model_cube_R64", "cube_v2", 0.5, 0.005, [1],
             model_path=mpath, nn_dims=(64, 1))


def main():
    from oracle import ref_cupy_shim
    root = ref_cupy_shim.install()
    cwd = os.getcwd()
    os.chdir(tempfile.mkdtemp())
    if "--r64" in sys.argv:  # only the 64-wide case
        try:
            make_r64(root)
        finally:
            os.chdir(cwd)
        return
    try:
        for m in ("model_th_C104", "model_th_C100", "model_nep_C104"):
            save_model(os.path.join(root, "models", m + ".pth"), m[len("model_"):])
        init = os.path.join(root, "init", "th_init_N200.gsd")
        from amlp.gsd import read_last_frame
        run_case(root, "th_C104", init, (10, 8, 4, 4.5), "model_th_C104", "th_v1", 0.5, 0.005, [1, 3],
                 long_run=(205, 100))
        run_case(root, "th_C100", init, (10, 10, 10, 4.5), "model_th_C100", "th_v1", 0.5, 0.005, [1])
        cpath = os.path.join(tempfile.mkdtemp(), "cube_init.gsd")
        cube_init(cpath)
        run_case(root, "cube_C104", cpath, (10, 8, 4, 4.5), "model_nep_C104", "cube_v2", 0.5, 0.005, [1, 3])
        if "--r64" in sys.argv or "--all" in sys.argv or len(sys.argv) == 1:
            make_r64(root)
        # the init frames themselves (the GPU box has no reference checkout)
        for nm in ("th_init_N200", "th_init_N200_seed20"):
            f = read_last_frame(os.path.join(root, "init", nm + ".gsd"))
            np.savez(os.path.join(HERE, f"init_{nm}.npz"), step=np.int64(f.step), box=f.box,
                     **{k: v for k, v in f.particles.items()})
    finally:
        os.chdir(cwd)


if __name__ == "__main__":
    main()
