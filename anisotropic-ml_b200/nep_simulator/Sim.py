"""Drop-in ``Sim`` (reference: ``nep_simulator/Sim.py``).

Same builder methods, call order and run loop as the reference
(``sim_input.py:50-61``, ``Sim.py:207-285``); the state lives on the GPU in
an ``amlp.engine.System`` and every step runs through ``libamlp``.

Run loop: the Verlet list is rebuilt every 100 steps and a GSD frame is
written every ``dump`` steps before the step (``Sim.py:218-234``); between
those events the steps replay as CUDA graphs.

Force methods (``setForceMethod``): "fd" (default, the reference's finite
differences in one fused kernel; nets wider than 64 use "fd_split"),
"fd_split" (the reference's data flow through ``DescriptorGenerator`` and
``ForceEvaluator``), "adjoint" (analytic forces and torques).

Additions to the reference, all off the reference's call path: the GSD dump
also stores the thermostat state under ``log/`` and ``initializeSystem`` reads
it back, so a run resumed from a dump continues exactly (the reference re-seeds
the thermostat, ``Sim.py:101-105``).
"""
import time

import numpy as np
import torch

import _amlp_path  # noqa: F401
from amlp import gsd as _gsd
from amlp.configs import State
from amlp.engine import Hypers, System
from DescriptorGenerator import DescriptorGenerator
from ForceEvaluator import ForceEvaluator
from GsdHandler import GsdHandler
import MathUtils as mu  # noqa: F401  (kept for API parity)

_THERMO_LOG = ("integrator_vars", "m_exp_thermo_fac")


class Sim:
    def __init__(self):
        print("A new simulation instance created.")
        self.method = None
        self.activation = "relu"
        self.nn_dims = (150, 3)  # Sim.py:60
        self.initial_ke_quirk = True
        self.nve = False
        self.gsdDumpPeriod = None
        self.system = None
        self._resume_thermo = None

    # ------------------------------------------------------------------ builders
    def setDevice(self, gpu_id):
        self.gpu_id = int(gpu_id)
        self.device = torch.device("cuda", self.gpu_id)
        torch.cuda.set_device(self.device)

    def initializeSystem(self, gsd_file):
        print("Simulation will be initialized from %s" % (gsd_file))
        h = GsdHandler(gsd_file)
        self.central_pos = h.get_central_pos()
        self.Nparticles = len(self.central_pos)
        self.N_dof = (self.Nparticles - 1) * 3
        self.RN_dof = self.Nparticles * 3
        self.velocities = h.get_COM_velocities()
        self.accel = np.zeros_like(self.velocities)
        self.mass = h.getMass()
        self.orientations = h.getOrientations()
        self.angmom = h.getAngmom()
        self.moi_to_dump = h.getMoi()
        self.moi = self.moi_to_dump[0]
        self.Lx = h.getLx()
        self.dx = 0.00001
        self.dteta = 0.00001
        with _gsd.GsdFile(gsd_file, "r") as f:
            log = f[h.frame].log
        if all(("thermostat/" + k) in log for k in _THERMO_LOG):
            self._resume_thermo = (np.asarray(log["thermostat/integrator_vars"], np.float32),
                                   np.float32(np.asarray(log["thermostat/m_exp_thermo_fac"]).reshape(-1)[0]))
            self.initial_ke_quirk = False

    def setNNShape(self, width, depth):
        """Width and hidden-layer count of the net (the reference fixes 150, 3)."""
        self.nn_dims = (int(width), int(depth))

    def setActivation(self, act):
        self.activation = act

    def setForceMethod(self, method):
        if method not in ("fd", "fd_split", "adjoint"):
            raise ValueError(f"unknown force method {method!r}")
        self.method = method

    def setEvaluator(self, model_path):
        self.evaluator = ForceEvaluator()
        self.evaluator.setDevice(self.gpu_id)
        self.evaluator.setNN_dimensions(*self.nn_dims)
        self.evaluator.setNd(self.N_descriptors)
        self.evaluator.setActivation(self.activation)
        self.evaluator.read_model(model_path)
        self.evaluator.set_dx_dteta(self.dx, self.dteta)
        self.evaluator.setNparticles(self.Nparticles)

    def setNepDescriptors(self, hypers):
        self.descriptor_generator = DescriptorGenerator()
        self.descriptor_generator.setDevice(self.device)
        self.descriptor_generator.setHyperParameters(hypers)
        self.descriptor_generator.setBoxSize(self.Lx)
        self.N_descriptors = self.descriptor_generator.getN_descriptor()
        self.descriptor_generator.set_dx_dteta(self.dx, self.dteta)

    def setShape(self, shape_str):
        self.shape_name = shape_str
        self.descriptor_generator.setShape(shape_str)
        en_min, en_max = self.descriptor_generator.get_en_min_max()
        self.evaluator.set_energy_range(en_min, en_max)
        self.cutoff = self.descriptor_generator.cutoff
        self.evaluator.move_data_to_device()
        self.descriptor_generator.move_data_to_device()

    def setNeighborList(self):
        self.Nlist_cutoff = self.cutoff + 2.0
        self.Nlist_freq = 100

    def setGsdDump(self, dump_period, filename):
        self.gsdDumpPeriod = dump_period
        self.gsdFilename = filename

    def setkT(self, kT):
        self.kT = kT

    def setdt(self, dt):
        self.dt = dt
        self.tau = 100.0 * dt

    def setNVE(self, nve=True):
        """Constant energy instead of the thermostat (not in the reference)."""
        self.nve = bool(nve)

    # ------------------------------------------------------------------ state
    def move_data_to_device(self):
        # the fields alias the device state after the first call (a second run continues from it)
        def host(a):
            return a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a, np.float32)
        state = State(pos=host(self.central_pos), orient=host(self.orientations), vel=host(self.velocities),
                      angmom=host(self.angmom), mass=host(self.mass), moi=np.asarray(self.moi, np.float32),
                      L=float(np.float32(self.Lx)))
        dg = self.descriptor_generator
        hyp = Hypers(dg.nrad, dg.nang, dg.lmax)
        if self.method is None:
            wide = max(self.evaluator.energy_net.dims[:-1]) > 64
            self.method = "fd_split" if wide else "fd"
        prev = self.system.thermostat() if self.system is not None else None
        self.system = System(state, dg.shape, hyp, self.evaluator.energy_net, self.kT, self.dt, device=self.device,
                             nve=self.nve, initial_ke_quirk=self.initial_ke_quirk and prev is None,
                             nlist_every=getattr(self, "Nlist_freq", 100), dx=self.dx, dteta=self.dteta,
                             moi=np.asarray(self.moi, np.float32))
        if prev is not None:  # a later run continues the thermostat of the previous one
            self.system.set_thermostat((prev["xi"], prev["eta"], prev["xi_rot"], prev["eta_rot"]),
                                       prev["thermo_fac"])
        elif self._resume_thermo is not None:
            self.system.set_thermostat(self._resume_thermo[0], self._resume_thermo[1])
        s = self.system
        self.central_pos, self.orientations, self.velocities, self.angmom = s.pos, s.quat, s.vel, s.angmom
        self.mass, self.accel, self.dp = s.mass, s.accel, s.dp
        self.forces, self.torks = s.F, s.T
        self.Nlist = s.vpairs[: int(s.nv.item())]

    def refreshNList(self):
        self.system.build_nlist()
        self.Nlist = self.system.vpairs[: int(self.system.nv.item())]

    def dumpConfig(self, ts):
        s = self.system
        f = _gsd.Frame()
        f.step = int(ts)
        f.box = np.array([s.L, s.L, s.L, 0, 0, 0], np.float32)
        f.N = s.N
        f.types = ["A", "B"]
        f.particles.update(position=s.pos.cpu().numpy(), typeid=np.zeros(s.N, np.uint32),
                           moment_inertia=np.asarray(self.moi_to_dump, np.float32), mass=s.mass.cpu().numpy(),
                           orientation=s.quat.cpu().numpy(), angmom=s.angmom.cpu().numpy(),
                           velocity=s.vel.cpu().numpy())
        th = s.thermostat()
        f.log["thermostat/integrator_vars"] = np.array([th["xi"], th["eta"], th["xi_rot"], th["eta_rot"]], np.float32)
        f.log["thermostat/m_exp_thermo_fac"] = np.array([th["thermo_fac"]], np.float32)
        with _gsd.GsdFile(self.gsdFilename, "w" if ts == 0 else "a") as g:
            g.append(f)

    def getRotKin(self):
        return self.system.thermostat()["ke_r"]

    def print_performance_info(self):
        if self.timestep > 0:
            total = time.time() - self.timer
            cur = time.time() - self.epoch_timer
            print("TPS : %.2f   - last TPS : %.2f" % (self.timestep / total, self.gsdDumpPeriod / cur))
            self.epoch_timer = time.time()

    def set_timers(self):
        self.t_gen = self.t_eval = self.t_s1 = self.t_s2 = self.t_nlist = 0

    # ------------------------------------------------------------------ run
    def run(self, Nsteps):
        self.is_sync = 1
        self.descriptor_generator.setSync(self.is_sync)
        self.evaluator.setSync(self.is_sync)
        self.set_timers()
        self.move_data_to_device()
        self.timestep = 0
        self.timer = time.time()
        self.epoch_timer = time.time()
        dump = self.gsdDumpPeriod
        while self.timestep < Nsteps:
            if self.timestep % self.Nlist_freq == 0 and self.timestep > 0:
                t0 = time.time()
                self.refreshNList()
                self.t_nlist += time.time() - t0
            if dump and self.timestep % dump == 0:
                self.print_performance_info()
                self.dumpConfig(self.timestep)
            nxt = Nsteps
            for period in (self.Nlist_freq, dump):
                if period:
                    nxt = min(nxt, (self.timestep // period + 1) * period)
            seg = nxt - self.timestep
            if self.method == "fd_split":
                for _ in range(seg):
                    self.step()
            else:
                self.system.timestep = self.timestep
                self.system.run(seg, method=self.method, graph=True)
                self.timestep += seg
        torch.cuda.synchronize(self.device)
        print("Timers:")
        print("t_nlist : %.2f" % (self.t_nlist))
        print("t_total : %.2f" % (time.time() - self.timer))
        print("Done")

    def step(self):
        """One step through ``DescriptorGenerator`` and ``ForceEvaluator`` when the
        method is "fd_split" (the reference's data flow), else through the engine."""
        if self.method != "fd_split":
            self.system.timestep = self.timestep
            self.system._step_kernels(self.method)
            self.timestep += 1
            return
        s = self.system
        g, pp, P = self.descriptor_generator.generate_nep_descriptors(s.pos, s.quat, self.Nlist)
        F, T = self.evaluator.evaluate_interactions(g, pp, P)
        s.F.copy_(F)
        s.T.copy_(T)
        self.integrate_step_two()
        self.integrate_step_one()
