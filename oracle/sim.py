"""Oracle simulation loop (test infrastructure only).

Restates ``Sim.run`` / ``Sim.step`` (``nep_simulator/Sim.py:207-285``): the
Verlet list is rebuilt every 100 steps (``Sim.py:87``, ``:220-228``) with the
reference's cKDTree call, then each step computes forces
(``DescriptorGenerator`` + ``ForceEvaluator``), ``integrate_step_two`` and
``integrate_step_one`` (``NVT.py:12-64``).
"""
from __future__ import annotations

import numpy as np

from . import nep, nlist


class OracleSim:
    def __init__(self, pos, vel, orient, angmom, mass, moi, L, shape, hypers, layers, act, kT, timestep,
                 dt=np.float32, form="direct", initial_ke_quirk=True):
        self.state = nep.NVTState(pos, vel, orient, angmom, mass, moi, L, kT, timestep, dt, initial_ke_quirk)
        self.shape, self.hypers, self.layers, self.act = shape, hypers, layers, act
        self.dt, self.form = dt, form
        self.r_verlet = shape["cutoff"] + 2.0
        self.nlist = nlist.reference_pairs(self.state.pos, self.state.L, self.r_verlet)
        self.timestep = 0
        self.last = None

    def forces(self):
        s = self.state
        self.last = nep.pair_forces(s.pos, s.orient, self.nlist, s.L, self.shape, self.hypers, self.layers,
                                    self.act, dt=self.dt, form=self.form)
        return self.last["forces"], self.last["torques"]

    def step(self):
        F, T = self.forces()
        self.state.step_two(F, T)
        self.state.step_one()
        self.timestep += 1

    def run(self, nsteps, on_dump=None, dump=None):
        end = self.timestep + nsteps
        while self.timestep < end:
            if self.timestep % 100 == 0 and self.timestep > 0:
                self.nlist = nlist.reference_pairs(self.state.pos, self.state.L, self.r_verlet)
            if dump and on_dump and self.timestep % dump == 0:
                on_dump(self.timestep, self.state)
            self.step()
