"""Drop-in ``GsdHandler`` (reference: ``nep_simulator/GsdHandler.py``).

Reads the last frame (or ``target_frame``) of a GSD 2.0 file with the HOOMD
schema through ``amlp.gsd``; the getters return only the rows with
``typeid == 0`` (the rigid-body centres), as in ``GsdHandler.py:72-128``.
A multi-frame file is accepted with a message (``:18-20``). Snapshot objects
with ``.particles`` / ``.box`` attributes are accepted like ``:46-60``.
"""
import numpy as np

import _amlp_path  # noqa: F401
from amlp import gsd as _gsd


class GsdHandler:
    def __init__(self, filename):
        self.read_system(filename, -1)

    def read_system(self, input, target_frame):
        self.target_frame = target_frame
        self.frame = 0
        if isinstance(input, (str, bytes)) or hasattr(input, "__fspath__"):
            with _gsd.GsdFile(input, "r") as f:
                if len(f) > 1:
                    print("init_gsd can't have more than one frames")
                if len(f) == 0:
                    raise _gsd.GsdError(f"{input}: no frames")
                self.frame = len(f) - 1 if target_frame == -1 else int(target_frame)
                fr = f[self.frame]
            get = fr.get
            self.positions = get("position").copy()
            self.velocities = get("velocity").copy()
            self.bodi = get("body").copy()
            self.moment_inertia = get("moment_inertia").copy()
            self.orientations = get("orientation").copy()
            self.mass = get("mass").copy()
            self.angmom = get("angmom").copy()
            self.types = list(fr.types)
            self.typeid = get("typeid").copy()
            self.charges = get("charge").copy()
            self.box = fr.box.copy()
            self.Lx, self.Ly, self.Lz = fr.box[0:3]
        else:
            p = input.particles
            self.positions = np.array(p.position)
            self.velocities = np.array(p.velocity)
            self.types = list(p.types)
            self.typeid = np.array(p.typeid)
            self.bodi = np.array(p.body)
            self.moment_inertia = np.array(p.moment_inertia)
            self.orientations = np.array(p.orientation)
            self.mass = np.array(p.mass)
            self.angmom = np.array(p.angmom)
            self.charges = np.array(p.charge)
            self.Lx = self.Ly = self.Lz = np.float32(input.box.Lx)
        self.body = np.array(self.bodi, dtype=np.int64)
        self.body[self.body > 9999999] = -1

    def _c(self, a):
        return a[self.typeid == 0]

    def get_central_pos(self):
        return self._c(self.positions)

    def get_COM_velocities(self):
        return self._c(self.velocities)

    def getMass(self):
        return self._c(self.mass)

    def getOrientations(self):
        return self._c(self.orientations)

    def getAngmom(self):
        return self._c(self.angmom)

    def getMoi(self):
        return self._c(self.moment_inertia)

    def getCharges(self):
        return np.copy(self.charges)

    def getAllbody(self):
        return self.body

    def getLx(self):
        return self.Lx
