"""Drop-in ``NVT`` (reference: ``nep_simulator/NVT.py``): the two halves of the
MTK Nose-Hoover step for rigid bodies, run by ``amlp_nvt_step_two`` and
``amlp_nvt_step_one`` for any number of bodies."""
from Sim import Sim


class NVT(Sim):
    def integrate_step_one(self):
        """Translation, rotation and kinetic energies (``NVT.py:12-15``, ``:67-129``)."""
        self.system.integrate_step_one()

    def integrate_step_two(self):
        """Thermostat update, velocity and angular-momentum kicks (``NVT.py:17-64``)."""
        self.system.integrate_step_two()
        self.timestep += 1
