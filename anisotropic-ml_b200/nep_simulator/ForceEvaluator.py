"""Drop-in ``ForceEvaluator`` (reference: ``nep_simulator/ForceEvaluator.py``).

``evaluate_interactions(g_all, pp, N_pair)`` returns per-body forces and
torques (N, 3) from the 10 finite-difference descriptor rows of every pair
(``ForceEvaluator.py:71-146``): net energies by ``amlp_mlp_energy`` (FP32),
differences, scaling by (en_max - en_min), +-100 clip and scatter by
``amlp_fd_scatter``. ``read_model`` loads the reference's ``.pth`` state dicts.
"""
import ctypes

import torch

import _amlp_path  # noqa: F401
from amlp._lib import Nep, call
from amlp.engine import EnergyNet


class TheEnergyNet(torch.nn.Module):
    """The reference's FFNN (``ForceEvaluator.py:6-26``), kept for loading and
    inspecting state dicts; evaluation runs in ``libamlp``."""

    def __init__(self, nn_width, num_hidden, input_size, activation="relu"):
        super().__init__()
        self.layer_first = torch.nn.Linear(input_size, nn_width)
        self.layer_hidden = torch.nn.ModuleList([torch.nn.Linear(nn_width, nn_width) for _ in range(num_hidden)])
        self.layer_last = torch.nn.Linear(nn_width, 1)
        self.activation = activation

    def forward(self, x):
        act = {"relu": torch.relu, "tanh": torch.tanh, "silu": torch.nn.functional.silu}[self.activation]
        u = act(self.layer_first(x))
        for hidden in self.layer_hidden:
            u = act(hidden(u))
        return self.layer_last(u)


class ForceEvaluator:
    def setDevice(self, gpu_id):
        self.gpu_id = int(gpu_id)
        self.torch_device = torch.device("cuda", self.gpu_id)

    def setNN_dimensions(self, w, d):
        self.width = w
        self.depth = d

    def set_dx_dteta(self, dx, dteta):
        self.dx = float(dx)
        self.dteta = float(dteta)

    def setNparticles(self, Nparticles):
        self.Nparticles = int(Nparticles)

    def setNd(self, Nd):
        self.Nd = int(Nd)

    def setSync(self, is_sync):
        self.is_sync = is_sync

    def setActivation(self, act):
        """Activation of the net ("relu" as in the reference, "tanh" or "silu")."""
        self.activation = act

    def read_model(self, model_path):
        """Load a state dict saved from ``TheEnergyNet`` (``ForceEvaluator.py:55-61``)."""
        sd = torch.load(model_path, map_location="cpu") if isinstance(model_path, str) else model_path
        net = TheEnergyNet(self.width, self.depth, self.Nd, getattr(self, "activation", "relu"))
        net.load_state_dict(sd)  # same shape checks as the reference
        self.energy_net = EnergyNet.from_state_dict(sd, getattr(self, "activation", "relu"), self.torch_device)

    def set_energy_range(self, en_min, en_max):
        self.en_min = en_min
        self.en_max = en_max

    def move_data_to_device(self):
        pass

    def evaluate_interactions(self, g_all, pp, N_pair):
        self.evaluate_gradients(g_all, N_pair)
        self.evaluate_forces_torques(pp)
        return self.forces, self.torks

    def evaluate_gradients(self, g_all, N_pair):
        """Net energies of all 10*N_pair rows (``ForceEvaluator.py:80-83``)."""
        g = g_all.contiguous()
        self.N_pair = int(N_pair)
        self.e_all = torch.empty(g.shape[0], dtype=torch.float32, device=self.torch_device)
        if g.shape[0]:
            call("amlp_mlp_energy", g.data_ptr(), g.shape[0], ctypes.byref(self.energy_net.struct),
                 self.e_all.data_ptr(), torch.cuda.current_stream(self.torch_device).cuda_stream)
        self.e0 = self.e_all[:self.N_pair]

    def evaluate_forces_torques(self, pp):
        """Differences, scale, clip and scatter (``ForceEvaluator.py:86-146``)."""
        n = Nep()
        n.dx, n.dteta = self.dx, self.dteta
        n.en_min, n.en_max = float(self.en_min), float(self.en_max)
        self.forces = torch.zeros(self.Nparticles, 3, dtype=torch.float32, device=self.torch_device)
        self.torks = torch.zeros(self.Nparticles, 3, dtype=torch.float32, device=self.torch_device)
        pairs = pp.to(self.torch_device, torch.int32).contiguous()
        if self.N_pair:
            call("amlp_fd_scatter", self.e_all.data_ptr(), self.N_pair, pairs.data_ptr(), ctypes.byref(n),
                 self.forces.data_ptr(), self.torks.data_ptr(), None,
                 torch.cuda.current_stream(self.torch_device).cuda_stream)
