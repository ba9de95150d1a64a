"""ctypes binding of ``libamlp.so`` (declared in ``include/amlp.h``).

The library is loaded from this package directory. There is no fallback: a
missing or unloadable library raises ``ImportError`` naming the build command.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libamlp.so")

AMLP_OK = 0
ACT = {"relu": 0, "tanh": 1, "silu": 2}
MAX_LAYERS = 8
MAX_PTS = 64


class AmlpError(RuntimeError):
    def __init__(self, fn: str, status: int, detail: str = ""):
        self.status = status
        super().__init__(f"{fn} failed: {status_string(status)}" + (f" ({detail})" if detail else ""))


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m amlp.build` in anisotropic-ml_b200/ "
                          "(or __graft_entry__.build())")
    try:
        return ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise ImportError(f"cannot load {LIB_PATH}: {e}") from e


lib = _load()


class Nep(ctypes.Structure):
    _fields_ = [("nrad", ctypes.c_int), ("nang", ctypes.c_int), ("lmax", ctypes.c_int), ("npts", ctypes.c_int),
                ("d_pts", ctypes.c_void_p), ("cutoff", ctypes.c_double), ("nep_cutoff", ctypes.c_float),
                ("en_min", ctypes.c_float), ("en_max", ctypes.c_float), ("dx", ctypes.c_float),
                ("dteta", ctypes.c_float)]


class Mlp(ctypes.Structure):
    _fields_ = [("n_layers", ctypes.c_int), ("dims", ctypes.c_int * (MAX_LAYERS + 1)), ("act", ctypes.c_int),
                ("d_w", ctypes.c_void_p)]


class Thermostat(ctypes.Structure):
    _fields_ = [("xi", ctypes.c_float), ("eta", ctypes.c_float), ("xi_rot", ctypes.c_float),
                ("eta_rot", ctypes.c_float), ("thermo_fac", ctypes.c_float), ("pad", ctypes.c_float * 3),
                ("ke_t", ctypes.c_double), ("ke_r", ctypes.c_double), ("pe", ctypes.c_double)]


class Nvt(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_float), ("tau", ctypes.c_float), ("kT", ctypes.c_float), ("n_dof", ctypes.c_float),
                ("rn_dof", ctypes.c_float), ("moi", ctypes.c_float * 3), ("box", ctypes.c_float),
                ("nve", ctypes.c_int)]


class Replica(ctypes.Structure):
    """``amlp_replica``: per-system parameters of a multi-system launch."""
    _fields_ = [("kT", ctypes.c_float), ("n_dof", ctypes.c_float), ("rn_dof", ctypes.c_float),
                ("box", ctypes.c_float), ("nve", ctypes.c_int), ("pad", ctypes.c_int * 3)]


class SimConfig(ctypes.Structure):
    """``amlp_sim_config``: parameters of a simulation handle."""
    _fields_ = [("n", ctypes.c_int), ("nrad", ctypes.c_int), ("nang", ctypes.c_int), ("lmax", ctypes.c_int),
                ("kT", ctypes.c_float), ("dt", ctypes.c_float), ("tau", ctypes.c_float), ("nve", ctypes.c_int),
                ("initial_ke_quirk", ctypes.c_int), ("nlist_every", ctypes.c_int), ("skin", ctypes.c_double),
                ("dx", ctypes.c_float), ("dteta", ctypes.c_float)]


class PoolConfig(ctypes.Structure):
    """``amlp_pool_config``: shape, net and integrator of a serving pool."""
    _fields_ = [("nrad", ctypes.c_int), ("nang", ctypes.c_int), ("lmax", ctypes.c_int), ("dt", ctypes.c_float),
                ("tau", ctypes.c_float), ("h_pts", ctypes.c_void_p), ("npts", ctypes.c_int),
                ("en_min", ctypes.c_float), ("en_max", ctypes.c_float), ("cutoff", ctypes.c_double),
                ("nep_cutoff", ctypes.c_float), ("skin", ctypes.c_double), ("h_moi", ctypes.c_void_p),
                ("mlp", ctypes.POINTER(Mlp))]


class PoolSystem(ctypes.Structure):
    """``amlp_pool_system``: one system admitted to a pool (host arrays)."""
    _fields_ = [("n", ctypes.c_int), ("box", ctypes.c_float), ("kT", ctypes.c_float), ("nve", ctypes.c_int),
                ("verlet_cap", ctypes.c_longlong), ("h_pos", ctypes.c_void_p), ("h_quat", ctypes.c_void_p),
                ("h_vel", ctypes.c_void_p), ("h_angmom", ctypes.c_void_p), ("h_mass", ctypes.c_void_p)]


FORCES = {"fd": 0, "adjoint": 1}
POOL_ACTIVE, POOL_PENDING = 0, 1

_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong
_F = ctypes.c_float
_D = ctypes.c_double
_SZ = ctypes.c_size_t
_PSZ = ctypes.POINTER(ctypes.c_size_t)

# name -> argtypes (all return int status except the three library queries)
SIGNATURES = {
    "amlp_nlist_workspace_bytes": [_I, _F, _D, _PSZ],
    "amlp_nlist_build": [_P, _I, _F, _D, _P, _LL, _P, _P, _SZ, _P],
    "amlp_nlist_build_noalloc": [_P, _I, _F, _D, _P, _LL, _P, _P],
    "amlp_nlist_check_displacement": [_P, _P, _I, _F, _F, _P, _P],
    "amlp_nlist_build_gated": [_P, _I, _F, _D, _P, _LL, _P, _P, _SZ, _P, _P, _P],
    "amlp_filter_workspace_bytes": [_LL, _PSZ],
    "amlp_pair_filter": [_P, _F, _D, _P, _P, _LL, _P, _P, _P, _SZ, _P],
    "amlp_descriptors": [_P, _P, _F, _P, _LL, ctypes.POINTER(Nep), _P, _P],
    "amlp_mlp_energy": [_P, _LL, ctypes.POINTER(Mlp), _P, _P],
    "amlp_mlp_loss_grad": [_P, _P, _LL, ctypes.POINTER(Mlp), _P, _P, _P],
    "amlp_fd_scatter": [_P, _LL, _P, ctypes.POINTER(Nep), _P, _P, _P, _P],
    "amlp_forces_fd": [_P, _P, _F, _P, _P, _LL, ctypes.POINTER(Nep), ctypes.POINTER(Mlp), _P, _P, _P, _P],
    "amlp_forces_fd_energies": [_P, _P, _F, _P, _P, _LL, ctypes.POINTER(Nep), ctypes.POINTER(Mlp), _P, _P, _P,
                                _P, _P],
    "amlp_forces_adjoint": [_P, _P, _F, _P, _P, _LL, ctypes.POINTER(Nep), ctypes.POINTER(Mlp), _P, _P, _P, _P],
    "amlp_adjoint_workspace_bytes": [_LL, _PSZ],
    "amlp_forces_adjoint_wide": [_P, _P, _F, _P, _P, _LL, ctypes.POINTER(Nep), ctypes.POINTER(Mlp), _P, _P, _P,
                                 _P, _SZ, _P],
    "amlp_multi_forces_adjoint_wide": [_P, _P, _P, _P, _P, _P, _LL, ctypes.POINTER(Nep), ctypes.POINTER(Mlp),
                                       _P, _P, _P, _P, _SZ, _P],
    "amlp_pair_descriptors": [_P, _P, _F, _P, _P, _LL, ctypes.POINTER(Nep), _P, _I, _P],
    "amlp_pair_energy_vjp": [_P, _P, _F, _P, _P, _LL, ctypes.POINTER(Nep), ctypes.POINTER(Mlp), _P, _I, _P, _P,
                             _P, _P, _SZ, _P],
    "amlp_mlp_backward": [_P, _P, _LL, ctypes.POINTER(Mlp), _P, _P],
    "amlp_device_error": [ctypes.POINTER(ctypes.c_uint), _I],
    "amlp_test_first_wait_limit": [_I],
    "amlp_stage_timing": [_I],
    "amlp_stage_times": [ctypes.POINTER(_F)],
    "amlp_fp32_fma_probe": [_P, _I, ctypes.POINTER(_D), _P],
    "amlp_nvt_workspace_bytes": [_I, _PSZ],
    "amlp_nvt_init": [_P, _P, _P, _P, _I, ctypes.POINTER(Nvt), _I, _P, _P, _SZ, _P],
    "amlp_nvt_step_two": [_P, _P, _P, _P, _P, _P, _P, _P, _I, ctypes.POINTER(Nvt), _P, _P],
    "amlp_nvt_step_one": [_P, _P, _P, _P, _P, _P, _P, _I, ctypes.POINTER(Nvt), _P, _P, _SZ, _P],
    "amlp_multi_pair_filter": [_P, _P, _P, _D, _P, _P, _LL, _P, _P, _P, _SZ, _P],
    "amlp_multi_forces_adjoint": [_P, _P, _P, _P, _P, _P, _LL, ctypes.POINTER(Nep), ctypes.POINTER(Mlp),
                                  _P, _P, _P, _P],
    "amlp_multi_nvt_init": [_P, _P, _P, _P, _P, _I, _I, ctypes.POINTER(Nvt), _P, _P],
    "amlp_multi_nvt_step_two": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _P, ctypes.POINTER(Nvt), _P, _P],
    "amlp_multi_nvt_step_one": [_P, _P, _P, _P, _P, _P, _P, _P, _I, _P, ctypes.POINTER(Nvt), _P, _P],
    # simulation handles and the serving pool (handles are opaque pointers)
    "amlp_create": [ctypes.POINTER(SimConfig), ctypes.POINTER(_P)],
    "amlp_set_shape": [_P, _P, _I, _F, _F, _D, _F],
    "amlp_set_model": [_P, ctypes.POINTER(Mlp), _P],
    "amlp_set_state": [_P, _P, _P, _P, _P, _P, _P, _F, _P],
    "amlp_build_nlist": [_P, _P],
    "amlp_sim_descriptors": [_P, _P, _P, _LL, ctypes.POINTER(_LL), _P],
    "amlp_forces": [_P, _P, _P, _I, _P],
    "amlp_step": [_P, _I, _I, _P],
    "amlp_get_state": [_P, _P, _P, _P, _P, _P],
    "amlp_get_thermostat": [_P, ctypes.POINTER(Thermostat), _P],
    "amlp_pool_create": [ctypes.POINTER(PoolConfig), ctypes.POINTER(_P)],
    "amlp_pool_admit": [_P, ctypes.POINTER(PoolSystem), ctypes.POINTER(_I)],
    "amlp_pool_evict": [_P, _I, _P, _P, _P, _P, ctypes.POINTER(Thermostat)],
    "amlp_pool_step_segment": [_P, _I, _P],
    "amlp_pool_system_status": [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_LL), ctypes.POINTER(Thermostat)],
}

# entry points that do not return a status: name -> (argtypes, restype)
OTHER_SIGNATURES = {
    "amlp_destroy": ([_P], None),
    "amlp_timestep": ([_P], _LL),
    "amlp_last_error": ([_P], ctypes.c_char_p),
    "amlp_pool_destroy": ([_P], None),
    "amlp_pool_size": ([_P], _I),
    "amlp_pool_last_error": ([_P], ctypes.c_char_p),
}

lib.amlp_version.restype = ctypes.c_int
lib.amlp_status_string.restype = ctypes.c_char_p
lib.amlp_status_string.argtypes = [ctypes.c_int]
lib.amlp_last_cuda_error.restype = ctypes.c_char_p
for _name, _args in SIGNATURES.items():
    _fn = getattr(lib, _name)
    _fn.argtypes = _args
    _fn.restype = ctypes.c_int
for _name, (_args, _res) in OTHER_SIGNATURES.items():
    _fn = getattr(lib, _name)
    _fn.argtypes = _args
    _fn.restype = _res


def status_string(s: int) -> str:
    return lib.amlp_status_string(s).decode()


def call(name: str, *args) -> None:
    """Call an entry point and raise ``AmlpError`` on a non-zero status."""
    st = getattr(lib, name)(*args)
    if st != AMLP_OK:
        detail = lib.amlp_last_cuda_error().decode() if st == 4 else ""
        raise AmlpError(name, st, detail)


def call_status(name: str, *args) -> int:
    return getattr(lib, name)(*args)


def size_query(name: str, *args) -> int:
    out = ctypes.c_size_t(0)
    call(name, *args, ctypes.byref(out))
    return int(out.value)


def device_error(clear: bool = True) -> int:
    """Sticky error bits of bounded device-side waits (0 = none)."""
    v = ctypes.c_uint(0)
    call("amlp_device_error", ctypes.byref(v), int(clear))
    return int(v.value)


class AmlpDeviceError(RuntimeError):
    """A bounded device-side wait gave up: the results of the launches since the
    last check are not to be trusted (the kernels stopped early, no fault)."""


def check_device() -> None:
    """Raise ``AmlpDeviceError`` if a bounded device-side wait gave up since the
    last check (the flags are cleared). Synchronises the device."""
    flags = device_error(clear=True)
    if flags:
        raise AmlpDeviceError(f"a bounded device-side wait gave up (flags {flags:#x})")


def exported_symbols() -> list[str]:
    return ["amlp_version", "amlp_status_string", "amlp_last_cuda_error"] + list(SIGNATURES) + list(OTHER_SIGNATURES)
