"""The C ABI from C: ``tests/c_caller.c`` drives a simulation handle
(amlp_create, amlp_set_shape / _model / _state, amlp_step, amlp_get_state,
amlp_get_thermostat, amlp_destroy) the way a C host program would.

* CPU: it compiles with gcc and links against libamlp.so and the CUDA runtime;
* GPU: 150 adjoint steps of 300 cubes (a Verlet rebuild at step 100) end on
  the trajectory of the same run through ``amlp.native.NativeSystem``, within
  float-atomics rounding (1e-3 of the scale after 150 steps), and on the same
  thermostat (1e-4).
"""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from conftest import PKG, REPO

CUDA = "/usr/local/cuda"
LIBDIR = os.path.join(PKG, "amlp")


def _compile(out_dir) -> str:
    gcc = shutil.which("gcc")
    if gcc is None or not os.path.exists(os.path.join(CUDA, "include", "cuda_runtime.h")):
        pytest.skip("gcc or the CUDA headers are missing")
    from amlp import build
    build.build()
    exe = os.path.join(str(out_dir), "c_caller")
    cmd = [gcc, "-O2", "-Wall", "-I", os.path.join(REPO, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(REPO, "tests", "c_caller.c"), "-L", LIBDIR, "-lamlp", "-L", os.path.join(CUDA, "lib64"),
           "-lcudart", f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    exe = _compile(tmp_path)
    assert os.path.exists(exe)


def _write_input(path, st, shape, net, kT, dt):
    f32 = lambda a: np.ascontiguousarray(np.asarray(a, np.float32)).tobytes()  # noqa: E731
    with open(path, "wb") as fh:
        fh.write(struct.pack("<iii", st.N, shape.npts, len(net.layers)))
        fh.write(struct.pack("<7f", np.float32(st.L), kT, dt, shape.en_min, shape.en_max, shape.cutoff,
                             shape.nep_cutoff))
        fh.write(f32(np.asarray(st.moi, np.float32).reshape(-1)[:3]))
        fh.write(struct.pack(f"<{len(net.dims)}i", *net.dims))
        fh.write(struct.pack("<i", {"relu": 0, "tanh": 1, "silu": 2}[net.act]))
        for a in (shape.pts, st.pos, st.orient, st.vel, st.angmom, st.mass):
            fh.write(f32(a))
        fh.write(net.d_w.cpu().numpy().astype(np.float32).tobytes())


@pytest.mark.gpu
def test_c_caller_matches_the_python_handle(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from amlp.configs import make_state
    from amlp.engine import EnergyNet, Hypers
    from amlp.native import NativeSystem
    from amlp.shapes import get_shape

    exe = _compile(tmp_path)
    st = make_state(300, "cube26", 0.30, kT=1.0, seed=9)
    shape = get_shape("cube26")
    base = EnergyNet.xavier(47, (64, 64), "tanh", seed=2, device="cpu")
    net = EnergyNet([(W * np.float32(0.1), b) for W, b in base.layers], "tanh", "cuda:0")
    inp, out = os.path.join(str(tmp_path), "in.bin"), os.path.join(str(tmp_path), "out.bin")
    _write_input(inp, st, shape, net, 1.0, 0.005)
    r = subprocess.run([exe, inp, out, "150", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = open(out, "rb").read()
    n = st.N
    arr = np.frombuffer(raw[:4 * 14 * n], np.float32)
    got = {"pos": arr[:3 * n].reshape(n, 3), "quat": arr[3 * n:7 * n].reshape(n, 4),
           "vel": arr[7 * n:10 * n].reshape(n, 3), "angmom": arr[10 * n:14 * n].reshape(n, 4)}
    xi, eta, pe = struct.unpack("<3d", raw[4 * 14 * n:])
    h = NativeSystem(st, shape, Hypers(), net, kT=1.0, dt=0.005, device="cuda:0")
    h.run(150, "adjoint")
    ref = {k: v.cpu().numpy() for k, v in h.state().items()}
    th = h.thermostat()
    h.close()
    for k in ("pos", "quat", "vel", "angmom"):
        assert np.isfinite(got[k]).all()
        assert np.abs(got[k] - ref[k]).max() <= 1e-3 * max(1.0, np.abs(ref[k]).max()), k
    assert abs(xi - th["xi"]) <= 1e-4 * max(1.0, abs(th["xi"]))
    assert abs(eta - th["eta"]) <= 1e-4 * max(1.0, abs(th["eta"]))
    assert abs(pe - th["pe"]) <= 1e-4 * max(1.0, abs(th["pe"]))
