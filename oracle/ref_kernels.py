"""Build recipe: compile the reference's CUDA kernel strings for the host CPU.

TEST INFRASTRUCTURE ONLY. The reference keeps every kernel as CUDA C inside a
Python raw string passed to ``cupy.RawKernel`` (``nep_simulator/cudakernels/*.py``).
This recipe reads those strings where they lie under the reference checkout,
wraps each in a tiny host shim (``__global__`` -> plain function, a loop over
``blockIdx.x`` / ``threadIdx.x``) and compiles it with g++ into
``oracle/_ref/ref_<kernel>.so``. Nothing of the reference source is written
into the repository; the generated wrapper and the library live in
``oracle/_ref`` only, which git ignores.

Kernels that synchronise threads through shared memory (``radial_grad``,
``NepDescriptorKernels.py:3-93``, and the dead ``g_all`` of
``SingleKernel.py``) cannot run one thread after another and are not built;
the oracle restates ``radial_grad`` instead.

Run ``python oracle/ref_kernels.py`` (or ``build()`` in ``__graft_entry__``).
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# The reference checkout: AMLP_REFERENCE_ROOT, else a directory named "reference" beside this
# repository. Without it nothing is built (the fixtures under tests/golden stand in for it).
REF_ROOT = os.environ.get("AMLP_REFERENCE_ROOT") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
KERNEL_DIR = os.path.join(REF_ROOT, "nep_simulator", "cudakernels")
SKIP = {"radial_grad", "g_all"}

_PRELUDE = r"""
#include <math.h>
#include <cmath>
#include <cstdint>
using std::sqrt;
struct amlp_dim3 { int x, y, z; };
static amlp_dim3 blockIdx, threadIdx, blockDim, gridDim;
#define __global__
#define __device__
#define __restrict__ __restrict
"""

_RAW = re.compile(r"cp\.RawKernel\(\s*r'''(.*?)'''\s*,\s*'(\w+)'\s*\)", re.S)


def _strip_comments(s: str) -> str:
    s = re.sub(r"/\*.*?\*/", "", s, flags=re.S)
    return re.sub(r"//[^\n]*", "", s)


def kernel_sources(kernel_dir: str = KERNEL_DIR) -> dict[str, tuple[str, str]]:
    """{kernel name: (source string, file name)} for every RawKernel string."""
    out = {}
    for fn in sorted(os.listdir(kernel_dir)):
        if not fn.endswith(".py"):
            continue
        with open(os.path.join(kernel_dir, fn)) as fh:
            text = fh.read()
        for m in _RAW.finditer(text):
            out[m.group(2)] = (m.group(1), fn)
    return out


def parse_params(src: str, name: str) -> list[tuple[str, str]]:
    """[(C type, parameter name)] of kernel ``name``."""
    s = _strip_comments(src)
    m = re.search(r"\b" + name + r"\s*\((.*?)\)\s*\{", s, re.S)
    if not m:
        raise RuntimeError(f"signature of {name} not found")
    params = []
    for p in m.group(1).split(","):
        p = " ".join(p.replace("__restrict__", "").split())
        pm = re.match(r"(.*?)(\w+)$", p)
        params.append((pm.group(1).strip(), pm.group(2)))
    return params


def _wrapper(src: str, name: str) -> str:
    params = parse_params(src, name)
    sig = ", ".join(f"{t} {n}" for t, n in params)
    args = ", ".join(n for _, n in params)
    return (_PRELUDE + src + f"""
extern "C" void launch_{name}(int gx, int bx{', ' if sig else ''}{sig}) {{
  blockDim.x = bx; blockDim.y = blockDim.z = 1;
  gridDim.x = gx; gridDim.y = gridDim.z = 1;
  for (int b = 0; b < gx; ++b)
    for (int t = 0; t < bx; ++t) {{
      blockIdx.x = b; blockIdx.y = blockIdx.z = 0;
      threadIdx.x = t; threadIdx.y = threadIdx.z = 0;
      {name}({args});
    }}
}}
""")


def build(kernel_dir: str = KERNEL_DIR, out_dir: str = OUT, verbose: bool = False) -> list[str]:
    """Compile every buildable kernel; returns the names built. No-op (empty
    list) when the reference checkout is absent."""
    if not os.path.isdir(kernel_dir):
        return []
    os.makedirs(out_dir, exist_ok=True)
    built = []
    for name, (src, fn) in kernel_sources(kernel_dir).items():
        if name in SKIP:
            continue
        cpp = os.path.join(out_dir, f"ref_{name}.cpp")
        so = os.path.join(out_dir, f"ref_{name}.so")
        code = f"// generated from {fn} kernel {name}; do not commit\n" + _wrapper(src, name)
        if not (os.path.exists(cpp) and open(cpp).read() == code and os.path.exists(so)):
            with open(cpp, "w") as fh:
                fh.write(code)
            cmd = ["g++", "-O2", "-shared", "-fPIC", "-ffp-contract=off", "-w", "-o", so, cpp]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        built.append(name)
    with open(os.path.join(out_dir, "params.txt"), "w") as fh:
        for name, (src, fn) in kernel_sources(kernel_dir).items():
            if name not in SKIP:
                fh.write(name + " " + ";".join(f"{t}|{n}" for t, n in parse_params(src, name)) + "\n")
    return built


def load(name: str, out_dir: str = OUT):
    """(ctypes function, [(type, name)]) of a built kernel launcher."""
    params = None
    with open(os.path.join(out_dir, "params.txt")) as fh:
        for line in fh:
            k, _, rest = line.strip().partition(" ")
            if k == name:
                params = [tuple(x.split("|")) for x in rest.split(";")] if rest else []
    if params is None:
        raise KeyError(name)
    lib = ctypes.CDLL(os.path.join(out_dir, f"ref_{name}.so"))
    fn = getattr(lib, f"launch_{name}")
    argtypes = [ctypes.c_int, ctypes.c_int]
    for t, _ in params:
        argtypes.append(ctypes.c_void_p if "*" in t else ctypes.c_int)
    fn.argtypes = argtypes
    fn.restype = None
    return fn, params


if __name__ == "__main__":
    print(build(verbose=True), file=sys.stderr)
