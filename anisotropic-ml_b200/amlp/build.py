"""Build recipe of ``libamlp.so`` (sm_100a) from ``csrc/``.

``python -m amlp.build`` (from the package root) or ``build()`` compiles every
``csrc/*.cu`` with nvcc for ``sm_100a`` into objects under ``_build/`` and links
``amlp/libamlp.so`` in the source tree, so that the library travels with the
repository. Rebuilds only what changed (source, shared headers or flags).
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG_ROOT), "include")
OBJ_DIR = os.path.join(PKG_ROOT, "_build")
LIB = os.path.join(PKG_ROOT, "amlp", "libamlp.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I", INCLUDE]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _headers_digest() -> str:
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for fn in sorted(os.listdir(d)):
            if fn.endswith((".cuh", ".h")):
                with open(os.path.join(d, fn), "rb") as fh:
                    h.update(fn.encode() + fh.read())
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()


def _compile(src: str, obj: str, stamp: str, verbose: bool, extra: list[str]) -> None:
    with open(src, "rb") as fh:
        key = hashlib.sha256(fh.read() + stamp.encode() + " ".join(extra).encode()).hexdigest()
    keyf = obj + ".key"
    if os.path.exists(obj) and os.path.exists(keyf) and open(keyf).read() == key:
        return
    cmd = [nvcc()] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    with open(keyf, "w") as fh:
        fh.write(key)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile and link; returns the library path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    stamp = _headers_digest()
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    objs = [os.path.join(OBJ_DIR, f[:-3] + ".o") for f in srcs]
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda so: _compile(os.path.join(CSRC, so[0]), so[1], stamp, verbose or ptxas_info, extra),
                    zip(srcs, objs)))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
