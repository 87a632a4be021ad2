"""Builds libsphradiometer_b200.so in-tree (sm_100a).

CUDA sources are compiled with nvcc for ``compute_100a/sm_100a`` only; the
C-ABI host sources (which use C99 ``double _Complex`` through the public
headers) with g++; everything is linked by nvcc with the static CUDA
runtime, so the library depends on the driver only.  Run as
``python -m sphradiometer_b200.build`` or through ``__graft_entry__.build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "libsphradiometer_b200.so")
OBJ = os.path.join(HERE, "_build")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]
CXX_FLAGS = ["-O2", "-std=gnu++17", "-fPIC", "-Wall", "-Wno-unused-function"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_include() -> str:
    return os.path.join(os.path.dirname(os.path.dirname(_nvcc())), "include")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("compile step failed: " + os.path.basename(cmd[-1]))
    return r


def sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _stale(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h") or f.endswith(".cuh")]
    headers += [os.path.join(dp, f) for dp, _, fs in os.walk(INCLUDE) for f in fs]
    objs = []
    cu, cpp = sources()
    for f in cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        if _stale(obj, [src] + headers):
            _run([nvcc] + NVCC_FLAGS + ["-I", INCLUDE, "-c", src, "-o", obj])
            if verbose:
                print("nvcc", f)
        objs.append(obj)
    for f in cpp:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        if _stale(obj, [src] + headers):
            _run(["g++"] + CXX_FLAGS + ["-I", INCLUDE, "-I", _cuda_include(), "-c", src, "-o", obj])
            if verbose:
                print("g++", f)
        objs.append(obj)
    if _stale(OUT, objs):
        _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", OUT] + objs + ["-Xlinker", "--no-undefined"])
        if verbose:
            print("link", os.path.basename(OUT))
    return OUT


if __name__ == "__main__":
    print(build(verbose=True))
