"""Build recipe for libmldgpu.so (sm_100a CUDA kernels + C ABI + host mirror).

Run ``python mld2p4-2_b200/build.py`` (or ``__graft_entry__.build()``).  nvcc
cross-compiles for sm_100a without a GPU; the shared library is written
in-tree next to this file so it travels with the repository snapshot.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmldgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["mldg_core.cu"]
CXX_SOURCES = ["mldg_tri.cpp", "host/mld_hier.cpp", "host/mld_prec.cpp", "host/mld_mmio.cpp"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} ({r.returncode})")
    return r.stdout + r.stderr


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers += [os.path.join(CSRC, "host", f) for f in os.listdir(os.path.join(CSRC, "host"))
                if f.endswith(".h")]
    headers += [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(o, [s] + headers):
            out = _run([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-fopenmp,-Werror=return-type",
                        "-Xptxas", "-v", "-I", INC, "-I", CSRC, "-c", s, "-o", o])
            with open(os.path.join(BUILD, os.path.basename(src) + ".ptxas.txt"), "w") as f:
                f.write(out)
            if verbose:
                print(out)
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if force or _stale(o, [s] + headers):
            _run(["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
                  "-I", INC, "-I", CSRC, "-I", "/usr/local/cuda/include", "-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
