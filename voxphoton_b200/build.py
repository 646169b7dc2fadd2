"""Build libvox.so in-tree with nvcc for sm_100a (B200).

    python -m voxphoton_b200.build          # incremental
    python -m voxphoton_b200.build --force  # rebuild

The shared library lands next to this file (voxphoton_b200/libvox.so) so that
it travels with the source tree; the ctypes loader in voxphoton_b200/_lib.py
loads exactly that file.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libvox.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _sources():
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".cpp", ".h"))]
    srcs.append(os.path.join(os.path.dirname(HERE), "include", "vox.h"))
    return srcs


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(s) > t for s in _sources())


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    """Compile api.cu (all device code) and assembly.cpp into libvox.so."""
    if not force and not _stale():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    extra = list(extra or [])
    cmds = [
        [NVCC, *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, "api.cu"),
         "-o", os.path.join(objdir, "api.o")],
        [os.environ.get("CXX", "g++"), "-O3", "-std=c++17", "-fPIC", "-pthread", "-c",
         os.path.join(CSRC, "assembly.cpp"), "-o", os.path.join(objdir, "assembly.o")],
        [NVCC, *ARCH, "-shared", "-o", OUT + ".tmp", os.path.join(objdir, "api.o"),
         os.path.join(objdir, "assembly.o"), "-lcudart", "-lpthread"],
    ]
    for c in cmds:
        if verbose:
            print(" ".join(c), flush=True)
        r = subprocess.run(c, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed ({' '.join(c)}):\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    force = "--force" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else None
    print(build(force=force, verbose=True, extra=extra))
