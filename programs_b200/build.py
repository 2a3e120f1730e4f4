"""Build the in-tree shared libraries.

* ``programs_b200/lib/libsolv_gpu.so`` -- the CUDA solvers and their C-ABI
  (``include/solv_gpu.h``), compiled for sm_100a only;
* ``programs_b200/lib/libfvmesh.so`` -- host C++ mesh generation, Gambit
  reading, renumbering and matrix assembly (``programs_b200/csrc/fvmesh.h``).

Run ``python -m programs_b200.build``.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
    "-diag-suppress", "177",
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA solver library cannot be built")
    return cand


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build failed: " + " ".join(cmd))


def build_solver(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libsolv_gpu.so")
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh")) and not f.startswith("fvmesh")]
    deps = srcs + [os.path.join(ROOT, "include", "solv_gpu.h")]
    if force or not _newer(out, deps):
        cu = [s for s in srcs if s.endswith(".cu")]
        _run([_nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-o", out, *cu])
    return out


def build_mesh(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libfvmesh.so")
    deps = [os.path.join(CSRC, "fvmesh.cpp"), os.path.join(CSRC, "fvmesh.h")]
    if force or not _newer(out, deps):
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", out, deps[0]])
    return out


def build_oracle(force: bool = False) -> str:
    """The CPU checker (test infrastructure) -- built, never linked in."""
    d = os.path.join(ROOT, "oracle")
    out = os.path.join(d, "liborc.so")
    deps = [os.path.join(d, f) for f in ("solv_oracle.c", "csr_oracle.c", "solv_oracle.h")]
    if force or not _newer(out, deps):
        _run(["make", "-C", d, "-B" if force else "liborc.so"])
    return out


def build_all(force: bool = False) -> None:
    build_mesh(force)
    build_oracle(force)
    build_solver(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built:", os.listdir(LIB))
