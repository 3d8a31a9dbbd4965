"""Builds the native library in-tree: autan_b200/_lib/libautan_b200.so (host set-up in C++ and the
sm_100a CUDA kernels behind the C ABI of include/autan_euler_device.h).

    python -m autan_b200.build          # incremental: recompiles sources newer than their object

Device code is compiled for sm_100a only, with --fmad=false: the kernels repeat the reference
host's arithmetic operation for operation (the reference builds its device code the same way,
CMakeLists.txt:49-50), so FMA contraction would change the last bits.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent
REPO = ROOT.parent
CSRC = ROOT / "csrc"
OBJ = ROOT / "_lib" / "obj"
LIB = ROOT / "_lib" / "libautan_b200.so"
INCLUDE = REPO / "include"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = Path(NVCC).resolve().parent.parent
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra"]
NVCC_FLAGS = [
    *ARCH,
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--fmad=false",
    "-Xcompiler",
    "-fPIC,-ffp-contract=off",
    "-Xptxas",
    "-warn-spills",
]

HOST_SOURCES = ["setup.cpp"]
CUDA_SOURCES = ["euler_device.cu", "norms_static.cu", "mlp.cu", "setup_device.cu"]
HEADERS = ["euler_bodies.cuh", "exact_sum.cuh", "device_mesh.hpp", "convergence.hpp",
           "setup_rules.cuh", "mlp_fused.cuh"]


def _newer(src: Path, obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.exists() and p.stat().st_mtime > t for p in [src, *deps])


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose_ptxas: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    deps = [CSRC / h for h in HEADERS] + sorted(INCLUDE.glob("*.h"))
    objs = []
    for s in HOST_SOURCES:
        src, obj = CSRC / s, OBJ / (s + ".o")
        if _newer(src, obj, deps):
            _run(["g++", *CXX_FLAGS, f"-I{INCLUDE}", "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    for s in CUDA_SOURCES:
        src, obj = CSRC / s, OBJ / (s + ".o")
        if not src.exists():
            continue
        if _newer(src, obj, deps) or verbose_ptxas:
            flags = list(NVCC_FLAGS)
            if verbose_ptxas:
                flags += ["-Xptxas", "-v"]
            _run([NVCC, *flags, f"-I{INCLUDE}", f"-I{CSRC}", "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        _run(
            [
                NVCC,
                *ARCH,
                "-shared",
                "-o",
                str(LIB),
                *map(str, objs),
                "-lcudart",
                f"-L{CUDA_HOME / 'lib64'}",
            ]
        )
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
