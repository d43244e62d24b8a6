"""Build the in-tree native libraries.

``libqas.so``: every CUDA kernel of the library, compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with ``--fmad=false`` so that no
multiply-add is contracted and each IEEE operation matches the reference CPU
build; cudart is linked statically, so the library needs only the driver.

Usage: ``python -m qasmhd_b200.build`` (or ``build_library()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libqas.so")
SOURCES = ["qas_api.cu"]
HEADERS = ["qas_device.cuh", "qas_kernels.cuh", "qas_dissip.cuh", "qas_batch.cuh", "qas_batch_api.inc",
           "qas_adjoint.cuh", "qas_adjoint_kernels.cuh", "qas_adjoint_api.inc", "qas_noalloc.inc",
           "qas_io.inc", "qas_tma.cuh", "qas_dd.inc", "qas_hall.cuh", "qas_pipe.cuh", "qas_pipe.inc"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "--fmad=false", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared", "-cudart=static",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "qas.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_library(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, "-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    print(LIB)
