"""Build libnb6b200.so in-tree for sm_100a.

    python nbody6ppgpu-beijing_b200/build.py [--force] [-v]

Every ``csrc/*.cu`` file is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into one
shared object next to this file, which the ``nb6b200`` package loads.  The
CUDA runtime is linked statically, so the library needs only the driver.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libnb6b200.so")
BUILD_DIR = os.path.join(HERE, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-O2",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    return any(os.path.getmtime(d) > t for d in deps)


DRIVER_SRCS = [os.path.join(HERE, "driver", f) for f in ("blockstep.cpp", "ensemble.cpp")]
DRIVER_DEPS = DRIVER_SRCS + [os.path.join(HERE, "driver", "hermite.h")]
DRIVER_LIB = os.path.join(HERE, "libnb6drive.so")


def build_driver(force: bool = False, verbose: bool = False) -> str:
    """The C++ block-step drivers, single cluster and ensemble (host code only,
    loads force backends with dlopen)."""
    if (not force and os.path.exists(DRIVER_LIB)
            and all(os.path.getmtime(DRIVER_LIB) >= os.path.getmtime(d) for d in DRIVER_DEPS)):
        return DRIVER_LIB
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-pthread", "-o", DRIVER_LIB + ".tmp",
           *DRIVER_SRCS, "-ldl"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(DRIVER_LIB + ".tmp", DRIVER_LIB)
    return DRIVER_LIB


def build(force: bool = False, verbose: bool = False) -> str:
    build_driver(force=force, verbose=verbose)
    if not force and not _stale():
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc, *NVCC_FLAGS, "-Xptxas", "-v" if verbose else "-O3", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
           "-Xcompiler", "-fPIC", "-cudart", "static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose=args.verbose))
    sys.exit(0)
