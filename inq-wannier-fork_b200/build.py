"""Build libinqb200.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python inq-wannier-fork_b200/build.py [--force] [-j N]

Objects go to inq-wannier-fork_b200/_build/, the library to
inq-wannier-fork_b200/lib/libinqb200.so.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libinqb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills", "-I" + INCLUDE, "-I" + CSRC]
SOURCES = ["grids_144.cu", "grids_128.cu", "grids_96.cu", "grids_72.cu", "grids_64.cu", "grids_mid.cu", "grids_small.cu",
           "hamiltonian.cu", "batch.cu", "project.cu", "observables.cu", "adjoint.cu", "propagators.cu", "potential.cu", "checkpoint.cu", "wannier.cu", "setup.cpp", "capi.cpp"]


def nvcc() -> str:
    for cand in [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]:
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps(src: str) -> list[str]:
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + \
        [os.path.join(INCLUDE, "inqb200.h"), src]


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, force: bool, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(BUILD, src + ".o")
    if force or _stale(obj, _deps(path)):
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", path, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nvcc(), "-x", "cu", *ARCH, *NVCC_FLAGS, "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if r.stderr.strip() and verbose:
            print(r.stderr, file=sys.stderr)
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_twiddles.py"), os.path.join(CSRC, "twiddles.cuh")],
                   check=True)
    jobs = jobs or min(len(SOURCES), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), SOURCES))
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.v))
