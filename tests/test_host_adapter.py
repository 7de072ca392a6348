"""The C++ host adapter (inq-wannier-fork_b200/host/inq_b200.hpp) compiles against the
C ABI and, on a GPU, drives the kernels through INQ's HamiltonianType seam."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "host_adapter_check.cpp")
LIBDIR = os.path.join(ROOT, "inq-wannier-fork_b200", "lib")


def _build(tmp_path):
    exe = os.path.join(str(tmp_path), "host_adapter_check")
    cmd = ["g++", "-std=c++17", "-O2", SRC, "-I/usr/local/cuda/include", "-L" + LIBDIR, "-linqb200",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_host_adapter_compiles_and_links(pb, tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_host_adapter_runs(pb, tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    vals = dict(line.split() for line in r.stdout.strip().splitlines())
    assert float(vals["ho_mean_abs_diff"]) == pytest.approx(0.0051420503, rel=1.2e-5)
    assert float(vals["exp_generic_vs_fused"]) < 1e-12
    assert float(vals["etrs_norm"]) > 0.0
