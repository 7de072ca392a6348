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
    r = subprocess.run([exe, str(tmp_path / "ckpt")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    vals = dict(line.split() for line in r.stdout.strip().splitlines())
    assert float(vals["ho_mean_abs_diff"]) == pytest.approx(0.0051420503, rel=1.2e-5)
    assert float(vals["exp_generic_vs_fused"]) < 1e-12
    assert float(vals["etrs_norm"]) > 0.0
    # the LDA step keeps the electron count (2 per state times the states' norm) up to
    # the fourth-order Taylor step's departure from unitarity, about 1e-4 for these
    # narrow Gaussians (1/2 |G_max|^2 dt / 2 = 0.5)
    assert 1 <= int(vals["scf_iterations"]) <= 5
    assert float(vals["scf_charge"]) == pytest.approx(2.0 * float(vals["etrs_norm"]), rel=1e-3)
    assert float(vals["scf_xc"]) < 0.0
    # the Crank-Nicolson step with Broyden mixing: capped at 60 iterations, it keeps
    # the charge to the solver's accuracy
    assert 2 <= int(vals["cn_scf_iterations"]) <= 60
    assert float(vals["cn_scf_charge"]) == pytest.approx(float(vals["scf_charge"]), rel=1e-3)
    assert int(vals["mlwf_lines"]) == 2 + 6
    assert vals["io_loaded"] == "1" and vals["io_missing_loaded"] == "0"
    assert float(vals["io_maxdiff"]) == 0.0
