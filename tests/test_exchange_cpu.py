"""Exact exchange is not provided: every theory this library runs has exchange
coefficient 0, where INQ's exchange_operator is disabled (exchange_operator.hpp:229-231)
and adds nothing to H|phi> (ks_hamiltonian.hpp:147).  Both host interfaces refuse a
coefficient INQ would treat as enabled, before any device work (runs on the CPU)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "exchange_check.cpp")
LIBDIR = os.path.join(ROOT, "inq-wannier-fork_b200", "lib")


def test_cpp_adapter_refuses_exact_exchange(pb, tmp_path):
    exe = os.path.join(str(tmp_path), "exchange_check")
    cmd = ["g++", "-std=c++17", "-O1", SRC, "-I/usr/local/cuda/include", "-L" + LIBDIR, "-linqb200",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "bad=0", r.stdout + r.stderr


@pytest.mark.parametrize("coefficient", [0.25, 1.0, -0.5])
def test_python_binding_refuses_exact_exchange(pb, coefficient):
    with pytest.raises(ValueError, match="exact exchange is not provided"):
        pb.KSHamiltonian([10.0, 10.0, 10.0], (16, 16, 16), "fp64", exchange_coefficient=coefficient)
