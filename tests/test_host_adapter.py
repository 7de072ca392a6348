"""The C++ host adapter (inq-wannier-fork_b200/host/inq_b200.hpp) compiles against the
C ABI and, on a GPU, drives the kernels through INQ's HamiltonianType seam.  Each value
the adapter check prints is compared with the oracle's run of the same chain: the
harmonic oscillator of ks_hamiltonian.hpp:356-397, a Taylor exponential, one ETRS step,
one self-consistent ETRS step (LDA), a capped self-consistent Crank-Nicolson step, the
TD-MLWF lines and a checkpoint round trip."""
import os
import subprocess

import numpy as np
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


def _oracle_chain(oracle_mod):
    """The adapter check's steps, in the oracle (FP64, same inputs and arguments)."""
    o = oracle_mod.System(np.diag([10.0, 10.0, 10.0]), (20, 20, 20))
    M, w = 6, 2.0
    s = (np.arange(20) - 20 * (np.arange(20) >= 10)) * 0.5
    r2 = (s[:, None, None] ** 2 + s[None, :, None] ** 2 + s[None, None, :] ** 2).reshape(-1)
    V = 0.5 * w * w * r2
    psi = np.repeat(np.exp(-w * r2)[:, None], M, axis=1).astype(np.complex128)
    o.set_potential(V)
    cov = lambda ax: o.cart_to_cov(np.array([ax, 0.0, 0.0]))
    dv = o.volume_element
    out = {}
    b = o.exponential(0.025j, psi)
    b = o.etrs_step(b, 0.05, cov(0.01), cov(0.02))
    out["etrs_norm"] = float((np.abs(b) ** 2).sum() * dv)
    occ = np.full(M, 2.0)
    rho = o.density(b, occ)
    o.ks_potential(rho, V, 2)
    b, rho, it, en = o.etrs_scf_step(b, rho, 0.05, cov(0.0), cov(0.01), occ, V, 2)
    q = float(rho.sum() * dv)
    out.update(scf_iterations=it, scf_charge=q, scf_xc=float(en[2]))
    b, rho, it, en, _ = o.crank_nicolson_scf_step(b, rho, 0.05, cov(0.01), cov(0.02), occ, V, 2, nelec=q,
                                                  max_iter=3)
    out.update(cn_scf_iterations=it, cn_scf_charge=float(rho.sum() * dv))
    return out


def test_host_adapter_compiles_and_links(pb, tmp_path):
    assert os.path.exists(_build(tmp_path))


def test_oracle_chain_of_the_adapter_check(oracle_mod):
    """The oracle's side on its own: the oscillator's step keeps the LDA charge at twice
    the norm, and the capped Crank-Nicolson loop runs its three iterations (the stiff
    oscillator never meets the density test, so the cap is what ends it)."""
    ref = _oracle_chain(oracle_mod)
    assert ref["scf_charge"] == pytest.approx(2.0 * ref["etrs_norm"], rel=1e-3)
    assert ref["cn_scf_iterations"] == 3 and ref["scf_xc"] < 0.0


@pytest.mark.gpu
def test_host_adapter_runs(pb, oracle_mod, tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "ckpt")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    vals = dict(line.split() for line in r.stdout.strip().splitlines())
    assert float(vals["ho_mean_abs_diff"]) == pytest.approx(0.0051420503, rel=1.2e-5)
    assert float(vals["exp_generic_vs_fused"]) < 1e-12
    assert vals["exchange_enabled"] == "0"  # exchange coefficient 0: INQ's operator disabled
    ref = _oracle_chain(oracle_mod)
    for key in ("scf_iterations", "cn_scf_iterations"):
        assert int(vals[key]) == ref[key], key
    for key in ("etrs_norm", "scf_charge", "scf_xc", "cn_scf_charge"):
        assert float(vals[key]) == pytest.approx(ref[key], rel=1e-9), key
    assert int(vals["mlwf_lines"]) == 2 + 6
    assert vals["io_loaded"] == "1" and vals["io_missing_loaded"] == "0"
    assert float(vals["io_maxdiff"]) == 0.0
