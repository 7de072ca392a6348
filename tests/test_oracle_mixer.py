"""The Broyden density mixer and the self-consistent Crank-Nicolson step on the CPU.

Golden values of the reference's own tests:
  * mixers/broyden.hpp:163-203: broyden(5, 0.5, 2), two calls;
  * solvers/least_squares.hpp:62-129: three symmetric 2 x 2 systems;
  * observables/density.hpp:269-279: normalize to a given charge.
Both the oracle (a restatement of dgelsd's minimum-norm solve) and the library's
host-side mixer logic (csrc/broyden_host.h: ring bookkeeping and a Cholesky solve,
driven by tests/cpp/broyden_host_check.cpp with plain loops in place of the device
passes) are pinned to them.  The oracle's Crank-Nicolson step with self-consistency
(real_time/crank_nicolson.hpp:41-114) is checked for what it must satisfy: the
non-interacting step equals the converged linear solve, the interacting one converges
and leaves the density of its orbitals, and the iteration cap holds."""
import os
import subprocess

import numpy as np
import pytest

from helpers import make_oracle, rel_max, small_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "broyden_host_check.cpp")

LSQ = {  # name: (matrix, rhs, solution, absolute tolerance of the printed digits)
    "lsq_diagonal": ([[4.0, 0.0], [0.0, 2.0]], [0.0, 1.0], [0.0, 0.5], 1e-12),
    "lsq_symmetric_1": ([[0.89653, 0.41072], [0.41072, 0.69479]], [0.21563, 0.40103], [-0.0327899021, 0.596579],
                        1e-6),
    "lsq_symmetric_2": ([[6432.12, 4502.48], [4502.48, 3151.74]], [1.0, 1.0], [-30.882245351, 44.1177546523], 1e-8),
}
BROYDEN = [([0.0, 22.2], [5.0, 1.1]), ([4.0, 5.5], [4.4419411001, 3.5554591594])]


def _wrap_map(x):
    return np.array([0.5 * x[1] + 1.0, 0.25 * x[0] - 0.5 * x[2], 0.1 * x[0] + 2.0])


def test_oracle_broyden_golden(oracle_mod):
    m = oracle_mod.Broyden(5, 0.5, 2)
    v = np.array([10.0, -20.0])
    for vout, expect in BROYDEN:
        v = m.mix(v, vout)
        assert v == pytest.approx(expect, abs=1e-10)  # the reference prints 10 decimals


@pytest.mark.parametrize("name", sorted(LSQ))
def test_oracle_least_squares_golden(oracle_mod, name):
    a, b, x, tol = LSQ[name]
    assert oracle_mod.least_squares_sym(a, b) == pytest.approx(x, abs=tol)


def test_oracle_least_squares_minimum_norm_when_singular(oracle_mod):
    a = np.array([[1.0, 1.0, 0.0], [1.0, 1.0, 0.0], [0.0, 0.0, 2.0]])
    b = np.array([1.0, 1.0, 4.0])
    x = oracle_mod.least_squares_sym(a, b)
    assert x == pytest.approx(np.linalg.lstsq(a, b, rcond=None)[0], abs=1e-14)
    assert x == pytest.approx([0.5, 0.5, 2.0], abs=1e-14)


def test_oracle_density_normalize(oracle_mod):
    s = oracle_mod.System(np.diag([6.0, 7.0, 8.0]), [10, 12, 14])
    rho = np.sqrt(np.arange(s.N, dtype=float))
    out = s.density_normalize(rho, 33.3)
    assert s.volume_element * out.sum() == pytest.approx(33.3, rel=1e-14)
    assert out == pytest.approx(rho * (out[1] / rho[1]), rel=1e-14)  # one common factor


def _host_check(tmp_path):
    exe = os.path.join(str(tmp_path), "broyden_host_check")
    r = subprocess.run(["g++", "-std=c++17", "-O1", SRC, "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    return {line.split()[0]: line.split()[1:] for line in r.stdout.strip().splitlines()}


def test_library_mixer_host_logic_golden_and_against_the_oracle(oracle_mod, tmp_path):
    out = _host_check(tmp_path)
    for name, (_, _, x, tol) in LSQ.items():
        ok, *vals = out[name]
        assert ok == "1" and [float(v) for v in vals] == pytest.approx(x, abs=tol), name
    for i, (_, expect) in enumerate(BROYDEN):
        ok, *vals = out[f"broyden_{i + 1}"]
        assert ok == "1" and [float(v) for v in vals] == pytest.approx(expect, abs=1e-10)
    # past the ring's wrap-around: the Cholesky solve and the oracle's minimum-norm
    # solve agree, and both reach the map's fixed point
    ok, calls, *vals = out["broyden_wrap"]
    assert ok == "1" and int(calls) == 12
    m = oracle_mod.Broyden(4, 0.3, 3)
    x = np.array([1.0, 0.0, 0.0])
    for _ in range(12):
        x = m.mix(x, _wrap_map(x))
    assert [float(v) for v in vals] == pytest.approx(x, rel=1e-12, abs=1e-14)
    fixed = np.linalg.solve(np.eye(3) - np.array([[0, 0.5, 0], [0.25, 0, -0.5], [0.1, 0, 0]]), [1.0, 0.0, 2.0])
    assert x == pytest.approx(fixed, abs=1e-9)


@pytest.fixture(scope="module")
def cn_system(oracle_mod):
    sysd = small_system(None, n=16, a=8.0, M=3, seed=5, ecut=8.0)
    sysd["positions"] = sysd["positions"][:2]
    k1 = np.array([0.01, 0.0, 0.0])
    k2 = np.array([0.02, 0.0, 0.0])
    return sysd, k1, k2


def test_oracle_cn_scf_noninteracting_equals_the_converged_solve(oracle_mod, cn_system):
    sysd, k1c, k2c = cn_system
    o = make_oracle(oracle_mod, sysd)
    k1, k2 = o.cart_to_cov(k1c), o.cart_to_cov(k2c)
    occ = np.full(3, 2.0)
    ref, _, res_ref = o.crank_nicolson_step(sysd["psi"], 0.05, k1, k2, 300, 1e-14)
    assert res_ref < 1e-14
    o.set_potential(sysd["V"])
    rho = o.density(sysd["psi"], occ)
    out, rho2, iters, en, res = o.crank_nicolson_scf_step(sysd["psi"], rho, 0.05, k1, k2, occ, sysd["V"], 0)
    assert 2 <= iters < 300
    assert rel_max(out, ref) < 1e-5  # stopped on the density, not the residual
    assert np.array_equal(rho2, o.density(out, occ))
    assert en[1] == en[2] == en[3] == 0.0


@pytest.mark.parametrize("theory", [1, 2])
def test_oracle_cn_scf_interacting_converges(oracle_mod, cn_system, theory):
    sysd, k1c, k2c = cn_system
    o = make_oracle(oracle_mod, sysd)
    k1, k2 = o.cart_to_cov(k1c), o.cart_to_cov(k2c)
    occ = np.full(3, 2.0)
    psi = sysd["psi"]
    rho = o.density(psi, occ)
    o.ks_potential(rho, sysd["V"], theory)
    out, rho2, iters, en, res = o.crank_nicolson_scf_step(psi, rho, 0.05, k1, k2, occ, sysd["V"], theory)
    assert 2 < iters < 300  # the mixer ran
    assert np.array_equal(rho2, o.density(out, occ))
    V, en_ref = o.ks_potential(rho2, sysd["V"], theory)
    assert en == pytest.approx(en_ref, rel=1e-13, abs=1e-15)
    assert en[1] > 0.0 and (theory == 1 or en[2] < 0.0)
    n0 = o.volume_element * (np.abs(psi) ** 2).sum(0)
    n1 = o.volume_element * (np.abs(out) ** 2).sum(0)
    assert np.abs(n1 - n0).max() < 1e-4


def test_oracle_cn_scf_iteration_cap(oracle_mod, cn_system):
    sysd, k1c, k2c = cn_system
    o = make_oracle(oracle_mod, sysd)
    occ = np.full(3, 2.0)
    rho = o.density(sysd["psi"], occ)
    o.ks_potential(rho, sysd["V"], 2)
    _, _, iters, _, _ = o.crank_nicolson_scf_step(sysd["psi"], rho, 0.05, o.cart_to_cov(k1c), o.cart_to_cov(k2c),
                                                  occ, sysd["V"], 2, max_iter=2)
    assert iters == 2
