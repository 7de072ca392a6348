"""GPU parity of the propagators and observables against the CPU FP64 oracle."""
import numpy as np
import pytest
import torch

from helpers import make_oracle, make_product, rel_max, rel_norm, small_system

pytestmark = pytest.mark.gpu


def _dev(a, dtype=torch.complex128):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.fixture(scope="module")
def sysd(pb):
    return small_system(pb, n=32, M=4, seed=11)


@pytest.mark.parametrize("factor,order", [(0.025j, 4), (-0.1, 4), (0.05j, 8)])
def test_exponential_fp64(pb, oracle_mod, sysd, factor, order):
    o = make_oracle(oracle_mod, sysd)
    h = make_product(pb, sysd)
    x = h.exponential_(_dev(sysd["psi"]), factor, order).cpu().numpy()
    assert rel_max(x, o.exponential(factor, sysd["psi"], order)) < 1e-10


def test_etrs_steps_fp64_and_mixed(pb, oracle_mod, sysd):
    """Three ETRS steps with a changing vector potential (etrs.hpp:22-82)."""
    o = make_oracle(oracle_mod, sysd)
    h64 = make_product(pb, sysd, "fp64")
    h32 = make_product(pb, sysd, "mixed")
    amps = [0.0, 0.02, -0.01, 0.015]
    ref = sysd["psi"].copy()
    x64 = _dev(sysd["psi"])
    x32 = _dev(sysd["psi"], torch.complex64)
    for n in range(3):
        k1 = o.cart_to_cov(np.array([amps[n], 0.0, 0.0]))
        k2 = o.cart_to_cov(np.array([amps[n + 1], 0.0, 0.0]))
        ref = o.etrs_step(ref, 0.05, k1, k2)
        h64.etrs_step_(x64, 0.05, k1, k2)
        h32.etrs_step_(x32, 0.05, k1, k2)
    assert rel_max(x64.cpu().numpy(), ref) < 1e-10
    # mixed path: complex64 FFTs leave ~4e-7 relative error per H apply, which the
    # 8 Horner applies of a step carry into ~4e-6 per step in the orbitals
    assert rel_norm(x32.cpu().numpy(), ref) < 3e-5


def test_density_and_dipole(pb, oracle_mod, sysd):
    o = make_oracle(oracle_mod, sysd)
    h = make_product(pb, sysd)
    occ = np.array([2.0, 2.0, 1.5, 0.5])
    rho = h.density(_dev(sysd["psi"]), occ)
    rho_ref = o.density(sysd["psi"], occ)
    assert rel_max(rho.cpu().numpy(), rho_ref) < 1e-13
    d = h.dipole(rho)
    d_ref = o.dipole(rho_ref)
    assert np.abs(d - d_ref).max() < 1e-11 * max(1.0, np.abs(d_ref).max())


def test_dipole_golden(pb):
    """The dipole reduction (dipole.hpp:23-40) on rho = x e^{-r^2} against a numpy sum
    (the reference's golden grid 11 x 9 x 16 needs no FFT but is checked on the oracle)."""
    from pinq_b200 import systems

    lat = np.eye(3) * 10.0
    nr = (20, 20, 20)
    r = systems.rvectors(lat, nr)
    rho = r[:, 0] * np.exp(-(r ** 2).sum(1))
    h = pb.KSHamiltonian(lat, nr, "fp64")
    d = h.dipole(torch.as_tensor(rho, device="cuda"))
    ref = (r * rho[:, None]).sum(0) * 1000.0 / 8000
    assert np.abs(d - ref).max() < 1e-13


@pytest.mark.parametrize("precision,M", [("fp64", 3), ("fp64", 40), ("mixed", 16)])
def test_orthonormalize(pb, oracle_mod, precision, M):
    lat = np.eye(3) * 6.3
    nr = (16, 16, 16)
    rng = np.random.default_rng(M)
    psi = rng.standard_normal((16 ** 3, M)) + 1j * rng.standard_normal((16 ** 3, M))
    h = pb.KSHamiltonian(lat, nr, precision)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    x = h.orthonormalize_(_dev(psi, dt)).cpu().numpy().astype(np.complex128)
    S = h.volume_element * x.conj().T @ x
    tol = 1e-13 if precision == "fp64" else 2e-6
    assert np.abs(S - np.eye(M)).max() < tol
    if precision == "fp64":
        o = oracle_mod.System(lat, nr)
        assert rel_max(x, o.orthonormalize(psi)) < 1e-10


def test_orthonormalize_rejects_dependent_set(pb):
    lat = np.eye(3) * 6.3
    nr = (16, 16, 16)
    # second orbital identically zero: the pivot is exactly 0 (zpotrf rejects pivots <= 0)
    psi = np.zeros((16 ** 3, 2), complex)
    psi[:, 0] = 1.0
    h = pb.KSHamiltonian(lat, nr, "fp64")
    with pytest.raises(pb.InqbError) as e:
        h.orthonormalize_(_dev(psi))
    assert e.value.status == 6


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 2e-5)])
def test_crank_nicolson_matches_oracle(pb, oracle_mod, sysd, precision, tol):
    """One Crank-Nicolson step (crank_nicolson.hpp:41-114, steepest_descent.hpp:22-80)
    with a vector potential changing over the step and a fixed three sweeps
    (tol = 0): the same fifteen solver steps on the GPU and in the oracle."""
    o = make_oracle(oracle_mod, sysd)
    h = make_product(pb, sysd, precision)
    k1 = o.cart_to_cov(np.array([0.01, 0.0, 0.0]))
    k2 = o.cart_to_cov(np.array([0.02, 0.0, 0.0]))
    ref, kref, rref = o.crank_nicolson_step(sysd["psi"], 0.05, k1, k2, max_sweeps=3, tol=0.0)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    x = _dev(sysd["psi"], dt)
    k, r = h.crank_nicolson_step_(x, 0.05, k1, k2, max_sweeps=3, tol=0.0)
    assert k == kref == 3
    err = rel_max(x.cpu().numpy(), ref) if precision == "fp64" else rel_norm(x.cpu().numpy(), ref)
    assert err <= tol, err
    assert abs(r - rref) <= 1e-3 * rref + 1e-12


def test_crank_nicolson_converges_and_keeps_norms(pb, oracle_mod, sysd):
    """Solved to a small residual the step is the Cayley transform of H: unitary, so
    the orbital norms are kept; and it agrees with ETRS run with -dt (the reference's
    CN propagates with exp(-i dt H), its ETRS with exp(+i dt H)) to O(dt^3)."""
    h = make_product(pb, sysd, "fp64")
    x = _dev(sysd["psi"])
    n0 = x.norm(dim=0)
    k, r = h.crank_nicolson_step_(x, 0.01, np.zeros(3), np.zeros(3), max_sweeps=300, tol=1e-22)
    assert r < 1e-22 and k < 300
    assert float(((x.norm(dim=0) - n0).abs() / n0).max()) < 1e-10
    o = make_oracle(oracle_mod, sysd)
    e = o.etrs_step(sysd["psi"], -0.01, np.zeros(3), np.zeros(3))
    assert rel_norm(x.cpu().numpy(), e) < 1e-3


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_kick_matches_oracle(pb, oracle_mod, sysd, precision):
    o = make_oracle(oracle_mod, sysd)
    h = make_product(pb, sysd, precision)
    k = np.array([0.05, -0.02, 0.1])
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    x = h.kick_(_dev(sysd["psi"], dt), k).cpu().numpy()
    ref = o.kick(sysd["psi"], k)
    assert rel_max(x, ref) < (1e-14 if precision == "fp64" else 1e-6)
