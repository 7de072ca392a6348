"""The benchmark sizes: the 64-atom cell (64^3, all 128 orbitals, 256 projectors) and
the large cell (144^3, 480 orbitals, 960 projectors).

On the 64-atom cell H|psi> of all 128 orbitals is compared with the oracle directly
(FP64 1e-12 max-relative; mixed 1e-6 relative in norm, the mixed-precision bound), and
so is one ETRS step of all of them (FP64 1e-11; mixed 1e-5).
Beside that, size-independent properties, which also cover the large cell, where the
oracle would take too long:

  * H is Hermitian: dV Psi^H (H Psi) equals its conjugate transpose (the kinetic term,
    the local potential and the Kleinman-Bylander projectors are each Hermitian).
  * the 3-D transform round trip returns the orbitals;
  * the periodic Poisson kernel is symmetric: <f|P g> = <P f|g> for real fields;
  * the density of orthonormal orbitals integrates to the sum of the occupations;
  * the six TD-MLWF matrices are Hermitian (real weights).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _cell(pb, name, precision, M):
    from pinq_b200 import systems

    if name == "cfg1":
        a, nr = 20.52, (64, 64, 64)
        pos = systems.diamond_positions(10.26, 2)
        ecut = 25.0
    else:
        a, nr = 30.0, (144, 144, 144)
        pos = systems.shell_positions(240, 6.7, seed=0)
        ecut = 30.0
    lat = systems.cubic(a)
    h = pb.KSHamiltonian(lat, nr, precision)
    h.set_scalar_potential(systems.gaussian_potential_device(lat, nr, pos))
    h.set_gaussian_projectors(pos)
    psi = systems.random_orbitals_device(h, M, ecut, seed=7)
    return h, psi


def _herm_defect(h, psi, hpsi, chunk=1 << 18):
    """||A - A^H|| / ||A|| for A = dV Psi^H (H Psi), summed in complex128 over point chunks"""
    M = psi.shape[1]
    a = torch.zeros((M, M), dtype=torch.complex128, device=psi.device)
    for p0 in range(0, psi.shape[0], chunk):
        a += psi[p0:p0 + chunk].to(torch.complex128).conj().T @ hpsi[p0:p0 + chunk].to(torch.complex128)
    a *= h.volume_element
    return float((a - a.conj().T).norm() / a.norm())


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_h_cfg1_all_orbitals_matches_oracle(pb, oracle_mod, precision, tol):
    from pinq_b200 import systems

    h, psi = _cell(pb, "cfg1", precision, 128)
    hpsi = h.apply(psi).to(torch.complex128).cpu().numpy()
    lat = systems.cubic(20.52)
    pos = systems.diamond_positions(10.26, 2)
    o = oracle_mod.System(lat, (64, 64, 64))
    o.set_potential(systems.gaussian_potential_device(lat, (64, 64, 64), pos))
    o.set_projectors(o.build_gaussian_kb(pos))
    ref = o.apply_h(psi.to(torch.complex128).cpu().numpy())
    if precision == "fp64":
        assert np.abs(hpsi - ref).max() / np.abs(ref).max() < tol
    else:
        assert np.linalg.norm(hpsi - ref) / np.linalg.norm(ref) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-11), ("mixed", 1e-5)])
def test_etrs_step_cfg1_all_orbitals_matches_oracle(pb, oracle_mod, precision, tol):
    """One ETRS step (etrs.hpp:22-82) of all 128 orbitals of the 64-atom cell with a
    changing vector potential."""
    from pinq_b200 import systems

    h, psi = _cell(pb, "cfg1", precision, 128)
    lat = systems.cubic(20.52)
    pos = systems.diamond_positions(10.26, 2)
    o = oracle_mod.System(lat, (64, 64, 64))
    o.set_potential(systems.gaussian_potential_device(lat, (64, 64, 64), pos))
    o.set_projectors(o.build_gaussian_kb(pos))
    k1 = o.cart_to_cov(np.array([0.01, 0.0, 0.0]))
    k2 = o.cart_to_cov(np.array([0.02, -0.01, 0.0]))
    ref = o.etrs_step(psi.to(torch.complex128).cpu().numpy(), 0.05, k1, k2)
    h.etrs_step_(psi, 0.05, k1, k2)
    out = psi.to(torch.complex128).cpu().numpy()
    if precision == "fp64":
        assert np.abs(out - ref).max() / np.abs(ref).max() < tol
    else:
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 2e-6)])
def test_h_hermitian_cfg1_all_orbitals(pb, precision, tol):
    h, psi = _cell(pb, "cfg1", precision, 128)
    assert _herm_defect(h, psi, h.apply(psi)) < tol


def test_h_hermitian_cfg4_480_orbitals(pb):
    h, psi = _cell(pb, "cfg4", "mixed", 480)
    hpsi = h.apply(psi)
    assert _herm_defect(h, psi, hpsi) < 2e-6
    del hpsi, psi


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-6)])
def test_fft_round_trip_cfg1(pb, precision, tol):
    h, psi = _cell(pb, "cfg1", precision, 128)
    back = h.to_real(h.to_fourier(psi))
    assert float((back - psi).norm() / psi.norm()) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 2e-6)])
def test_poisson_symmetric_and_density_normalised_cfg1(pb, precision, tol):
    h, psi = _cell(pb, "cfg1", precision, 128)
    occ = np.full(128, 2.0)
    rho = h.density(psi, occ)
    assert abs(float(rho.sum()) * h.volume_element - 256.0) < 256.0 * (1e-12 if precision == "fp64" else 1e-6)
    g = torch.rand(h.N, dtype=torch.float64, device="cuda") - 0.5
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    fields = torch.stack([rho, g], 1).to(dt).contiguous()
    pot = h.poisson(fields).to(torch.complex128)
    f, gg = fields.to(torch.complex128)[:, 0], fields.to(torch.complex128)[:, 1]
    lhs = torch.vdot(f, pot[:, 1]).real
    rhs = torch.vdot(pot[:, 0], gg).real
    # normwise: <f|Pg> with a random g cancels, so its own size is not the scale
    scale = f.norm() * pot[:, 1].norm() + pot[:, 0].norm() * gg.norm()
    assert float(abs(lhs - rhs) / scale) < (1e-14 if precision == "fp64" else 1e-7)


def test_mlwf_matrices_hermitian_cfg1(pb):
    h, psi = _cell(pb, "cfg1", "fp64", 128)
    a = h.mlwf_matrices(psi)
    for k in range(6):
        assert float((a[k] - a[k].conj().T).abs().max()) < 1e-12
