"""The 144^3 grid of the large-cell configuration (cubic a = 30 bohr, h = 0.2083):
H|psi> against the oracle on a few orbitals and four shell atoms, both precisions,
and the FFT against numpy.  A 144^3 tile is 16 rows x 144 points x one 64-byte
run (147 KB of shared memory)."""
import numpy as np
import pytest
import torch

from helpers import rel_max, rel_norm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big(pb):
    from pinq_b200 import systems

    lattice = systems.cubic(30.0)
    nr = (144, 144, 144)
    pos = systems.shell_positions(240, seed=4)[::60]  # four atoms of the shell
    V = systems.gaussian_potential(lattice, nr, pos)
    psi = systems.random_orbitals(lattice, nr, 4, 30.0, seed=5)
    return dict(lattice=lattice, nr=nr, positions=pos, V=V, psi=psi)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_apply_h_144(pb, oracle_mod, big, precision, tol):
    o = oracle_mod.System(big["lattice"], big["nr"])
    o.set_potential(big["V"])
    o.set_projectors(o.build_gaussian_kb(big["positions"]))
    kA = o.cart_to_cov(np.array([0.01, -0.02, 0.005]))
    o.set_vector_potential_cov(kA)
    ref = o.apply_h(big["psi"])
    h = pb.KSHamiltonian(big["lattice"], big["nr"], precision)
    h.set_scalar_potential(big["V"])
    h.set_gaussian_projectors(big["positions"])
    h.set_vector_potential_cov(kA)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    out = h.apply(torch.as_tensor(big["psi"]).to("cuda", dt)).cpu().numpy().astype(np.complex128)
    err = rel_max(out, ref) if precision == "fp64" else rel_norm(out, ref)
    assert err <= tol, err


def test_fft_144_fp64(pb, big):
    h = pb.KSHamiltonian(big["lattice"], big["nr"], "fp64")
    x = torch.as_tensor(big["psi"][:, :2].copy()).to("cuda")
    f = h.to_fourier(x).cpu().numpy()
    ref = np.fft.fftn(big["psi"][:, :2].reshape(144, 144, 144, 2), axes=(0, 1, 2)).reshape(-1, 2)
    assert rel_max(f, ref) < 1e-12
    b = h.to_real(torch.as_tensor(f).to("cuda")).cpu().numpy()
    assert rel_max(b, big["psi"][:, :2]) < 1e-13
