"""H|psi> and the FFT on the grids beyond the configurations' own (the lengths of the
FFT size table as cubic grids, and orthorhombic / tetragonal grids) against the oracle
through the C ABI.  INQ takes its grid from the cell and the spacing
(src/basis/real_space.hpp:183-194); here the spacing is 0.32 bohr on every axis and two
atoms carry the Gaussian KB projectors.  FP64 1e-10 max-relative, mixed 1e-6 in norm."""
import numpy as np
import pytest
import torch

from helpers import rel_max, rel_norm

pytestmark = pytest.mark.gpu

GRIDS = [(12, 12, 12), (36, 36, 36), (60, 60, 60), (72, 72, 72), (80, 80, 80), (96, 96, 96), (128, 128, 128),
         (36, 48, 60), (24, 24, 48), (32, 32, 48), (64, 64, 96)]


def _system(nr, M, seed):
    from pinq_b200 import systems

    h = 0.3206
    lattice = np.diag([n * h for n in nr])
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, 1, (2, 3)) * np.array([n * h for n in nr])
    V = systems.gaussian_potential(lattice, nr, pos)
    psi = systems.random_orbitals(lattice, nr, M, 10.0, seed)
    return lattice, pos, V, psi


@pytest.mark.parametrize("nr", GRIDS, ids=lambda nr: "x".join(map(str, nr)))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_apply_h_on_grid_matches_oracle(pb, oracle_mod, nr, precision):
    lattice, pos, V, psi = _system(nr, 3, sum(nr))
    o = oracle_mod.System(lattice, nr)
    o.set_potential(V)
    o.set_projectors(o.build_gaussian_kb(pos))
    kA = o.cart_to_cov(np.array([0.02, -0.01, 0.03]))
    o.set_vector_potential_cov(kA)
    ref = o.apply_h(psi)
    h = pb.KSHamiltonian(lattice, nr, precision)
    h.set_scalar_potential(V)
    h.set_gaussian_projectors(pos)
    h.set_vector_potential_cov(kA)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    out = h(torch.as_tensor(psi).to("cuda", dt)).cpu().numpy()
    err = rel_max(out, ref) if precision == "fp64" else rel_norm(out, ref)
    assert err < (1e-10 if precision == "fp64" else 1e-6), err


@pytest.mark.parametrize("nr", [(36, 48, 60), (96, 96, 96), (128, 128, 128)], ids=lambda nr: "x".join(map(str, nr)))
def test_fft_on_grid_matches_numpy(pb, nr):
    rng = np.random.default_rng(7)
    N = int(np.prod(nr))
    psi = rng.standard_normal((N, 2)) + 1j * rng.standard_normal((N, 2))
    h = pb.KSHamiltonian(np.diag([10.0, 11.0, 12.0]), nr, "fp64")
    f = h.to_fourier(torch.as_tensor(psi).to("cuda")).cpu().numpy()
    ref = np.fft.fftn(psi.reshape(*nr, 2), axes=(0, 1, 2)).reshape(-1, 2)
    assert rel_max(f, ref) < 1e-13
    b = h.to_real(torch.as_tensor(f).to("cuda")).cpu().numpy()
    assert rel_max(b, psi) < 1e-13
