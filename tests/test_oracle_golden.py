"""Pins the CPU oracle to the reference's own unit-test golden values.

Each test restates one reference unit test (file:line in its docstring) on the
oracle.  The oracle is then trusted as the checker of the CUDA kernels.
"""
import numpy as np
import pytest

from pinq_b200 import systems

SPACING = 0.49672941  # the reference tests' grid spacing


def _grid(lengths, spacing=SPACING):
    return tuple(int(round(L / spacing)) for L in lengths)


def test_harmonic_oscillator_golden(oracle_mod):
    """ks_hamiltonian.hpp:356-397: V = w^2 r^2 / 2, psi = exp(-w r^2), w = 2, 20^3 grid,
    6 states -> mean |H psi - 1.5 w psi| = 0.0051420503 (Catch Approx, rel 1.2e-5)."""
    lat = np.eye(3) * 10.0
    nr = _grid([10.0] * 3)
    assert nr == (20, 20, 20)
    o = oracle_mod.System(lat, nr)
    assert o.volume_element == pytest.approx(0.125)
    r = o.rvectors()
    r2 = (r ** 2).sum(1)
    w = 2.0
    o.set_potential(0.5 * w * w * r2)
    psi = np.tile(np.exp(-w * r2)[:, None], (1, 6)).astype(complex)
    h = o.apply_h(psi)
    diff = np.abs(h - 1.5 * w * psi).sum() / h.size
    assert diff == pytest.approx(0.0051420503, rel=1.2e-5)


def test_constant_and_plane_waves(oracle_mod):
    """ks_hamiltonian.hpp:276-354: H 1 = 0 and H e^{i n k x} = (n k)^2/2 e^{i n k x}, < 1e-14."""
    lat = np.eye(3) * 10.0
    nr = _grid([10.0] * 3)
    o = oracle_mod.System(lat, nr)
    M = 6
    psi = np.ones((o.N, M), complex)
    assert np.abs(o.apply_h(psi)).sum() / psi.size < 1e-14
    kk = 2 * np.pi / 10.0
    x = o.rvectors()[:, 0]
    psi = np.stack([np.exp(1j * n * kk * x) for n in range(M)], 1)
    h = o.apply_h(psi)
    assert np.abs(h - 0.5 * (np.arange(M) * kk) ** 2 * psi).sum() / h.size < 1e-14


@pytest.mark.parametrize("cell", ["orthorhombic", "rotated", "fcc"])
def test_plane_wave_kinetic_cells(oracle_mod, cell):
    """laplacian.hpp:92-299: plane waves in orthorhombic, rotated and non-orthogonal
    cells, 13 states scaled by (ist+1); the reference sums |error| over the grid and
    states and requires < 1e-8 (at factor 0.673214; the factor of H is 1/2)."""
    if cell == "orthorhombic":
        lat = np.diag([9.0, 12.0, 10.0])
        kvec = 2 * np.pi * np.array([1 / 9.0, 1 / 12.0, 1 / 10.0])
    elif cell == "rotated":
        ll = 9.0
        lat = np.array([[ll / np.sqrt(2), ll / np.sqrt(2), 0.0], [-ll / np.sqrt(2), ll / np.sqrt(2), 0.0],
                        [0.0, 0.0, ll]])
        kvec = 2 * np.pi * np.array([np.sqrt(2.0) / ll, np.sqrt(2.0) / ll, 0.0])
    else:
        ll = 5.89
        lat = np.array([[0.0, ll, ll], [ll, 0.0, ll], [ll, ll, 0.0]])
        recip = 2 * np.pi * np.linalg.inv(lat).T
        kvec = (2.0 + 3.0 - 1.0) * recip[2]
    nr = _grid(np.linalg.norm(lat, axis=1))
    o = oracle_mod.System(lat, nr)
    r = o.rvectors()
    psi = np.stack([(ist + 1.0) * np.exp(1j * r @ kvec) for ist in range(13)], 1)
    h = o.apply_h(psi)
    diff = np.abs(h - 0.5 * (kvec @ kvec) * psi).sum()
    assert diff < 1e-8


def test_fft_round_trip_gaussians(oracle_mod):
    """transform.hpp:442-545: to_fourier of zero is zero; Gaussians e^{-s r^2} survive a
    round trip with mean |error| < 1e-15 (7 states, s = (ist+1)/2)."""
    lat = np.eye(3) * 10.0
    nr = _grid([10.0] * 3)
    o = oracle_mod.System(lat, nr)
    zero = np.zeros((o.N, 7), complex)
    assert np.abs(o.fft3d(zero, -1)).sum() / zero.size < 1e-15
    r2 = (o.rvectors() ** 2).sum(1)
    psi = np.stack([np.exp(-0.5 * (ist + 1) * r2) for ist in range(7)], 1).astype(complex)
    back = o.fft3d(o.fft3d(psi, -1), +1, normalize=True)
    assert np.abs(back - psi).sum() / psi.size < 1e-15


def test_fft_matches_numpy(oracle_mod):
    """The oracle's own mixed-radix FFT against numpy's (sign -1, unnormalised)."""
    for nr in [(20, 20, 20), (18, 24, 20), (17, 9, 16)]:
        o = oracle_mod.System(np.diag([5.0, 6.0, 7.0]), nr)
        rng = np.random.default_rng(1)
        psi = rng.standard_normal((o.N, 3)) + 1j * rng.standard_normal((o.N, 3))
        ref = np.fft.fftn(psi.reshape(*nr, 3), axes=(0, 1, 2)).reshape(o.N, 3)
        assert np.abs(o.fft3d(psi, -1) - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("nr,M", [((32, 32, 32), 2), ((64, 8, 45), 3), ((7, 12, 30), 1), ((25, 36, 16), 5),
                                  ((2, 3, 49), 4)])
def test_fft_forward_and_inverse_match_numpy(oracle_mod, nr, M):
    """Radices 4, 2, 3, 5, 7 and a prime, with the orbitals as the batch: sign -1
    unnormalised (to_fourier) and sign +1 with 1/N (to_real, transform.hpp:325-331)."""
    o = oracle_mod.System(np.diag([5.0, 6.0, 7.0]), nr)
    rng = np.random.default_rng(sum(nr) + M)
    psi = rng.standard_normal((o.N, M)) + 1j * rng.standard_normal((o.N, M))
    grid = psi.reshape(*nr, M)
    fwd = np.fft.fftn(grid, axes=(0, 1, 2)).reshape(o.N, M)
    inv = np.fft.ifftn(grid, axes=(0, 1, 2)).reshape(o.N, M)
    assert np.abs(o.fft3d(psi, -1) - fwd).max() < 1e-13 * np.abs(fwd).max()
    assert np.abs(o.fft3d(psi, +1, normalize=True) - inv).max() < 1e-13 * np.abs(inv).max()


@pytest.mark.parametrize("center", [(0, 0, 0), (-5, 0, 0), (5, 0, 0), (-5, -5, -5), (5, 5, 5), (2.5, 2.5, 2.5)])
def test_sphere_257_points(oracle_mod, center):
    """spherical_grid.hpp:264-376: radius 2 on a 10 bohr / 0.4967 grid -> 257 points,
    size * dV / (4/3 pi r^3) = 0.9586598525."""
    o = oracle_mod.System(np.eye(3) * 10.0, _grid([10.0] * 3))
    n = len(o.sphere(np.array(center, float), 2.0)[1])
    assert n == 257
    assert n * o.volume_element / (4.0 / 3.0 * np.pi * 8.0) == pytest.approx(0.9586598525, rel=1.2e-5)


def test_dipole_golden(oracle_mod):
    """dipole.hpp:80-100: rho = x e^{-r^2} on orthorhombic 4.2 x 3.5 x 6.4 -> 2.6692428234."""
    lat = np.diag([4.2, 3.5, 6.4])
    o = oracle_mod.System(lat, _grid([4.2, 3.5, 6.4], 0.39770182))
    r = o.rvectors()
    d = o.dipole(r[:, 0] * np.exp(-(r ** 2).sum(1)))
    assert d[0] == pytest.approx(2.6692428234, rel=1.2e-5)
    assert abs(d[1]) < 1e-14 and abs(d[2]) < 1e-14


@pytest.mark.parametrize("factor", [-0.1, -0.1j])
def test_taylor_exponential_on_eigenstates(oracle_mod, factor):
    """exponential.hpp:83-235 pins the order-16 Taylor series on diagonal operators;
    here on plane waves, eigenstates of H with E_n = (n k)^2 / 2."""
    lat = np.eye(3) * 10.0
    o = oracle_mod.System(lat, _grid([10.0] * 3))
    kk = 2 * np.pi / 10.0
    x = o.rvectors()[:, 0]
    M = 6
    psi = np.stack([np.exp(1j * n * kk * x) for n in range(M)], 1)
    E = 0.5 * (np.arange(M) * kk) ** 2
    out = o.exponential(factor, psi, order=16)
    assert np.abs(out - np.exp(factor * E) * psi).max() < 1e-12


@pytest.mark.parametrize("M,tol", [(3, 1e-14), (100, 1e-13)])
def test_orthonormalize(oracle_mod, M, tol):
    """orthogonalize.hpp:79-140: after orthogonalize, |S - I| < 1e-14 (3 states) / 1e-13 (100)."""
    lat = np.eye(3) * 6.3
    nr = _grid([6.3] * 3, 0.44428829)
    o = oracle_mod.System(lat, nr)
    rng = np.random.default_rng(M)
    psi = rng.standard_normal((o.N, M)) + 1j * rng.standard_normal((o.N, M))
    out = o.orthonormalize(psi)
    S = o.volume_element * out.conj().T @ out
    assert np.abs(S - np.eye(M)).max() < tol


def test_etrs_reduces_to_two_taylor_half_steps(oracle_mod):
    """etrs.hpp:22-82 with a density-independent H: psi(t+dt) = T4(i dt/2 H2) T4(i dt/2 H1) psi."""
    lat = np.eye(3) * 10.0
    o = oracle_mod.System(lat, _grid([10.0] * 3))
    r2 = (o.rvectors() ** 2).sum(1)
    o.set_potential(0.5 * r2)
    psi = systems.random_orbitals(lat, o.nr, 3, 5.0, 0)
    kA1 = np.array([0.1, 0.0, 0.0])
    kA2 = np.array([0.3, 0.0, 0.0])
    out = o.etrs_step(psi, 0.05, kA1, kA2)
    o.set_vector_potential_cov(kA1)
    ref = o.exponential(0.025j, psi)
    o.set_vector_potential_cov(kA2)
    ref = o.exponential(0.025j, ref)
    assert np.abs(out - ref).max() == 0.0


def test_fourier_sphere_mask(oracle_mod):
    """transform.hpp:428-440: zero_outside_sphere keeps 0.5160349854 of a 14^3 box
    (cubic 6.66 / 0.46320257); with the mask H's Laplacian acts on those points only."""
    lat = np.eye(3) * 6.66
    nr = _grid([6.66] * 3, 0.46320257)
    assert nr == (14, 14, 14)
    f = [np.where(np.arange(n) >= (n + 1) // 2, np.arange(n) - n, np.arange(n)) / n for n in nr]
    inside = (f[0][:, None, None] ** 2 + f[1][None, :, None] ** 2 + f[2][None, None, :] ** 2) <= 0.25
    assert inside.mean() == pytest.approx(0.5160349854, rel=1.2e-5)
    o = oracle_mod.System(lat, nr)
    o.set_fourier_mask(True)
    rng = np.random.default_rng(4)
    psi = rng.standard_normal((o.N, 2)) + 1j * rng.standard_normal((o.N, 2))
    G = 2 * np.pi * np.stack(np.meshgrid(*[fi * n for fi, n in zip(f, nr)], indexing="ij"), -1) / 6.66
    lap = 0.5 * (G ** 2).sum(-1) * inside
    ref = np.fft.ifftn(lap[..., None] * np.fft.fftn(psi.reshape(*nr, 2), axes=(0, 1, 2)), axes=(0, 1, 2))
    assert np.abs(o.apply_h(psi) - ref.reshape(-1, 2)).max() < 1e-12 * np.abs(ref).max()


def test_band_energies_normalized_overlap(oracle_mod):
    """overlap_diagonal_normalized on the complex field_set of its unit test
    (operations/overlap_diagonal.hpp:280-343): 800 points, 12 vectors,
    aa = 20 (i+1) sqrt(j+1) e^{i(-pi/4 + pi i/7)}, bb = -0.05/(i+1) sqrt(j+1)
    e^{i(pi/4 + pi i/7)}.  Band energies take the real part with phi1 = H psi = aa
    and phi2 = psi = bb.  In closed form conj(aa) bb = -i (j+1), so the ratio is
    -i K with K = 800 / (0.0025 sum_i 1/(i+1)^2) for every vector: real part 0;
    with aa rotated by e^{i pi/3} the real part is -K sqrt(3)/2."""
    i = np.arange(800)[:, None]
    j = np.arange(12)[None, :]
    aa = 20.0 * (i + 1) * np.sqrt(j + 1) * np.exp(1j * (-np.pi / 4 + np.pi / 7 * i))
    bb = -0.05 / (i + 1) * np.sqrt(j + 1) * np.exp(1j * (np.pi / 4 + np.pi / 7 * i))
    K = 800.0 / (0.0025 * (1.0 / (np.arange(800) + 1.0) ** 2).sum())
    o = oracle_mod.System(np.diag([8.0, 10.0, 10.0]), (8, 10, 10))
    eps = o.band_energies(bb, aa)
    assert np.abs(eps).max() < 1e-13 * K
    eps = o.band_energies(bb, aa * np.exp(1j * np.pi / 3))
    assert np.allclose(eps, -K * np.sqrt(3.0) / 2.0, rtol=1e-13, atol=0)
