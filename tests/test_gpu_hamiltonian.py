"""GPU parity of H|psi> and the FFTs (CUDA kernels through the C ABI) against the
CPU FP64 oracle.  FP64 path: max |diff| / max |ref| <= 1e-10.  Mixed path
(complex64 FFT and pointwise, FP64 projection accumulators): ||diff|| / ||ref|| <= 1e-6."""
import numpy as np
import pytest
import torch

from helpers import make_oracle, make_product, rel_max, rel_norm, small_system

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MIXED_TOL = 1e-6


def _dev(a, dtype=torch.complex128):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.fixture(scope="module")
def cfg0_small(pb):
    return small_system(pb, n=32, M=8, seed=3)


@pytest.mark.parametrize("M", [1, 5, 8])
def test_fft_forward_backward_fp64(pb, oracle_mod, M):
    lat = np.diag([9.0, 10.0, 11.0])
    nr = (32, 32, 32)
    rng = np.random.default_rng(M)
    psi = rng.standard_normal((32 ** 3, M)) + 1j * rng.standard_normal((32 ** 3, M))
    o = oracle_mod.System(lat, nr)
    h = pb.KSHamiltonian(lat, nr, "fp64")
    f = h.to_fourier(_dev(psi)).cpu().numpy()
    assert rel_max(f, o.fft3d(psi, -1)) < 1e-13
    b = h.to_real(_dev(f)).cpu().numpy()
    assert rel_max(b, psi) < 1e-13


@pytest.mark.parametrize("n", [16, 20, 24, 40, 48, 64])
def test_fft_sizes_fp64(pb, n):
    lat = np.eye(3) * 10.0
    nr = (n, n, n)
    rng = np.random.default_rng(n)
    M = 3
    psi = rng.standard_normal((n ** 3, M)) + 1j * rng.standard_normal((n ** 3, M))
    h = pb.KSHamiltonian(lat, nr, "fp64")
    f = h.to_fourier(_dev(psi)).cpu().numpy()
    ref = np.fft.fftn(psi.reshape(n, n, n, M), axes=(0, 1, 2)).reshape(-1, M)
    assert rel_max(f, ref) < 1e-13


def test_fft_strided_ld(pb, oracle_mod):
    lat = np.eye(3) * 10.0
    nr = (24, 24, 24)
    rng = np.random.default_rng(0)
    full = rng.standard_normal((24 ** 3, 10)) + 1j * rng.standard_normal((24 ** 3, 10))
    h = pb.KSHamiltonian(lat, nr, "fp64")
    x = _dev(full)
    view = x[:, 2:7]  # M = 5, ld = 10
    out = torch.zeros_like(x)
    h.to_fourier(view, out[:, 2:7])
    o = oracle_mod.System(lat, nr)
    res = out.cpu().numpy()
    assert rel_max(res[:, 2:7], o.fft3d(full[:, 2:7], -1)) < 1e-13
    assert np.all(res[:, :2] == 0) and np.all(res[:, 7:] == 0)


def test_apply_h_fp64_matches_oracle(pb, oracle_mod, cfg0_small):
    s = cfg0_small
    o = make_oracle(oracle_mod, s)
    h = make_product(pb, s)
    out = h(_dev(s["psi"])).cpu().numpy()
    assert rel_max(out, o.apply_h(s["psi"])) < FP64_TOL


def test_apply_h_fp64_vector_potential(pb, oracle_mod, cfg0_small):
    s = cfg0_small
    o = oracle_mod.System(s["lattice"], s["nr"])
    kA = o.cart_to_cov(np.array([0.05, -0.02, 0.03]))
    o = make_oracle(oracle_mod, s, kA)
    h = make_product(pb, s, "fp64", kA)
    out = h(_dev(s["psi"])).cpu().numpy()
    assert rel_max(out, o.apply_h(s["psi"])) < FP64_TOL


def test_apply_h_in_place_and_ragged(pb, oracle_mod):
    s = small_system(pb, n=32, M=7, seed=5)
    o = make_oracle(oracle_mod, s)
    h = make_product(pb, s)
    x = _dev(s["psi"])
    h.apply(x, out=x)
    assert rel_max(x.cpu().numpy(), o.apply_h(s["psi"])) < FP64_TOL


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_apply_h_repeatable(pb, cfg0_small, precision):
    """The projections are summed in a fixed order (the projection kernel), so two
    applies agree bit for bit."""
    h = make_product(pb, cfg0_small, precision)
    x = _dev(cfg0_small["psi"], torch.complex128 if precision == "fp64" else torch.complex64)
    a = h(x)
    b = h(x)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_harmonic_oscillator_golden(pb):
    """ks_hamiltonian.hpp:356-397 through the CUDA path: 0.0051420503."""
    from pinq_b200 import systems

    lat = np.eye(3) * 10.0
    nr = (20, 20, 20)
    r2 = (systems.rvectors(lat, nr) ** 2).sum(1)
    w = 2.0
    h = pb.KSHamiltonian(lat, nr, "fp64")
    h.set_scalar_potential(0.5 * w * w * r2)
    psi = np.tile(np.exp(-w * r2)[:, None], (1, 6)).astype(complex)
    out = h(_dev(psi)).cpu().numpy()
    diff = np.abs(out - 1.5 * w * psi).sum() / out.size
    assert diff == pytest.approx(0.0051420503, rel=1.2e-5)


def test_constant_and_plane_waves(pb):
    """ks_hamiltonian.hpp:276-354 through the CUDA path (< 1e-14)."""
    from pinq_b200 import systems

    lat = np.eye(3) * 10.0
    nr = (20, 20, 20)
    h = pb.KSHamiltonian(lat, nr, "fp64")
    M = 6
    one = np.ones((8000, M), complex)
    assert np.abs(h(_dev(one)).cpu().numpy()).sum() / one.size < 1e-14
    kk = 2 * np.pi / 10.0
    x = systems.rvectors(lat, nr)[:, 0]
    psi = np.stack([np.exp(1j * n * kk * x) for n in range(M)], 1)
    out = h(_dev(psi)).cpu().numpy()
    assert np.abs(out - 0.5 * (np.arange(M) * kk) ** 2 * psi).sum() / out.size < 1e-14


def test_orthorhombic_plane_wave(pb):
    """laplacian.hpp:99-151 cell (9 x 12 x 10 -> 18 x 24 x 20), 13 states."""
    from pinq_b200 import systems

    lat = np.diag([9.0, 12.0, 10.0])
    nr = (18, 24, 20)
    h = pb.KSHamiltonian(lat, nr, "fp64")
    kvec = 2 * np.pi * np.array([1 / 9.0, 1 / 12.0, 1 / 10.0])
    r = systems.rvectors(lat, nr)
    psi = np.stack([(ist + 1.0) * np.exp(1j * r @ kvec) for ist in range(13)], 1)
    out = h(_dev(psi)).cpu().numpy()
    assert np.abs(out - 0.5 * (kvec @ kvec) * psi).sum() < 1e-8


def test_apply_h_mixed_matches_oracle(pb, oracle_mod, cfg0_small):
    s = cfg0_small
    o = make_oracle(oracle_mod, s)
    h = make_product(pb, s, "mixed")
    out = h(_dev(s["psi"], torch.complex64)).cpu().numpy()
    ref = o.apply_h(s["psi"])
    err = rel_norm(out, ref)
    assert err < MIXED_TOL, err


def test_apply_h_host_buffers(pb, cfg0_small):
    s = cfg0_small
    h = make_product(pb, s)
    dev = h(_dev(s["psi"])).cpu().numpy()
    host = h.apply_host(np.ascontiguousarray(s["psi"]))
    assert rel_max(host, dev) < 1e-14


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_apply_h_host_buffers_chunked(pb, precision):
    """inqb_apply_h_host with more orbitals than one chunk and a ragged last chunk (77
    orbitals: chunks of 32, 32 and 13, copied in, applied and copied out on three
    streams) gives the device-resident apply bit for bit."""
    s = small_system(pb, n=32, M=77, seed=31)
    h = make_product(pb, s, precision)
    psi = np.ascontiguousarray(s["psi"])
    if precision == "mixed":
        psi = psi.astype(np.complex64)
    dev = h(torch.as_tensor(psi).to("cuda")).cpu().numpy()
    host = h.apply_host(psi)
    assert host.dtype == dev.dtype and np.array_equal(host, dev)


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("mixed", MIXED_TOL)])
def test_apply_h_fourier_mask(pb, oracle_mod, cfg0_small, precision, tol):
    """INQ's zero_outside_sphere on the Laplacian term (transform.hpp:363-364), k + A != 0."""
    s = cfg0_small
    o = oracle_mod.System(s["lattice"], s["nr"])
    kA = o.cart_to_cov(np.array([0.03, 0.01, -0.02]))
    o = make_oracle(oracle_mod, s, kA)
    o.set_fourier_mask(True)
    h = make_product(pb, s, precision, kA)
    h.set_fourier_sphere_mask(True)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    out = h(_dev(s["psi"], dt)).cpu().numpy()
    ref = o.apply_h(s["psi"])
    err = rel_max(out, ref) if precision == "fp64" else rel_norm(out, ref)
    assert err < tol, err


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_band_energies_match_oracle(pb, oracle_mod, cfg0_small, precision, tol):
    """inqb_band_energies (overlap_diagonal_normalized(H psi, psi, real_part)) against
    the oracle's H psi and band energies, relative to the largest |eps|."""
    s = cfg0_small
    o = make_oracle(oracle_mod, s)
    ref = o.band_energies(s["psi"], o.apply_h(s["psi"]))
    h = make_product(pb, s, precision)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    eps = h.band_energies(_dev(s["psi"], dt))
    assert np.abs(eps - ref).max() <= tol * np.abs(ref).max(), (eps, ref)
