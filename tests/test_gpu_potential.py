"""GPU parity of the density -> potential step (Poisson, LDA, update_hamiltonian) and
of the ETRS step with its self-consistency loop, against the CPU FP64 oracle."""
import numpy as np
import pytest
import torch

from helpers import make_oracle, make_product, rel_max, rel_norm, small_system

pytestmark = pytest.mark.gpu


def _dev(a, dtype=torch.complex128):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.fixture(scope="module")
def sysd(pb):
    return small_system(pb, n=32, M=4, seed=21)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_poisson_matches_oracle(pb, oracle_mod, sysd, precision):
    o = make_oracle(oracle_mod, sysd)
    h = make_product(pb, sysd, precision)
    rho = o.density(sysd["psi"], [2.0, 2.0, 2.0, 2.0])
    rng = np.random.default_rng(5)
    fields = np.stack([rho.astype(complex), sysd["psi"][:, 0], rng.standard_normal(o.N) + 0j], 1)
    ref = o.poisson(fields)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    out = h.poisson(_dev(fields, dt)).cpu().numpy()
    if precision == "fp64":
        assert rel_max(out, ref) < 1e-12
    else:
        # complex64 transforms: ~1e-7 relative per transform
        assert rel_norm(out, ref) < 2e-6


def test_poisson_plane_waves_64(pb):
    """V = 4 pi / |k|^2 rho for plane waves on the 64^3 grid (poisson.hpp:301-373)."""
    from pinq_b200 import systems

    a = 20.52
    lat = systems.cubic(a)
    h = pb.KSHamiltonian(lat, (64, 64, 64), "fp64")
    r = systems.rvectors(lat, (64, 64, 64))
    ks = [np.array([1.0, 0.0, 0.0]), np.array([2.0, -1.0, 3.0])]
    fields = np.stack([np.exp(1j * (2 * np.pi / a) * (r @ k)) for k in ks], 1)
    out = h.poisson(_dev(fields)).cpu().numpy()
    for j, k in enumerate(ks):
        k2 = (2 * np.pi / a) ** 2 * (k @ k)
        assert np.abs(out[:, j] - 4 * np.pi / k2 * fields[:, j]).max() < 1e-11


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("theory", [0, 1, 2])
def test_ks_potential_matches_oracle(pb, oracle_mod, sysd, precision, theory):
    """update_hamiltonian on the device: H|psi> with the new potential and the four
    energies against the oracle."""
    o = make_oracle(oracle_mod, sysd)
    h = make_product(pb, sysd, precision)
    occ = [2.0, 2.0, 2.0, 2.0]
    rho = o.density(sysd["psi"], occ)
    vion = sysd["V"]
    _, en_ref = o.ks_potential(rho, vion, theory)
    en = h.ks_potential(_dev(rho, torch.float64), _dev(vion, torch.float64), theory)
    en = np.array([en["external"], en["hartree"], en["xc"], en["nvxc"]])
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    hp = h.apply(_dev(sysd["psi"], dt)).cpu().numpy()
    hp_ref = o.apply_h(sysd["psi"])
    if precision == "fp64":
        assert rel_max(hp, hp_ref) < 1e-12
        assert np.abs(en - en_ref).max() < 1e-11 * max(1.0, np.abs(en_ref).max())
    else:
        assert rel_norm(hp, hp_ref) < 2e-6
        assert np.abs(en - en_ref).max() < 2e-6 * max(1.0, np.abs(en_ref).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_etrs_scf_steps_match_oracle(pb, oracle_mod, sysd, precision):
    """Two ETRS steps with the LDA self-consistency loop and a changing vector
    potential (etrs.hpp:22-82)."""
    o = make_oracle(oracle_mod, sysd)
    h = make_product(pb, sysd, precision)
    occ = np.array([2.0, 2.0, 2.0, 2.0])
    vion = sysd["V"]
    psi_ref = sysd["psi"].copy()
    rho_ref = o.density(psi_ref, occ)
    o.ks_potential(rho_ref, vion, 2)
    dt_ = torch.complex128 if precision == "fp64" else torch.complex64
    psi = _dev(sysd["psi"], dt_)
    rho = _dev(rho_ref, torch.float64)
    vion_d = _dev(vion, torch.float64)
    h.ks_potential(rho, vion_d, 2, energies=False)
    amps = [0.0, 0.02, -0.01]
    for n in range(2):
        k1 = o.cart_to_cov(np.array([amps[n], 0.0, 0.0]))
        k2 = o.cart_to_cov(np.array([amps[n + 1], 0.0, 0.0]))
        psi_ref, rho_ref, it_ref, en_ref = o.etrs_scf_step(psi_ref, rho_ref, 0.05, k1, k2, occ, vion, 2)
        it, en = h.etrs_scf_step_(psi, rho, 0.05, k1, k2, occ, vion_d, 2)
        en = np.array([en["external"], en["hartree"], en["xc"], en["nvxc"]])
        if precision == "fp64":
            assert it == it_ref
            assert np.abs(en - en_ref).max() < 1e-10 * np.abs(en_ref).max()
        else:
            assert abs(it - it_ref) <= 1
            assert np.abs(en - en_ref).max() < 1e-5 * np.abs(en_ref).max()
    if precision == "fp64":
        assert rel_max(psi.cpu().numpy(), psi_ref) < 1e-10
        assert rel_max(rho.cpu().numpy(), rho_ref) < 1e-10
    else:
        assert rel_norm(psi.cpu().numpy(), psi_ref) < 5e-5
        assert rel_norm(rho.cpu().numpy(), rho_ref) < 5e-5


def test_etrs_scf_noninteracting_equals_etrs(pb, oracle_mod, sysd):
    """Theory NONE: the SCF loop stops at its second pass and the step is the plain
    ETRS step of inqb_etrs_step."""
    h = make_product(pb, sysd, "fp64")
    occ = np.array([2.0, 2.0, 2.0, 2.0])
    k1 = h.cart_to_cov(np.array([0.01, 0.0, 0.0]))
    k2 = h.cart_to_cov(np.array([0.03, 0.0, 0.0]))
    a = _dev(sysd["psi"])
    b = a.clone()
    vion = _dev(sysd["V"], torch.float64)
    rho = h.density(a, occ)
    h.ks_potential(rho, vion, 0, energies=False)
    it, _ = h.etrs_scf_step_(a, rho, 0.05, k1, k2, occ, vion, 0)
    h.set_vector_potential_cov(k1)
    h.etrs_step_(b, 0.05, k1, k2)
    assert it == 2
    assert rel_max(a.cpu().numpy(), b.cpu().numpy()) < 1e-12


def test_etrs_scf_sharded_two_blocks_equals_whole(pb, oracle_mod, sysd):
    """Orbital sharding of the SCF step: two contexts, each with half of the orbitals,
    run the step concurrently in two host threads; the density-reduction hook sums
    their densities (the exchange step).  The union equals the one-context step."""
    import threading

    occ = np.array([2.0, 2.0, 2.0, 2.0])
    k1 = np.zeros(3)
    k2 = np.array([0.01, 0.0, 0.0])
    vion = _dev(sysd["V"], torch.float64)
    whole = make_product(pb, sysd, "fp64")
    x = _dev(sysd["psi"])
    rho = whole.density(x, occ)
    whole.ks_potential(rho, vion, 2, energies=False)
    it_ref, en_ref = whole.etrs_scf_step_(x, rho, 0.05, k1, k2, occ, vion, 2)

    halves = [make_product(pb, sysd, "fp64") for _ in range(2)]
    xs = [_dev(sysd["psi"][:, :2]), _dev(sysd["psi"][:, 2:])]
    rhos = [h.density(xx, occ[:2]) for h, xx in zip(halves, xs)]
    total = rhos[0] + rhos[1]
    for h, r in zip(halves, rhos):
        r.copy_(total)
        h.ks_potential(r, vion, 2, energies=False)
    torch.cuda.synchronize()
    bar = threading.Barrier(2, timeout=60)
    calls = [0, 0]

    def make_reducer(i):
        def reduce_(r):
            calls[i] += 1
            torch.cuda.synchronize()
            bar.wait()
            if i == 0:
                s = rhos[0] + rhos[1]
                torch.cuda.synchronize()
                reduce_.shared[0] = s
            bar.wait()
            r.copy_(reduce_.shared[0])
            torch.cuda.synchronize()
            bar.wait()
            return r
        return reduce_

    shared = [None]
    out = [None, None]
    for i, h in enumerate(halves):
        red = make_reducer(i)
        red.shared = shared
        h.set_density_reducer(red)

    def run(i):
        out[i] = halves[i].etrs_scf_step_(xs[i], rhos[i], 0.05, k1, k2, occ[:2], vion, 2)

    ts = [threading.Thread(target=run, args=(i,)) for i in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(120)
    assert out[0] is not None and out[1] is not None
    assert out[0][0] == out[1][0] == it_ref and calls == [it_ref + 1, it_ref + 1]
    both = torch.cat(xs, 1).cpu().numpy()
    assert rel_max(both, x.cpu().numpy()) < 1e-12
    assert rel_max(rhos[0].cpu().numpy(), rho.cpu().numpy()) < 1e-12
    for k in ("external", "hartree", "xc", "nvxc"):
        assert abs(out[0][1][k] - en_ref[k]) < 1e-11 * max(1.0, abs(en_ref[k]))
