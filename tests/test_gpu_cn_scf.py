"""inqb_crank_nicolson_scf_step against the oracle: Crank-Nicolson with its
self-consistency loop and Broyden density mixing (src/real_time/crank_nicolson.hpp:41-114,
src/mixers/broyden.hpp:26-160), through the C ABI.

  * one LDA step with a changing vector potential, FP64 (iterations equal, 1e-9) and
    mixed precision (within one iteration, 1e-4);
  * the iteration cap: two iterations, so the mixer's first call (plain mixing) and
    its second (one ring slot, the small solve) both run, FP64 against the oracle;
  * without interaction the step lands on the converged linear solve of
    inqb_crank_nicolson_step;
  * orbital sharding: two contexts with half of the orbitals each, in two host
    threads, exchange the density through the reduce hook and equal one context.
"""
import threading

import numpy as np
import pytest
import torch

from helpers import make_oracle, make_product, rel_max, rel_norm, small_system

pytestmark = pytest.mark.gpu

OCC = np.array([2.0, 2.0, 2.0, 2.0])


def _dev(a, dtype=torch.complex128):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.fixture(scope="module")
def sysd(pb):
    return small_system(pb, n=32, M=4, seed=61)


def _kA(o):
    return o.cart_to_cov(np.array([0.01, 0.0, 0.005])), o.cart_to_cov(np.array([0.02, 0.0, 0.005]))


def _energies(en):
    return np.array([en["external"], en["hartree"], en["xc"], en["nvxc"]])


def _run_both(pb, oracle_mod, sysd, precision, theory=2, max_iter=300):
    o = make_oracle(oracle_mod, sysd)
    h = make_product(pb, sysd, precision)
    k1, k2 = _kA(o)
    vion = sysd["V"]
    rho_ref = o.density(sysd["psi"], OCC)
    o.ks_potential(rho_ref, vion, theory)
    psi_ref, rho_ref, it_ref, en_ref, _ = o.crank_nicolson_scf_step(sysd["psi"], rho_ref, 0.05, k1, k2, OCC, vion,
                                                                    theory, max_iter=max_iter)
    psi = _dev(sysd["psi"], torch.complex128 if precision == "fp64" else torch.complex64)
    rho = h.density(psi, OCC)
    vion_d = _dev(vion, torch.float64)
    h.ks_potential(rho, vion_d, theory, energies=False)
    it, res, en = h.crank_nicolson_scf_step_(psi, rho, 0.05, k1, k2, OCC, vion_d, theory, max_iter=max_iter)
    assert np.isfinite(res)
    return (psi.cpu().numpy(), rho.cpu().numpy(), it, _energies(en)), (psi_ref, rho_ref, it_ref, en_ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cn_scf_lda_step_matches_oracle(pb, oracle_mod, sysd, precision):
    (psi, rho, it, en), (psi_ref, rho_ref, it_ref, en_ref) = _run_both(pb, oracle_mod, sysd, precision)
    assert 2 < it_ref < 300
    if precision == "fp64":
        assert it == it_ref
        assert rel_max(psi, psi_ref) < 1e-9
        assert rel_max(rho, rho_ref) < 1e-9
        assert np.abs(en - en_ref).max() < 1e-9 * np.abs(en_ref).max()
    else:
        assert abs(it - it_ref) <= 1
        assert rel_norm(psi, psi_ref) < 1e-4
        assert rel_norm(rho, rho_ref) < 1e-4
        assert np.abs(en - en_ref).max() < 1e-4 * np.abs(en_ref).max()


def test_cn_scf_iteration_cap_matches_oracle(pb, oracle_mod, sysd):
    (psi, rho, it, en), (psi_ref, rho_ref, it_ref, en_ref) = _run_both(pb, oracle_mod, sysd, "fp64", max_iter=2)
    assert it == it_ref == 2
    assert rel_max(psi, psi_ref) < 1e-10
    assert rel_max(rho, rho_ref) < 1e-10
    assert np.abs(en - en_ref).max() < 1e-10 * np.abs(en_ref).max()


def test_cn_scf_noninteracting_lands_on_the_converged_solve(pb, sysd):
    h = make_product(pb, sysd, "fp64")
    k1 = h.cart_to_cov(np.array([0.01, 0.0, 0.005]))
    k2 = h.cart_to_cov(np.array([0.02, 0.0, 0.005]))
    a = _dev(sysd["psi"])
    b = a.clone()
    vion = _dev(sysd["V"], torch.float64)
    rho = h.density(a, OCC)
    h.ks_potential(rho, vion, 0, energies=False)
    it, _, en = h.crank_nicolson_scf_step_(a, rho, 0.05, k1, k2, OCC, vion, 0)
    assert 2 <= it < 300 and en["hartree"] == en["xc"] == 0.0
    h.set_scalar_potential(sysd["V"])
    h.set_vector_potential_cov(k1)
    _, res = h.crank_nicolson_step_(b, 0.05, k1, k2, 300, 1e-14)
    assert res < 1e-14
    assert rel_max(a.cpu().numpy(), b.cpu().numpy()) < 1e-5  # stopped on the density


def test_cn_scf_sharded_two_blocks_equals_whole(pb, sysd):
    k1 = np.zeros(3)
    k2 = np.array([0.01, 0.0, 0.0])
    vion = _dev(sysd["V"], torch.float64)
    whole = make_product(pb, sysd, "fp64")
    x = _dev(sysd["psi"])
    rho = whole.density(x, OCC)
    whole.ks_potential(rho, vion, 2, energies=False)
    it_ref, _, en_ref = whole.crank_nicolson_scf_step_(x, rho, 0.05, k1, k2, OCC, vion, 2)

    halves = [make_product(pb, sysd, "fp64") for _ in range(2)]
    xs = [_dev(sysd["psi"][:, :2]), _dev(sysd["psi"][:, 2:])]
    rhos = [h.density(xx, OCC[:2]) for h, xx in zip(halves, xs)]
    total = rhos[0] + rhos[1]
    for h, r in zip(halves, rhos):
        r.copy_(total)
        h.ks_potential(r, vion, 2, energies=False)
    torch.cuda.synchronize()
    bar = threading.Barrier(2, timeout=60)
    calls = [0, 0]
    shared = [None]

    def make_reducer(i):
        def reduce_(r):
            calls[i] += 1
            torch.cuda.synchronize()
            bar.wait()
            if i == 0:
                s = rhos_seen[0] + rhos_seen[1]
                torch.cuda.synchronize()
                shared[0] = s
            bar.wait()
            r.copy_(shared[0])
            torch.cuda.synchronize()
            bar.wait()
            return r
        return reduce_

    # the library hands the reducer the buffer it just filled: the step's own density
    # output on the last call, its scratch "new density" before; both threads register
    # theirs here before the sum
    rhos_seen = [None, None]

    def make_wrapped(i):
        inner = make_reducer(i)

        def wrapped(r):
            rhos_seen[i] = r
            return inner(r)
        return wrapped

    for i, h in enumerate(halves):
        h.set_density_reducer(make_wrapped(i))
    out = [None, None]

    def run(i):
        out[i] = halves[i].crank_nicolson_scf_step_(xs[i], rhos[i], 0.05, k1, k2, OCC[:2], vion, 2,
                                                    num_electrons=float(OCC.sum()))

    ts = [threading.Thread(target=run, args=(i,)) for i in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(300)
    assert out[0] is not None and out[1] is not None
    assert out[0][0] == out[1][0] == it_ref and calls == [it_ref + 1, it_ref + 1]
    # the halves' densities round differently (two partial sums), and the mixer's small
    # solve (condition number up to about 1e6) can amplify that: 1e-10, not 1e-12
    both = torch.cat(xs, 1).cpu().numpy()
    assert rel_max(both, x.cpu().numpy()) < 1e-10
    assert rel_max(rhos[0].cpu().numpy(), rho.cpu().numpy()) < 1e-10
    for k in ("external", "hartree", "xc", "nvxc"):
        assert abs(out[0][2][k] - en_ref[k]) < 1e-9 * max(1.0, abs(en_ref[k]))
