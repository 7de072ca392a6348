"""Adjoint of the ETRS propagation (cfg2 system: a = 10.26 bohr, 8 atoms, 32^3 grid,
16 occupied orbitals, dt = 0.05): gradients of the final x-dipole with respect to
the piecewise-constant field amplitudes and the local potential, checked against
central finite differences (h = 1e-4) and between the mixed and FP64 paths."""
import numpy as np
import pytest
import torch

from helpers import make_product, small_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cfg2(pb):
    s = small_system(pb, n=32, M=16, seed=2)
    rng = np.random.default_rng(3)
    s["amps"] = rng.normal(0.0, 0.01, 200)
    s["occ"] = np.full(16, 2.0)
    return s


def _prop(pb, s, precision, every):
    """cfg2 propagation; the Fourier sphere mask keeps Taylor-4 stable: on this 32^3 grid
    1/2|G|^2 reaches 144 Ha at the box corners and dt/2 * 144 = 3.6 > 2 sqrt(2)."""
    from pinq_b200.adjoint import DipolePropagation

    h = make_product(pb, s, precision)
    h.set_fourier_sphere_mask(True)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    psi0 = torch.as_tensor(s["psi"]).to("cuda", dt)
    return DipolePropagation(h, psi0, s["occ"], 0.05, every)


def _fd(prop, amps, V, which, idx, h=1e-4):
    out = []
    for k in idx:
        vals = []
        for sgn in (+1, -1):
            a = amps.copy()
            v = V.copy()
            if which == "A":
                a[k] += sgn * h
            else:
                v[k] += sgn * h
            prop.h.set_scalar_potential(v)
            vals.append(prop.forward(a, keep=False))
        out.append((vals[0] - vals[1]) / (2 * h))
    prop.h.set_scalar_potential(V)
    return np.array(out)


@pytest.mark.parametrize("nsteps,every", [(40, 10), (200, 20)])
def test_adjoint_fp64_matches_finite_differences(pb, cfg2, nsteps, every):
    from pinq_b200.adjoint import etrs_dipole

    prop = _prop(pb, cfg2, "fp64", every)
    amps = cfg2["amps"][:nsteps].copy()
    V = cfg2["V"].copy()
    a_t = torch.tensor(amps, requires_grad=True)
    V_t = torch.tensor(V, requires_grad=True)
    d = etrs_dipole(a_t, V_t, prop)
    d.backward()
    gA = a_t.grad.numpy()
    gV = V_t.grad.numpy()
    ia = [0, nsteps // 2, nsteps - 1]
    fa = _fd(prop, amps, V, "A", ia)
    scaleA = np.abs(gA).max()
    assert np.abs(gA[ia] - fa).max() <= 1e-5 * scaleA, (gA[ia], fa)
    iv = [int(np.argmax(np.abs(gV))), 12345, 32767]
    fv = _fd(prop, amps, V, "V", iv)
    scaleV = np.abs(gV).max()
    assert np.abs(gV[iv] - fv).max() <= 1e-5 * scaleV, (gV[iv], fv)


def test_adjoint_mixed_matches_fp64(pb, cfg2):
    from pinq_b200.adjoint import etrs_dipole

    amps = cfg2["amps"][:40].copy()
    V = cfg2["V"].copy()
    res = {}
    for precision in ("fp64", "mixed"):
        prop = _prop(pb, cfg2, precision, 10)
        a_t = torch.tensor(amps, requires_grad=True)
        V_t = torch.tensor(V, requires_grad=True)
        d = etrs_dipole(a_t, V_t, prop)
        d.backward()
        res[precision] = (float(d), a_t.grad.numpy().copy(), V_t.grad.numpy().copy())
    d64, gA64, gV64 = res["fp64"]
    d32, gA32, gV32 = res["mixed"]
    assert abs(d32 - d64) <= 1e-5 * max(1.0, abs(d64))
    assert np.linalg.norm(gA32 - gA64) <= 1e-4 * np.linalg.norm(gA64)
    assert np.linalg.norm(gV32 - gV64) <= 1e-4 * np.linalg.norm(gV64)


@pytest.mark.parametrize("precision,tol,mask", [("fp64", 1e-8, False), ("fp64", 1e-8, True), ("mixed", 2e-5, True)])
def test_dH_dA_matches_oracle_difference(pb, oracle_mod, precision, tol, mask):
    """<u| dH/dA_d |w> from the kinetic + nonlocal derivative kernels against a central
    difference of the oracle's H (h = 1e-5) at k + A != 0, for d = x, y, z."""
    from helpers import make_oracle

    s = small_system(pb, n=32, M=4, seed=7)
    rng = np.random.default_rng(8)
    u = s["psi"]
    w = np.roll(s["psi"], 1, axis=1) + 0.3j * s["psi"]
    A0 = np.array([0.04, -0.03, 0.02])
    o = oracle_mod.System(s["lattice"], s["nr"])
    h = make_product(pb, s, precision, o.cart_to_cov(A0))
    h.set_fourier_sphere_mask(mask)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    gA = torch.zeros(3, dtype=torch.float64, device="cuda")
    h.accum_vector_potential_gradient_(gA, torch.as_tensor(u).to("cuda", dt), torch.as_tensor(w).to("cuda", dt), 1.0)
    gA = gA.cpu().numpy()
    ref = np.zeros(3)
    eps = 1e-5
    for d in range(3):
        vals = []
        for sgn in (+1, -1):
            A = A0.copy()
            A[d] += sgn * eps
            oo = make_oracle(oracle_mod, s, o.cart_to_cov(A))
            oo.set_fourier_mask(mask)
            vals.append(np.vdot(u, oo.apply_h(w)))
        ref[d] = ((vals[0] - vals[1]) / (2 * eps)).real
    assert np.abs(gA - ref).max() <= tol * np.abs(ref).max(), (gA, ref)
    del rng


def test_stored_powers_mode_matches_checkpointed(pb, cfg2):
    """Keeping every step's Taylor powers in the forward pass (no recompute) gives
    the checkpointed backward's gradients: the same kernels on the same powers."""
    from pinq_b200.adjoint import DipolePropagation

    h = make_product(pb, cfg2, "fp64")
    h.set_fourier_sphere_mask(True)
    psi0 = torch.as_tensor(cfg2["psi"]).to("cuda", torch.complex128)
    amps = cfg2["amps"][:30]
    out = []
    for store in (False, True):
        prop = DipolePropagation(h, psi0, cfg2["occ"], 0.05, 10, store_powers=store)
        prop.forward(amps, keep=True)
        gA, gV = prop.backward()
        out.append((gA.cpu().numpy(), gV.cpu().numpy()))
    assert np.abs(out[0][0] - out[1][0]).max() <= 1e-10 * np.abs(out[0][0]).max()
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-10 * np.abs(out[0][1]).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_overlapped_recompute_equals_sequential(pb, cfg2, precision):
    """The checkpointed backward with each segment's recompute on a second stream and a
    cloned context (the default) gives the sequential backward's gradients: the same
    kernels on the same inputs, ordered by events (the gradient sums use atomics, so
    agreement is to rounding: 1e-12 in FP64, 1e-6 in the mixed precision)."""
    from pinq_b200.adjoint import DipolePropagation

    h = make_product(pb, cfg2, precision)
    h.set_fourier_sphere_mask(True)
    dt = torch.complex128 if precision == "fp64" else torch.complex64
    psi0 = torch.as_tensor(cfg2["psi"]).to("cuda", dt)
    amps = cfg2["amps"][:35]
    out = []
    # overlapped; sequential; overlap asked for but the second powers buffer does not
    # fit (the fallback of large cells: one buffer, the forward's, reused)
    for overlap, room in ((True, True), (False, True), (True, False)):
        prop = DipolePropagation(h, psi0, cfg2["occ"], 0.05, 10)
        prop.overlap = overlap
        if not room:
            prop._try_powers_buffer = lambda nsteps: None
        prop.forward(amps, keep=True)
        gA, gV = prop.backward()
        torch.cuda.synchronize()
        out.append((gA.cpu().numpy(), gV.cpu().numpy()))
    tol = 1e-12 if precision == "fp64" else 1e-6
    for k in range(2):
        assert np.abs(out[0][k] - out[1][k]).max() <= tol * np.abs(out[1][k]).max()
        assert np.abs(out[2][k] - out[1][k]).max() <= tol * np.abs(out[1][k]).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_terms_equals_step_powers(pb, cfg2, precision):
    """inqb_etrs_step_terms, which keeps nothing, steps the orbitals bit for bit as
    inqb_etrs_step_powers does (the checkpointed forward relies on it: the backward
    recomputes its segments with the powers step), for a strided block too."""
    prop = _prop(pb, cfg2, precision, 20)
    h = prop.h
    x = prop.psi0.clone()
    wide = torch.zeros((h.N, x.shape[1] + 3), dtype=x.dtype, device="cuda")
    y = wide[:, :x.shape[1]]
    y.copy_(x)
    buf = h.powers_buffer(1, x.shape[1])
    for n in range(3):
        a, b = prop._kA(cfg2["amps"][n]), prop._kA(cfg2["amps"][n + 1])
        h.etrs_step_powers_(x, 0.05, a, b, buf[0])
        h.etrs_step_terms_(y, 0.05, a, b)
        assert torch.equal(x, y)
