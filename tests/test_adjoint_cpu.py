"""CPU check of the adjoint orchestration (pinq_b200.adjoint) with a dense stand-in
Hamiltonian H(a) = K + a D + diag(V) that exposes the library's method names:
the discrete-adjoint gradients must match central finite differences."""
import numpy as np
import torch

from pinq_b200.adjoint import DipolePropagation, etrs_dipole


class DenseHam:
    def __init__(self, N, seed=0):
        rng = np.random.default_rng(seed)
        A = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        self.K = torch.tensor((A + A.conj().T) / 4)
        B = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        self.D = torch.tensor((B + B.conj().T) / 8)
        self.N = N
        self.V = torch.zeros(N, dtype=torch.float64)
        self.a = 0.0
        self.x = torch.linspace(-1.0, 1.0, N, dtype=torch.float64)
        self.volume_element = 0.5

    def H(self):
        return self.K + self.a * self.D + torch.diag(self.V.to(torch.complex128))

    def cart_to_cov(self, v):
        return np.asarray(v, float)

    def set_vector_potential_cov(self, kA):
        self.a = float(kA[0])

    def set_scalar_potential(self, V):
        self.V = torch.as_tensor(np.asarray(V, float))

    def apply(self, psi):
        return self.H() @ psi

    def axpby_(self, a, x, b, y):
        y.mul_(b).add_(a * x)
        return y

    def position_scale(self, psi, occ, direction, scale):
        return scale * self.x[:, None] * torch.as_tensor(occ)[None, :] * psi

    def accum_potential_gradient_(self, gV, u, w, c):
        gV += (complex(c) * (u.conj() * w).sum(1)).real

    def accum_vector_potential_gradient_(self, gA, u, w, c):
        gA[0] += (complex(c) * (u.conj() * (self.D @ w)).sum()).real

    def _T(self, a, dt, psi):
        self.a = a
        f = 0.5j * dt
        out, term = psi.clone(), psi.clone()
        for k in range(1, 5):
            term = (f / k) * (self.H() @ term)
            out = out + term
        return out

    def etrs_step_(self, psi, dt, kA1, kA2):
        psi.copy_(self._T(float(kA2[0]), dt, self._T(float(kA1[0]), dt, psi)))
        return psi

    def powers_buffer(self, nsteps, M):
        return torch.empty((nsteps, 8, self.N, M), dtype=torch.complex128)

    @staticmethod
    def _c(dt):
        c = [1.0 + 0j]
        for k in range(1, 5):
            c.append(c[-1] * 0.5j * dt / k)
        return c

    def _half(self, a, dt, x, P):
        # the library's half step with powers: P[k] = H^k x, result sum_k c_k H^k x
        self.a = a
        c = self._c(dt)
        P[0].copy_(x)
        for k in range(1, 4):
            P[k].copy_(self.H() @ P[k - 1])
        h4 = self.H() @ P[3]
        return sum(c[k] * P[k] for k in range(4)) + c[4] * h4

    def etrs_step_powers_(self, psi, dt, kA1, kA2, powers):
        phi = self._half(float(kA1[0]), dt, psi, powers[0:4])
        psi.copy_(self._half(float(kA2[0]), dt, phi, powers[4:8]))
        return psi

    def etrs_step_terms_(self, psi, dt, kA1, kA2):
        # the same sums as etrs_step_powers_, the powers dropped
        return self.etrs_step_powers_(psi, dt, kA1, kA2, self.powers_buffer(1, psi.shape[1])[0])

    def _back(self, a, dt, lam, Phi, gV, gA):
        self.a = a
        cc = [np.conj(x) for x in self._c(dt)]
        L = [lam.clone()]
        for _ in range(4):
            L.append(self.H() @ L[-1])
        for i in range(4):
            xi = sum(cc[i + j + 1] * L[j] for j in range(4 - i))
            gV += (2.0 * (xi.conj() * Phi[i]).sum(1)).real
            gA[0] += (2.0 * (xi.conj() * (self.D @ Phi[i])).sum()).real
        return sum(cc[k] * L[k] for k in range(5))

    def etrs_adjoint_step_(self, lam, dt, kA1, kA2, powers, gV, gA_t, gA_tdt):
        lam.copy_(self._back(float(kA2[0]), dt, lam, powers[4:8], gV, gA_tdt))
        lam.copy_(self._back(float(kA1[0]), dt, lam, powers[0:4], gV, gA_t))
        return lam

    def density(self, psi, occ):
        return ((psi.abs() ** 2) * torch.as_tensor(occ)[None, :]).sum(1)

    def dipole(self, rho):
        return np.array([float(self.volume_element * (self.x * rho).sum()), 0.0, 0.0])


def test_adjoint_orchestration_matches_finite_differences():
    N, M, nsteps = 24, 3, 9
    ham = DenseHam(N)
    rng = np.random.default_rng(1)
    psi0 = torch.tensor(rng.standard_normal((N, M)) + 1j * rng.standard_normal((N, M)))
    prop = DipolePropagation(ham, psi0, [2.0, 2.0, 1.0], dt=0.3, every=4)
    amps = rng.normal(0.0, 0.3, nsteps)
    V = rng.normal(0.0, 0.5, N)
    a_t = torch.tensor(amps, requires_grad=True)
    V_t = torch.tensor(V, requires_grad=True)
    d = etrs_dipole(a_t, V_t, prop)
    d.backward()

    def f(a, v):
        ham.set_scalar_potential(v)
        return prop.forward(a, keep=False)

    h = 1e-6
    for k in range(nsteps):
        e = np.zeros(nsteps)
        e[k] = h
        fd = (f(amps + e, V) - f(amps - e, V)) / (2 * h)
        assert abs(fd - float(a_t.grad[k])) < 1e-7 * max(1.0, abs(fd))
    for p in [0, 5, 17, 23]:
        e = np.zeros(N)
        e[p] = h
        fd = (f(amps, V + e) - f(amps, V - e)) / (2 * h)
        assert abs(fd - float(V_t.grad[p])) < 1e-7 * max(1.0, abs(fd))


def test_recompute_overlap_follows_the_block_size():
    """The checkpointed backward recomputes beside its walk only for small blocks
    (grid points x orbitals up to OVERLAP_MAX_ELEMENTS); True / False force either form."""
    limit = DipolePropagation.OVERLAP_MAX_ELEMENTS
    for N, M, expect in ((32 ** 3, 16, True), (64 ** 3, 16, True), (64 ** 3, 128, False), (144 ** 3, 16, False)):
        ham = DenseHam(4)
        ham.N = N
        prop = DipolePropagation(ham, torch.zeros((4, M), dtype=torch.complex128), np.ones(M), 0.05, 10)
        assert prop._overlapped() is expect and (N * M <= limit) is expect
        for forced in (True, False):
            prop.overlap = forced
            assert prop._overlapped() is forced
