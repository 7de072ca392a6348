"""Real-time propagation of a dipole observable and its hand-written adjoint.

Forward: ETRS steps (src/real_time/etrs.hpp:22-82) under a uniform vector
potential along x given as piecewise-constant amplitudes a_n (A(t) = a_n for
t in [n dt, (n+1) dt), the last amplitude held), for a density-independent H:

    psi_{n+1} = T(f H(a_{n+1})) T(f H(a_n)) psi_n,   T(fH) = sum_{k<=4} (fH)^k / k!,  f = i dt/2

Observable: the electronic dipole d_x = dV sum_p x_p rho_p with rho = sum_m occ_m |psi_m|^2
(src/observables/dipole.hpp:23-40).

Backward (discrete adjoint, exact for the discretised propagator):

    lambda_N = dV occ x psi_N,   lambda_n = T(f* H(a_n)) T(f* H(a_{n+1})) lambda_{n+1}
    dd/dtheta = 2 Re sum_n <lambda_{n+1}| dU_n/dtheta |psi_n>

with, per half step, <lam| dT |phi> = sum_i <Xi_i| dH |Phi_i>, Phi_i = H^i phi and
Xi_i = sum_j conj(c_{i+j+1}) H^j lam.  dH/dV(p) is pointwise; dH/dA_x is the
kinetic (G + A)_x plus the nonlocal position commutator.  The forward orbitals are
checkpointed every `every` steps and recomputed segment by segment.

Everything runs in libinqb200's kernels; torch holds device memory and supplies
the autograd interface.
"""
from __future__ import annotations

import numpy as np
import torch


def _coeffs(dt: float, order: int = 4):
    f = 0.5j * dt
    c = [1.0 + 0j]
    for k in range(1, order + 1):
        c.append(c[-1] * f / k)
    return c


class DipolePropagation:
    """ETRS propagation of one orbital block with checkpoints, forward and adjoint."""

    def __init__(self, ham, psi0: torch.Tensor, occ, dt: float, every: int = 20, direction: int = 0):
        self.h = ham
        self.psi0 = psi0
        self.M = psi0.shape[1]
        self.occ = torch.as_tensor(np.asarray(occ, float), dtype=torch.float64, device=psi0.device)
        self.dt = float(dt)
        self.every = int(every)
        self.direction = int(direction)
        self.c = _coeffs(self.dt)

    # -- helpers
    def _kA(self, a: float):
        v = np.zeros(3)
        v[self.direction] = a
        return self.h.cart_to_cov(v)

    @staticmethod
    def _amp(amps, n):
        return float(amps[min(n, len(amps) - 1)])

    def _set_A(self, a):
        self.h.set_vector_potential_cov(self._kA(a))

    # -- forward
    def forward(self, amplitudes, keep=True) -> float:
        amps = np.asarray(amplitudes, float)
        psi = self.psi0.clone()
        cps = {}
        for n in range(len(amps)):
            if keep and n % self.every == 0:
                cps[n] = psi.clone()
            self.h.etrs_step_(psi, self.dt, self._kA(self._amp(amps, n)), self._kA(self._amp(amps, n + 1)))
        rho = self.h.density(psi, self.occ)
        d = float(self.h.dipole(rho)[self.direction])
        if keep:
            self.amps = amps
            self.checkpoints = cps
            self.psi_final = psi
        return d

    def _powers(self, a, phi):
        """[H^0 phi .. H^4 phi] at amplitude a."""
        self._set_A(a)
        out = [phi]
        for _ in range(4):
            out.append(self.h.apply(out[-1]))
        return out

    def _combine(self, coefs, blocks):
        """sum_k coefs[k] blocks[k] with the library's axpby."""
        acc = torch.zeros_like(blocks[0])
        for c, b in zip(coefs, blocks):
            if c != 0:
                self.h.axpby_(c, b, 1.0, acc)
        return acc

    def _half_back(self, a, lam, Phi, gV, gA_row):
        L = self._powers(a, lam)  # Lambda_j = H^j lam, k + A set to a
        cc = [np.conj(x) for x in self.c]
        for i in range(4):
            xi = self._combine([cc[i + j + 1] for j in range(4 - i)], L[: 4 - i])
            self.h.accum_potential_gradient_(gV, xi, Phi[i], 2.0)
            self.h.accum_vector_potential_gradient_(gA_row, xi, Phi[i], 2.0)
        return self._combine(cc, L)

    # -- backward
    def backward(self):
        """(d d/d amplitudes [len(amps)], d d/d V [N]) as FP64 device tensors."""
        h = self.h
        amps = self.amps
        nsteps = len(amps)
        dev = self.psi0.device
        gV = torch.zeros(h.N, dtype=torch.float64, device=dev)
        gA = torch.zeros((nsteps, 3), dtype=torch.float64, device=dev)
        lam = h.position_scale(self.psi_final, self.occ, self.direction, h.volume_element)
        for s0 in reversed(range(0, nsteps, self.every)):
            s1 = min(s0 + self.every, nsteps)
            psi = self.checkpoints[s0].clone()
            store = []
            for n in range(s0, s1):
                P1 = self._powers(self._amp(amps, n), psi)
                phi = self._combine(self.c, P1)
                P2 = self._powers(self._amp(amps, n + 1), phi)
                psi = self._combine(self.c, P2)
                store.append((P1[:4], P2[:4]))
            for n in reversed(range(s0, s1)):
                P1, P2 = store[n - s0]
                n2 = min(n + 1, nsteps - 1)
                lam = self._half_back(self._amp(amps, n + 1), lam, P2, gV, gA[n2])
                lam = self._half_back(self._amp(amps, n), lam, P1, gV, gA[n])
            del store
        return gA[:, self.direction].clone(), gV


class _ETRSDipoleFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, amplitudes, V, prop):
        prop.h.set_scalar_potential(V.detach().cpu().numpy())
        d = prop.forward(amplitudes.detach().cpu().numpy(), keep=True)
        ctx.prop = prop
        return torch.tensor(d, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        gA, gV = ctx.prop.backward()
        g = float(grad_out)
        return (g * gA).cpu(), (g * gV).cpu(), None


def etrs_dipole(amplitudes: torch.Tensor, V: torch.Tensor, prop: DipolePropagation) -> torch.Tensor:
    """Final-time dipole as a differentiable function of the field amplitudes and V."""
    return _ETRSDipoleFunction.apply(amplitudes, V, prop)
