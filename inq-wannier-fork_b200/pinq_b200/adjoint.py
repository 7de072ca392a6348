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

The steps run in libinqb200 (inqb_etrs_step, inqb_etrs_step_powers,
inqb_etrs_adjoint_step); torch holds device memory and supplies the autograd
interface.  With more than one checkpoint segment and a block small enough that one
step's kernels leave the GPU partly idle, the recompute of the segment before runs on
a second CUDA stream, with a second context (inqb_ctx_clone), beside the backward walk
of the current one: the recompute's launches fill the gaps of the backward's.  Larger
blocks recompute and walk the segments one after the other.
"""
from __future__ import annotations

import numpy as np
import torch


class DipolePropagation:
    """ETRS propagation of one orbital block with checkpoints, forward and adjoint."""

    def __init__(self, ham, psi0: torch.Tensor, occ, dt: float, every: int = 20, direction: int = 0,
                 store_powers: bool = False):
        """every: checkpoint interval of the recomputing backward.  store_powers:
        keep the Taylor powers of every step during the forward pass instead (8
        orbital blocks and their Fourier coefficients per step; no recompute in the
        backward)."""
        self.h = ham
        self.psi0 = psi0
        self.M = psi0.shape[1]
        self.occ = torch.as_tensor(np.asarray(occ, float), dtype=torch.float64, device=psi0.device)
        self.dt = float(dt)
        self.every = int(every)
        self.direction = int(direction)
        self.store_powers = bool(store_powers)
        self.powers = None
        # recompute the previous segment on a second stream: True, False, or None to
        # decide by the block size (overlap while one step's kernels leave the GPU idle)
        self.overlap = None
        self._tail = None  # (first step, powers) of the last segment, kept by the forward
        self._h2 = None
        self._h2_version = None

    # -- helpers
    def _kA(self, a: float):
        v = np.zeros(3)
        v[self.direction] = a
        return self.h.cart_to_cov(v)

    @staticmethod
    def _amp(amps, n):
        return float(amps[min(n, len(amps) - 1)])

    # -- forward
    def forward(self, amplitudes, keep=True) -> float:
        amps = np.asarray(amplitudes, float)
        psi = self.psi0.clone()
        cps = {}
        self.powers = None
        self._tail = None
        if keep and self.store_powers:
            powers = self.h.powers_buffer(len(amps), self.M)
            for n in range(len(amps)):
                self.h.etrs_step_powers_(psi, self.dt, self._kA(self._amp(amps, n)),
                                         self._kA(self._amp(amps, n + 1)), powers[n])
            self.powers = powers
        elif keep:
            # the same term-by-term step the backward recomputes each segment with, so
            # that the recomputed trajectory is this one exactly (keeping no powers);
            # the last segment's powers are kept, since the backward walks it first
            nsteps = len(amps)
            last0 = ((nsteps - 1) // self.every) * self.every
            tail = self.h.powers_buffer(min(self.every, nsteps), self.M)
            for n in range(nsteps):
                if n % self.every == 0:
                    cps[n] = psi.clone()
                a, b = self._kA(self._amp(amps, n)), self._kA(self._amp(amps, n + 1))
                if n >= last0:
                    self.h.etrs_step_powers_(psi, self.dt, a, b, tail[n - last0])
                else:
                    self.h.etrs_step_terms_(psi, self.dt, a, b)
            self._tail = (last0, tail)
        else:
            for n in range(len(amps)):
                self.h.etrs_step_(psi, self.dt, self._kA(self._amp(amps, n)), self._kA(self._amp(amps, n + 1)))
        rho = self.h.density(psi, self.occ)
        d = float(self.h.dipole(rho)[self.direction])
        if keep:
            self.amps = amps
            self.checkpoints = cps
            self.psi_final = psi
        return d

    # -- backward
    def backward(self):
        """(d d/d amplitudes [len(amps)], d d/d V [N]) as FP64 device tensors.

        Each checkpoint segment is recomputed with inqb_etrs_step_powers, which keeps
        the Taylor powers of every step, then walked backwards with
        inqb_etrs_adjoint_step; both run entirely in the library."""
        h = self.h
        amps = self.amps
        nsteps = len(amps)
        dev = self.psi0.device
        gV = torch.zeros(h.N, dtype=torch.float64, device=dev)
        gA = torch.zeros((nsteps, 3), dtype=torch.float64, device=dev)
        lam = h.position_scale(self.psi_final, self.occ, self.direction, h.volume_element)
        if self.powers is not None:
            for n in reversed(range(nsteps)):
                n2 = min(n + 1, nsteps - 1)
                h.etrs_adjoint_step_(lam, self.dt, self._kA(self._amp(amps, n)), self._kA(self._amp(amps, n + 1)),
                                     self.powers[n], gV, gA[n], gA[n2])
            return gA[:, self.direction].clone(), gV
        segments = [(s0, min(s0 + self.every, nsteps)) for s0 in range(0, nsteps, self.every)][::-1]
        seg = min(self.every, nsteps)
        have_tail = self._tail is not None and segments[0][0] == self._tail[0]
        if self._overlapped() and len(segments) > 1 and self.psi0.is_cuda:
            # two powers buffers alternate; where the second does not fit beside the
            # first (large cells in FP64), the segments run one after the other in one
            second = self._try_powers_buffer(seg)
            if second is not None:
                self._backward_overlapped(segments, lam, gV, gA, second)
                return gA[:, self.direction].clone(), gV
        # one buffer: the forward's copy of the last segment's powers, reused for the
        # recompute of every earlier segment once that segment has been walked back
        store = self._tail[1] if have_tail else h.powers_buffer(seg, self.M)
        for s0, s1 in segments:
            if not (have_tail and s0 == self._tail[0]):  # else the forward kept its powers
                psi = self.checkpoints[s0].clone()
                for n in range(s0, s1):
                    h.etrs_step_powers_(psi, self.dt, self._kA(self._amp(amps, n)),
                                        self._kA(self._amp(amps, n + 1)), store[n - s0])
            for n in reversed(range(s0, s1)):
                n2 = min(n + 1, nsteps - 1)
                h.etrs_adjoint_step_(lam, self.dt, self._kA(self._amp(amps, n)), self._kA(self._amp(amps, n + 1)),
                                     store[n - s0], gV, gA[n], gA[n2])
        del store
        return gA[:, self.direction].clone(), gV

    def _recompute_context(self):
        """The second context for the recompute stream: a clone of the Hamiltonian,
        made again whenever the Hamiltonian changed since."""
        if self._h2 is None or self._h2_version != self.h.state_version:
            self._h2 = self.h.clone()
            self._h2_version = self.h.state_version
        return self._h2

    # Grid points x orbitals up to which the recompute runs beside the backward walk.
    # Measured (ratio of forward + backward to the plain forward): 32^3 x 16 orbitals
    # 2.9x overlapped against 4.1x one after the other; 144^3 x 16 orbitals 4.27x
    # overlapped against 3.15x, where each step's kernels already fill the GPU and the
    # two streams only compete.
    OVERLAP_MAX_ELEMENTS = 1 << 22

    def _overlapped(self) -> bool:
        if self.overlap is None:
            return self.h.N * self.M <= self.OVERLAP_MAX_ELEMENTS
        return bool(self.overlap)

    def _try_powers_buffer(self, nsteps):
        """A powers buffer of nsteps steps, or None where the device has no room for it."""
        try:
            return self.h.powers_buffer(nsteps, self.M)
        except torch.OutOfMemoryError:
            return None

    def _backward_overlapped(self, segments, lam, gV, gA, second):
        """Segments in reverse time order; segment i + 1's recompute (second context,
        second stream) overlaps segment i's backward walk.  Two powers buffers
        alternate (the forward's copy of the last segment, or a new one, and `second`);
        events order each buffer's write after its previous read."""
        h, h2 = self.h, self._recompute_context()
        amps, nsteps = self.amps, len(self.amps)
        dev = self.psi0.device
        caller = torch.cuda.current_stream(dev)
        # the walk is the critical path: it runs on a high-priority stream, so the block
        # scheduler gives the recompute (default priority) only the SMs the walk leaves
        main = torch.cuda.Stream(device=dev, priority=-1)
        main.wait_stream(caller)
        side = torch.cuda.Stream(device=dev)
        seg = min(self.every, nsteps)
        have_tail = self._tail is not None and segments[0][0] == self._tail[0]
        first = self._tail[1] if have_tail else h.powers_buffer(seg, self.M)
        stores = [first, second]
        for b in stores:
            b.record_stream(side)
        ready = [torch.cuda.Event() for _ in segments]
        done = [torch.cuda.Event() for _ in segments]
        side.wait_stream(main)  # the checkpoints were written on the main stream

        # the recompute is enqueued by a second host thread (ctypes releases the GIL), so
        # the two streams are fed in parallel; host flags order each event wait after
        # the event's record
        import threading

        host_ready = [threading.Event() for _ in segments]
        host_done = [threading.Event() for _ in segments]
        failure = []
        limit_s = 600.0

        def recompute(i):
            s0, s1 = segments[i]
            buf = stores[i % 2]
            with torch.cuda.stream(side):
                if i >= 2:
                    if not host_done[i - 2].wait(limit_s):
                        raise RuntimeError("adjoint: the backward walk did not release a powers buffer")
                    side.wait_event(done[i - 2])  # the buffer's previous segment is walked back
                psi = self.checkpoints[s0].clone()
                for n in range(s0, s1):
                    h2.etrs_step_powers_(psi, self.dt, self._kA(self._amp(amps, n)),
                                         self._kA(self._amp(amps, n + 1)), buf[n - s0])
                ready[i].record(side)
            host_ready[i].set()

        def worker():
            try:
                torch.cuda.set_device(dev)
                for i in range(1 if have_tail else 0, len(segments)):
                    recompute(i)
            except BaseException as ex:  # reported by the main thread
                failure.append(ex)
                for e in host_ready:
                    e.set()

        if have_tail:
            ready[0].record(main)  # the forward kept the last segment's powers
            host_ready[0].set()
        thread = threading.Thread(target=worker, daemon=True)
        thread.start()
        try:
            with torch.cuda.stream(main):
                for i, (s0, s1) in enumerate(segments):
                    if not host_ready[i].wait(limit_s) or failure:
                        raise RuntimeError("adjoint: segment recompute failed") from (failure[0] if failure else None)
                    main.wait_event(ready[i])
                    buf = stores[i % 2]
                    for n in reversed(range(s0, s1)):
                        n2 = min(n + 1, nsteps - 1)
                        h.etrs_adjoint_step_(lam, self.dt, self._kA(self._amp(amps, n)),
                                             self._kA(self._amp(amps, n + 1)), buf[n - s0], gV, gA[n], gA[n2])
                    done[i].record(main)
                    host_done[i].set()
        finally:
            for e in host_done:
                e.set()  # let the worker finish (or fail) on every path
            thread.join(limit_s)
        if failure:
            raise RuntimeError("adjoint: segment recompute failed") from failure[0]
        caller.wait_stream(main)
        caller.wait_stream(side)
        if have_tail and len(segments) > 2:
            self._tail = None  # its buffer held later segments' powers: recompute next time


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
