"""real_time::propagate for static ions (src/real_time/propagate.hpp:33-140).

One call runs the time loop the reference runs: the zero-time kick, the initial
update of the Hamiltonian from the density, then per step the ETRS step (with its
self-consistency loop when the theory is interacting) or the Crank-Nicolson step (with
its Broyden-mixed self-consistency loop when the theory is interacting), the
TD-MLWF transformation when asked (propagate.hpp:105-111), the energy, the
real_time::results series, and a checkpoint every `checkpoint_every` steps
(results.hpp:52-66).  Every numerical step is a library call; this module only
orders them.

The energy is hamiltonian::energy::total without the ionic terms (energy.hpp:109-115):
sum_m occ_m eps_m - E_H - nvxc + E_xc, with eps_m = Re<psi_m|H|psi_m> / <psi_m|psi_m>
(energy.hpp:74-76).  The ion-ion term is a constant for static ions and is not added.
"""
from __future__ import annotations

import logging
import time

import numpy as np
import torch

from ._lib import THEORY_NONE
from .checkpoint import RealTimeResults, save_checkpoint
from .wannier import MLWFProperties

# The reference's console lines (propagate.hpp:89-90,130,134), at INFO; the start and
# end markers at DEBUG (the reference's trace level).
log = logging.getLogger("pinq_b200.propagate")


def _energy(ham, psi, occ, en):
    hpsi = ham.apply(psi)
    eps = ham.band_energies(psi, hpsi)
    del hpsi
    e = float(np.dot(occ, eps))
    if en is not None:
        e += -en["hartree"] - en["nvxc"] + en["xc"]
    return e


def propagate(ham, psi, occ, dt, num_steps, *, vion=None, theory=THEORY_NONE, propagator="etrs",
              vector_potential=None, kick=None, kick_gauge="velocity", tdmlwf=False, mlwf_out=None,
              results=None, checkpoint_dir=None, checkpoint_every=500, start_step=0, callback=None, nscf=5,
              scf_threshold=5e-5, cn_max_sweeps=300, cn_tol=1e-10, cn_max_iter=300, cn_dens_tol=1e-5,
              num_electrons=None):
    """Propagate psi ([N, M] CUDA tensor, in place) from start_step to num_steps.

    vion: FP64 CUDA tensor [N] of the ionic potential (the context's current potential
    when None and the theory is non-interacting).  theory: THEORY_NONE, THEORY_HARTREE or
    THEORY_LDA.  propagator: "etrs" or "crank_nicolson".  With an interacting theory, ETRS
    runs its SCF loop (nscf, scf_threshold) and Crank-Nicolson its Broyden-mixed loop
    (cn_max_iter, cn_dens_tol; num_electrons defaults to sum(occ)); without one,
    Crank-Nicolson runs solver sweeps to cn_tol (cn_max_sweeps).  vector_potential: callable t -> cartesian A(t)
    (zero when None).  kick: cartesian kick field (perturbations::kick); in the velocity
    gauge it adds the constant vector potential -kick, in the length gauge it multiplies
    the orbitals by exp(-i kick . r) at step 0.  mlwf_out: open text file for the TD-MLWF
    lines.  results: a RealTimeResults to append to (new when None).  callback(step, t,
    psi, rho, energy) runs after step 0 and after every step.  Returns the results."""
    if propagator not in ("etrs", "crank_nicolson"):
        raise ValueError("propagator must be 'etrs' or 'crank_nicolson'")
    if kick_gauge not in ("velocity", "length"):
        raise ValueError("kick_gauge must be 'velocity' or 'length'")
    occ = np.ascontiguousarray(occ, np.float64).reshape(psi.shape[1])
    results = RealTimeResults() if results is None else results
    kick_a = np.zeros(3) if (kick is None or kick_gauge == "length") else -np.asarray(kick, float)

    def kA(t):
        a = np.zeros(3) if vector_potential is None else np.asarray(vector_potential(t), float).reshape(3)
        return ham.cart_to_cov(a + kick_a)

    if start_step == 0 and kick is not None and kick_gauge == "length":
        ham.kick_(psi, kick)
    rho = ham.density(psi, occ)
    interacting = theory != THEORY_NONE
    en = None
    if interacting or vion is not None:
        en = ham.ks_potential(rho, vion, theory)
    ham.set_vector_potential_cov(kA(start_step * dt))
    energy = _energy(ham, psi, occ, en if interacting else None)
    if start_step == 0:
        results.record(0, 0.0, energy, ham.dipole(rho))
        if callback:
            callback(0, 0.0, psi, rho, energy)
    mlwf = MLWFProperties(ham) if tdmlwf else None

    log.debug("starting real-time propagation")
    log.info("step %9d :  t =  %9.3f  e = %.12f", start_step, start_step * dt, energy)
    t_last = time.perf_counter()
    for istep in range(start_step, num_steps):
        t = istep * dt
        k1, k2 = kA(t), kA(t + dt)
        if propagator == "etrs" and interacting:
            _, en = ham.etrs_scf_step_(psi, rho, dt, k1, k2, occ, vion, theory, nscf, scf_threshold)
        elif interacting:
            _, _, en = ham.crank_nicolson_scf_step_(psi, rho, dt, k1, k2, occ, vion, theory, cn_max_iter, cn_dens_tol,
                                                    num_electrons)
        else:
            if propagator == "etrs":
                ham.etrs_step_(psi, dt, k1, k2)
            else:
                ham.crank_nicolson_step_(psi, dt, k1, k2, cn_max_sweeps, cn_tol)
            rho = ham.density(psi, occ)
        if mlwf is not None:
            mlwf.calculate(mlwf_out, istep, psi)
        energy = _energy(ham, psi, occ, en if interacting else None)
        tt = (istep + 1) * dt
        results.record(istep + 1, tt, energy, ham.dipole(rho))
        if checkpoint_dir is not None and (istep + 1) % checkpoint_every == 0:
            torch.cuda.synchronize()
            save_checkpoint(checkpoint_dir, ham, psi, occ, rho, results)
        if callback:
            callback(istep + 1, tt, psi, rho, energy)
        now = time.perf_counter()
        log.info("step %9d :  t =  %9.3f  e = %.12f  wtime = %9.3f", istep + 1, tt, energy, now - t_last)
        t_last = now
    log.debug("real-time propagation ended normally")
    return results
