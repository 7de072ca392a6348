"""Shared builders for the parity tests: one synthetic system, set up identically
in the oracle (CPU FP64) and in the CUDA library."""
from __future__ import annotations

import numpy as np


def rel_max(a, b) -> float:
    """max |a - b| / max |b|"""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def rel_norm(a, b) -> float:
    """||a - b|| / ||b||"""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def small_system(pb, n=32, a=10.26, M=8, seed=0, with_proj=True, ecut=25.0, reps=1):
    from pinq_b200 import systems

    lattice = systems.cubic(a)
    nr = (n, n, n)
    pos = systems.diamond_positions(a / reps, reps)
    V = systems.gaussian_potential(lattice, nr, pos)
    psi = systems.random_orbitals(lattice, nr, M, ecut, seed)
    return dict(lattice=lattice, nr=nr, positions=pos if with_proj else np.zeros((0, 3)), V=V, psi=psi, M=M)


def make_oracle(oracle_mod, sysd, kA_cov=(0.0, 0.0, 0.0)):
    o = oracle_mod.System(sysd["lattice"], sysd["nr"])
    o.set_potential(sysd["V"])
    o.set_vector_potential_cov(np.asarray(kA_cov, float))
    if len(sysd["positions"]):
        o.set_projectors(o.build_gaussian_kb(sysd["positions"]))
    return o


def make_product(pb, sysd, precision="fp64", kA_cov=(0.0, 0.0, 0.0)):
    h = pb.KSHamiltonian(sysd["lattice"], sysd["nr"], precision)
    h.set_scalar_potential(sysd["V"])
    if len(sysd["positions"]):
        h.set_gaussian_projectors(sysd["positions"])
    h.set_vector_potential_cov(np.asarray(kA_cov, float))
    return h
