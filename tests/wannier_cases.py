"""Shared input of the TD-MLWF tests: localised Gaussians in a cubic cell, mixed by a
seeded unitary so that the Wannier transformation has something to undo."""
import numpy as np

A = 10.0
NR = (24, 24, 24)
SIGMA = 0.8
CENTRES = np.array([[-2.5, -2.5, -2.5], [2.5, 0.0, -1.25], [0.0, 2.5, 2.5], [-2.5, 2.5, 0.0],
                    [2.5, -2.5, 2.5], [0.0, 0.0, 0.0]])


def gaussian_states(oracle_mod, seed=0):
    """(oracle System, mixed orthonormal states [N, M], lattice)"""
    lat = np.eye(3) * A
    o = oracle_mod.System(lat, NR)
    r = o.rvectors()
    psi = np.zeros((o.N, len(CENTRES)), complex)
    for j, c in enumerate(CENTRES):
        d = r - c
        d -= A * np.round(d / A)  # nearest periodic image
        psi[:, j] = np.exp(-(d * d).sum(1) / (2 * SIGMA**2))
    psi = o.orthonormalize(psi)
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((len(CENTRES),) * 2) + 1j * rng.standard_normal((len(CENTRES),) * 2))
    return o, psi @ q, lat


def jade_case(case):
    """(a [6][n][n], maxsweep, tol) of one golden case"""
    n = case["n"]
    a = np.zeros((6, n, n), complex)
    for key, (re, im) in case["a"].items():
        k, i, j = (int(x) for x in key.split(","))
        a[k, i, j] = complex(re, im)
    return a, case["maxsweep"], case["tol"]


def check_value(case_check, u, adiag):
    arr = u if case_check["array"] == "u" else adiag
    v = arr[tuple(case_check["index"])]
    return v.real if case_check["part"] == "real" else v.imag
