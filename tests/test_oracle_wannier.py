"""The oracle's TD-MLWF against the reference's jade_complex test values
(src/wannier/jade_complex.hpp, fixture tests/golden/jade_cases.json made by
tests/golden/make_jade_cases.py) and against localised states with known centres."""
import json
import os

import numpy as np
import pytest

from wannier_cases import CENTRES, SIGMA, check_value, gaussian_states, jade_case

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "jade_cases.json")


@pytest.mark.parametrize("idx", [0, 1])
def test_jade_golden(oracle_mod, idx):
    case = json.load(open(GOLDEN))[idx]
    a, maxsweep, tol = jade_case(case)
    _, u, adiag, sweeps = oracle_mod.jade(a, maxsweep, tol)
    assert 1 <= sweeps < maxsweep
    for chk in case["checks"]:
        # the reference prints 8 decimal places
        assert check_value(chk, u, adiag) == pytest.approx(chk["value"], abs=5e-8), chk
    assert np.allclose(u @ u.conj().T, np.eye(case["n"]), atol=1e-12)


def test_mlwf_recovers_gaussian_centres(oracle_mod):
    o, psi, lat = gaussian_states(oracle_mod)
    a = o.mlwf_matrices(psi)
    for k in range(6):
        assert np.allclose(a[k], a[k].conj().T, atol=1e-13)  # Hermitian (real weights)
    _, u, adiag, sweeps = oracle_mod.jade(a)
    assert sweeps < 100
    found = np.array([oracle_mod.mlwf_center(adiag, i, lat) for i in range(len(CENTRES))])
    for c in CENTRES:
        d = found - c
        d -= lat[0, 0] * np.round(d / lat[0, 0])
        assert np.linalg.norm(d, axis=1).min() < 2e-2
    # a Gaussian with |psi|^2 ~ exp(-r^2 / sigma^2): |<e^{i k x}>| = exp(-k^2 sigma^2 / 4), so
    # the periodic spread is sqrt(3 (1 - exp(-k^2 sigma^2 / 2))) / k with k = 2 pi / L
    k = 2 * np.pi / lat[0, 0]
    expect = np.sqrt(3 * (1 - np.exp(-k * k * SIGMA**2 / 2))) / k
    spreads = np.array([oracle_mod.mlwf_spread(adiag, i, lat) for i in range(len(CENTRES))])
    assert np.allclose(spreads, expect, rtol=0.01)
    # the rotation is unitary: the rotated states stay orthonormal
    w = o.mlwf_rotate(psi, u)
    assert np.allclose(w.conj().T @ w * o.volume_element, np.eye(len(CENTRES)), atol=1e-12)
