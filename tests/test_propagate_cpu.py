"""Host logic of pinq_b200.propagate (real_time::propagate, src/real_time/propagate.hpp:33-140)
on the CPU, against a recording stand-in for the Hamiltonian: the order of the calls,
the two kick gauges (perturbations/kick.hpp:20-61), the vector potential at t and t + dt
(etrs.hpp:22-82), resuming from a step, the checkpoint cadence (results.hpp:52-66), the
energy bookkeeping (hamiltonian/energy.hpp:109-115) and the TD-MLWF lines
(observables/mlwf_properties.hpp:28-44).  No library call runs here; the numerical steps
themselves are covered by the GPU tests."""
import io
import sys

import numpy as np
import pytest
import torch


class RecordingHamiltonian:
    """The members propagate() calls, on CPU tensors.  H acts as 3 times the identity,
    so every band energy is 3; each propagation step multiplies psi by exp(-0.1 i)."""

    def __init__(self, M, energies=None):
        self.M = M
        self.log = []
        self.energies = energies or {"external": 0.5, "hartree": 1.25, "xc": -0.75, "nvxc": -0.5}

    def cart_to_cov(self, a):
        return 2.0 * np.asarray(a, float)

    def kick_(self, psi, kick):
        self.log.append(("kick", tuple(float(x) for x in kick)))
        return psi

    def density(self, psi, occ):
        self.log.append(("density",))
        return (psi.abs() ** 2) @ torch.as_tensor(occ, dtype=torch.float64)

    def ks_potential(self, rho, vion, theory, energies=True):
        self.log.append(("ks_potential", theory))
        return dict(self.energies)

    def set_vector_potential_cov(self, k):
        self.log.append(("set_A", tuple(float(x) for x in k)))

    def apply(self, psi):
        return 3.0 * psi

    def band_energies(self, psi, hpsi):
        return np.full(self.M, 3.0)

    def dipole(self, rho):
        return [float(rho.sum()), 0.0, 0.0]

    def _advance(self, psi):
        psi.mul_(complex(np.cos(0.1), -np.sin(0.1)))

    def etrs_step_(self, psi, dt, k1, k2):
        self.log.append(("etrs", dt, tuple(k1), tuple(k2)))
        self._advance(psi)
        return psi

    def crank_nicolson_step_(self, psi, dt, k1, k2, sweeps, tol):
        self.log.append(("cn", dt, tuple(k1), tuple(k2), sweeps, tol))
        self._advance(psi)
        return 4, 1e-12

    def etrs_scf_step_(self, psi, rho, dt, k1, k2, occ, vion, theory, nscf, threshold):
        self.log.append(("etrs_scf", dt, tuple(k1), tuple(k2), theory, nscf, threshold))
        self._advance(psi)
        rho.copy_(self.density(psi, occ))
        return 2, dict(self.energies)

    def crank_nicolson_scf_step_(self, psi, rho, dt, k1, k2, occ, vion, theory, max_iter, dens_tol, num_electrons):
        self.log.append(("cn_scf", dt, tuple(k1), tuple(k2), theory, max_iter, dens_tol, num_electrons))
        self._advance(psi)
        rho.copy_(self.density(psi, occ))
        return 3, 1e-9, dict(self.energies)

    def mlwf_step_(self, psi, maxsweep, tol):
        self.log.append(("mlwf", maxsweep, tol))
        return np.zeros((self.M, 3)), np.full(self.M, 1.5), 1


def _psi(M=3, N=8):
    g = torch.Generator().manual_seed(5)
    return torch.randn((N, M), dtype=torch.complex128, generator=g)


def _steps(h, kind):
    return [e for e in h.log if e[0] == kind]


def test_velocity_gauge_kick_is_a_constant_vector_potential():
    from pinq_b200 import propagate

    h = RecordingHamiltonian(3)
    res = propagate(h, _psi(), np.full(3, 2.0), 0.05, 2, kick=(0.01, 0.0, 0.0), vector_potential=lambda t: (t, 0.0, 0.0))
    assert not _steps(h, "kick")
    etrs = _steps(h, "etrs")
    assert len(etrs) == 2
    for n, (_, dt, k1, k2) in enumerate(etrs):
        assert dt == 0.05
        # A(t) - kick, then to covariant components
        assert k1 == pytest.approx((2 * (n * 0.05 - 0.01), 0.0, 0.0))
        assert k2 == pytest.approx((2 * ((n + 1) * 0.05 - 0.01), 0.0, 0.0))
    assert h.log[0][0] == "density" and _steps(h, "set_A")[0][1] == pytest.approx((-0.02, 0.0, 0.0))
    assert res.total_steps == 2 and res.time == pytest.approx([0.0, 0.05, 0.1])


def test_length_gauge_kick_multiplies_the_orbitals_once_before_the_first_density():
    from pinq_b200 import propagate

    h = RecordingHamiltonian(3)
    propagate(h, _psi(), np.full(3, 2.0), 0.05, 3, kick=(0.0, 0.02, 0.0), kick_gauge="length")
    assert h.log[0] == ("kick", (0.0, 0.02, 0.0))
    assert h.log[1] == ("density",)
    assert len(_steps(h, "kick")) == 1
    assert all(k1 == (0.0, 0.0, 0.0) and k2 == (0.0, 0.0, 0.0) for _, _, k1, k2 in _steps(h, "etrs"))


def test_resume_appends_to_the_results_and_skips_the_zero_time_work():
    from pinq_b200 import propagate
    from pinq_b200.checkpoint import RealTimeResults

    occ = np.full(3, 2.0)
    first = RecordingHamiltonian(3)
    psi = _psi()
    res = propagate(first, psi, occ, 0.05, 2, kick=(0.0, 0.02, 0.0), kick_gauge="length")
    again = RealTimeResults()
    for s in range(3):
        again.record(s, res.time[s], res.total_energy[s], res.dipole[s])
    h = RecordingHamiltonian(3)
    calls = []
    res2 = propagate(h, psi, occ, 0.05, 5, kick=(0.0, 0.02, 0.0), kick_gauge="length", results=again, start_step=2,
                     callback=lambda step, t, *_: calls.append(step))
    assert not _steps(h, "kick")
    assert len(_steps(h, "etrs")) == 3
    assert res2 is again and res2.total_steps == 5 and len(res2.time) == 6
    assert res2.time[3:] == pytest.approx([0.15, 0.2, 0.25])
    assert calls == [3, 4, 5]


def test_checkpoint_every_n_steps(monkeypatch):
    import pinq_b200  # noqa: F401

    pm = sys.modules["pinq_b200.propagate"]  # the package's `propagate` is the function

    saved = []
    monkeypatch.setattr(pm, "save_checkpoint", lambda d, ham, psi, occ, rho, results: saved.append(
        (d, results.total_steps)))
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    h = RecordingHamiltonian(3)
    pm.propagate(h, _psi(), np.full(3, 2.0), 0.05, 7, checkpoint_dir="ckpt", checkpoint_every=3)
    assert saved == [("ckpt", 3), ("ckpt", 6)]


def test_energy_without_and_with_the_density_terms():
    from pinq_b200 import THEORY_LDA, propagate

    occ = np.array([2.0, 2.0, 1.0])
    h = RecordingHamiltonian(3)
    res = propagate(h, _psi(), occ, 0.05, 2)
    assert res.total_energy == pytest.approx([15.0, 15.0, 15.0])  # sum occ * 3
    h = RecordingHamiltonian(3)
    vion = torch.zeros(8, dtype=torch.float64)
    res = propagate(h, _psi(), occ, 0.05, 2, vion=vion, theory=THEORY_LDA, nscf=4, scf_threshold=1e-6)
    # sum occ eps - E_H - nvxc + E_xc
    assert res.total_energy == pytest.approx([15.0 - 1.25 + 0.5 - 0.75] * 3)
    scf = _steps(h, "etrs_scf")
    assert len(scf) == 2 and all(e[4:] == (THEORY_LDA, 4, 1e-6) for e in scf)
    assert _steps(h, "ks_potential") == [("ks_potential", THEORY_LDA)]
    assert not _steps(h, "etrs")


def test_non_interacting_ionic_potential_is_set_once_and_not_counted_in_the_energy():
    from pinq_b200 import propagate

    occ = np.full(3, 2.0)
    h = RecordingHamiltonian(3)
    res = propagate(h, _psi(), occ, 0.05, 2, vion=torch.zeros(8, dtype=torch.float64))
    assert _steps(h, "ks_potential") == [("ks_potential", 0)]
    assert len(_steps(h, "etrs")) == 2
    assert res.total_energy == pytest.approx([18.0] * 3)


def test_crank_nicolson_passes_the_solver_settings():
    from pinq_b200 import propagate

    h = RecordingHamiltonian(3)
    propagate(h, _psi(), np.full(3, 2.0), 0.1, 2, propagator="crank_nicolson", cn_max_sweeps=50, cn_tol=1e-9)
    cn = _steps(h, "cn")
    assert len(cn) == 2 and all(e[1] == 0.1 and e[4:] == (50, 1e-9) for e in cn)


def test_tdmlwf_lines_after_every_step():
    from pinq_b200 import propagate

    out = io.StringIO()
    h = RecordingHamiltonian(2)
    propagate(h, _psi(M=2), np.full(2, 2.0), 0.05, 2, tdmlwf=True, mlwf_out=out)
    text = out.getvalue()
    assert text.count("MLWFs:") == 2 and "Time step: 1\n" in text and "Time step: 2\n" in text
    assert text.count("Spread:") == 4
    # the transformation runs after the propagation step of the same time step
    kinds = [e[0] for e in h.log if e[0] in ("etrs", "mlwf")]
    assert kinds == ["etrs", "mlwf", "etrs", "mlwf"]


def test_callback_sees_every_step_from_zero():
    from pinq_b200 import propagate

    seen = []
    h = RecordingHamiltonian(3)
    propagate(h, _psi(), np.full(3, 2.0), 0.05, 3, callback=lambda step, t, psi, rho, e: seen.append((step, t, e)))
    assert [s for s, _, _ in seen] == [0, 1, 2, 3]
    assert [t for _, t, _ in seen] == pytest.approx([0.0, 0.05, 0.1, 0.15])


def test_crank_nicolson_with_a_density_dependent_potential_runs_the_mixed_loop():
    from pinq_b200 import THEORY_HARTREE, propagate

    occ = np.full(3, 2.0)
    h = RecordingHamiltonian(3)
    res = propagate(h, _psi(), occ, 0.1, 2, vion=torch.zeros(8, dtype=torch.float64), theory=THEORY_HARTREE,
                    propagator="crank_nicolson", cn_max_iter=40, cn_dens_tol=1e-6, num_electrons=6.0,
                    vector_potential=lambda t: (0.0, t, 0.0))
    cn = _steps(h, "cn_scf")
    assert len(cn) == 2 and not _steps(h, "cn") and not _steps(h, "etrs_scf")
    for n, e in enumerate(cn):
        assert e[1] == 0.1 and e[4:] == (THEORY_HARTREE, 40, 1e-6, 6.0)
        assert e[2] == pytest.approx((0.0, 2 * n * 0.1, 0.0)) and e[3] == pytest.approx((0.0, 2 * (n + 1) * 0.1, 0.0))
    assert res.total_energy == pytest.approx([18.0 - 1.25 + 0.5 - 0.75] * 3)


@pytest.mark.parametrize("kwargs,exc", [
    ({"propagator": "rk4"}, ValueError),
    ({"kick_gauge": "coulomb"}, ValueError),
])
def test_argument_errors(kwargs, exc):
    from pinq_b200 import propagate

    h = RecordingHamiltonian(3)
    with pytest.raises(exc):
        propagate(h, _psi(), np.full(3, 2.0), 0.05, 1, **kwargs)
    assert h.log == []


def test_console_lines_follow_the_reference(caplog):
    """propagate.hpp:89-90,130: one line at the start step, one per step with the wall
    time of that step."""
    import logging
    import re

    from pinq_b200 import propagate

    h = RecordingHamiltonian(3)
    with caplog.at_level(logging.DEBUG, logger="pinq_b200.propagate"):
        propagate(h, _psi(), np.full(3, 2.0), 0.05, 2)
    msgs = [r.getMessage() for r in caplog.records if r.name == "pinq_b200.propagate"]
    assert msgs[0] == "starting real-time propagation" and msgs[-1] == "real-time propagation ended normally"
    assert msgs[1] == "step         0 :  t =      0.000  e = 18.000000000000"
    for n, m in enumerate(msgs[2:4], start=1):
        assert re.fullmatch(rf"step {n:9d} :  t =  {n * 0.05:9.3f}  e = 18\.000000000000  wtime = +\d+\.\d{{3}}", m), m
