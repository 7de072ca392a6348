"""Checkpoint layout on the CPU: number formatting, the real_time::results text
series and the order of a checkpoint's files (src/real_time/results.hpp:52-100,
src/utils/load_save.hpp:45-210, src/utils/num_str.hpp:20-24,75-80)."""
import os

import numpy as np
import pytest

from pinq_b200.checkpoint import RealTimeResults, load_checkpoint, save_checkpoint


def test_num_to_str_golden(oracle_mod):
    # the reference's own test values (num_str.hpp:75-77)
    assert oracle_mod.num_to_str(0) == "0000000000"
    assert oracle_mod.num_to_str(1024) == "0000001024"
    assert oracle_mod.num_to_str(-333) == "-000000333"


def _results(n=4, with_current=False):
    r = RealTimeResults()
    rng = np.random.default_rng(1)
    for i in range(n):
        r.record(i, 0.05 * i, -12.5 + 1e-3 * rng.standard_normal(), rng.standard_normal(3),
                 rng.standard_normal(3) if with_current else None)
    return r


def test_results_text_format_and_round_trip(tmp_path):
    r = _results()
    d = tmp_path / "obs"
    r.save(str(d))
    # precision(25) formatting of std::ostream: %.25g, integers plain
    assert (d / "total_steps").read_text() == "3\n"
    assert (d / "total_time").read_text() == format(0.15000000000000002, ".25g") + "\n"
    assert (d / "time").read_text().split("\n")[1] == "0.05000000000000000277555756"
    x, y, z = r.dipole[2]
    assert (d / "dipole").read_text().split("\n")[2] == "\t".join(format(v, ".25g") for v in (x, y, z))
    assert not (d / "current").exists()  # an empty container leaves no file
    back = RealTimeResults.load(str(d))
    assert back.total_steps == 3 and back.time == r.time and back.total_energy == r.total_energy
    assert back.dipole == r.dipole and back.current == []


def test_results_require_one_record_per_step():
    r = RealTimeResults()
    r.record(0, 0.0, 1.0)
    with pytest.raises(ValueError):
        r.record(2, 0.1, 1.0)


class _LayoutHam:
    """Stands in for KSHamiltonian's save/load on the CPU: the oracle's restatement
    of the orbital layout."""

    def __init__(self, oracle_mod, N):
        self.o = oracle_mod
        self.N = N
        self.calls = []

    def save_orbitals(self, d, psi, occ, kpin=0, first_state=0):
        self.calls.append(("orbitals", os.path.exists(os.path.join(os.path.dirname(os.path.dirname(d)), "type"))))
        self.o.save_orbitals_layout(d, psi, occ, kpin, first_state)

    def save_density(self, d, rho):
        os.makedirs(os.path.join(d, "spin_density"), exist_ok=True)
        np.asarray(rho, np.float64).tofile(os.path.join(d, "spin_density", "0000000000"))

    def load_orbitals(self, d, psi, kpin=0, first_state=0):
        p, occ = self.o.load_orbitals_layout(d, self.N, psi.shape[1], kpin, first_state)
        psi[...] = p
        return occ

    def load_density(self, d, rho):
        rho[...] = np.fromfile(os.path.join(d, "spin_density", "0000000000"))


def test_checkpoint_order_and_round_trip(oracle_mod, tmp_path):
    N, M = 50, 3
    rng = np.random.default_rng(2)
    psi = rng.standard_normal((N, M)) + 1j * rng.standard_normal((N, M))
    rho = rng.random(N)
    occ = np.array([2.0, 2.0, 1.0])
    ham = _LayoutHam(oracle_mod, N)
    d = str(tmp_path / "ckpt")
    os.makedirs(d)
    open(os.path.join(d, "type"), "w").write("real-time\n")  # a previous checkpoint
    r = _results(3, with_current=True)
    save_checkpoint(d, ham, psi, occ, rho, r)
    assert ham.calls == [("orbitals", False)]  # the type file is gone while data is written
    assert open(os.path.join(d, "type")).read() == "real-time\n"
    files = sorted(os.listdir(os.path.join(d, "real-time", "orbitals", "kpin0000000000", "states")))
    assert files == ["0000000000_0000000000", "0000000001_0000000000", "0000000002_0000000000"]
    psi2 = np.zeros_like(psi)
    rho2 = np.zeros_like(rho)
    back, occ2 = load_checkpoint(d, ham, psi2, rho2)
    assert np.array_equal(psi2, psi) and np.array_equal(rho2, rho) and np.array_equal(occ2, occ)
    assert back.current == r.current
    os.remove(os.path.join(d, "type"))
    with pytest.raises(FileNotFoundError):
        load_checkpoint(d, ham, psi2, rho2)
