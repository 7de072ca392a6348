"""Real-time checkpoints in INQ's on-disk layout, for resume and for exchange with INQ.

A checkpoint directory (INQ writes ``.inq/default_checkpoint/`` every 500 steps,
src/real_time/results.hpp:52-66) holds

    type                                   "real-time"
    real-time/observables/total_steps      text, one value
    real-time/observables/total_time
    real-time/observables/time             one value per line
    real-time/observables/total_energy
    real-time/observables/dipole           "x<TAB>y<TAB>z" per line (absent when empty)
    real-time/observables/current
    real-time/orbitals/...                 the electrons (KSHamiltonian.save_orbitals,
                                           save_density: C ABI, raw binary)

Text values are written as ``std::ofstream`` with ``precision(25)`` writes them
(utils::save_value / save_container, src/utils/load_save.hpp:45-135), i.e. C's
``%.25g``; ``type`` is removed first and written last, so a partial checkpoint has
no type file (results.hpp:58-66).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np


def _fmt(v) -> str:
    """A number as std::ostream << v with precision 25 prints it."""
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return format(float(v), ".25g")


def _write_value(path, v):
    with open(path, "w") as f:
        f.write(_fmt(v) + "\n")


def _write_container(path, values, vec3=False):
    if len(values) == 0:  # save_container removes the file of an empty container
        if os.path.exists(path):
            os.remove(path)
        return
    with open(path, "w") as f:
        for v in values:
            f.write("\t".join(_fmt(x) for x in v) + "\n" if vec3 else _fmt(v) + "\n")


def _read_lines(path):
    if not os.path.exists(path):
        return []
    with open(path) as f:
        return [ln for ln in f.read().split("\n") if ln.strip()]


@dataclass
class RealTimeResults:
    """real_time::results (src/real_time/results.hpp:18-100): one entry per step
    including step 0."""
    total_steps: int = 0
    total_time: float = 0.0
    time: list = field(default_factory=list)
    total_energy: list = field(default_factory=list)
    dipole: list = field(default_factory=list)
    current: list = field(default_factory=list)

    def record(self, step, t, energy, dipole=None, current=None):
        self.total_steps = int(step)
        self.total_time = float(t)
        self.time.append(float(t))
        self.total_energy.append(float(energy))
        if dipole is not None:
            self.dipole.append(tuple(float(x) for x in dipole))
        if current is not None:
            self.current.append(tuple(float(x) for x in current))
        if self.total_steps + 1 != len(self.time):
            raise ValueError("one record per step, starting at step 0")

    def save(self, dirname):
        """results::save (results.hpp:68-78)"""
        os.makedirs(dirname, exist_ok=True)
        _write_value(os.path.join(dirname, "total_steps"), self.total_steps)
        _write_value(os.path.join(dirname, "total_time"), self.total_time)
        _write_container(os.path.join(dirname, "time"), self.time)
        _write_container(os.path.join(dirname, "total_energy"), self.total_energy)
        _write_container(os.path.join(dirname, "dipole"), self.dipole, vec3=True)
        _write_container(os.path.join(dirname, "current"), self.current, vec3=True)

    @classmethod
    def load(cls, dirname):
        """results::load (results.hpp:80-100)"""
        for name in ("total_steps", "total_time", "time", "total_energy"):
            if not os.path.exists(os.path.join(dirname, name)):
                raise FileNotFoundError(f"cannot load real_time::results from directory '{dirname}'")
        r = cls()
        r.total_steps = int(_read_lines(os.path.join(dirname, "total_steps"))[0])
        r.total_time = float(_read_lines(os.path.join(dirname, "total_time"))[0])
        r.time = [float(x) for x in _read_lines(os.path.join(dirname, "time"))[: r.total_steps + 1]]
        r.total_energy = [float(x) for x in _read_lines(os.path.join(dirname, "total_energy"))[: r.total_steps + 1]]
        r.dipole = [tuple(float(x) for x in ln.split()) for ln in _read_lines(os.path.join(dirname, "dipole"))]
        r.current = [tuple(float(x) for x in ln.split()) for ln in _read_lines(os.path.join(dirname, "current"))]
        if len(r.time) != r.total_steps + 1:
            raise ValueError("time series shorter than total_steps + 1")
        for s in (r.dipole, r.current):
            if len(s) not in (0, r.total_steps + 1):
                raise ValueError("observable series of the wrong length")
        return r


def save_checkpoint(dirname, ham, psi, occ, rho, results, kpin=0, first_state=0, root=True):
    """The checkpoint results::operator() writes (results.hpp:52-66).  With the states
    sharded over ranks, every rank calls this with its own block (first_state) and
    root=True on one rank only, which writes the observables, the density and the
    type file; the caller synchronises the ranks before and after."""
    typef = os.path.join(dirname, "type")
    if root and os.path.exists(typef):
        os.remove(typef)
    if root:
        results.save(os.path.join(dirname, "real-time", "observables"))
    edir = os.path.join(dirname, "real-time", "orbitals")
    ham.save_orbitals(edir, psi, occ, kpin=kpin, first_state=first_state)
    if root:
        ham.save_density(edir, rho)
        with open(typef, "w") as f:
            f.write("real-time\n")


def load_checkpoint(dirname, ham, psi, rho=None, kpin=0, first_state=0):
    """Inverse of save_checkpoint: fills psi (and rho), returns (results, occupations).
    A directory without the type file "real-time" is not a complete checkpoint."""
    typef = os.path.join(dirname, "type")
    if not os.path.exists(typef) or open(typef).read().split()[:1] != ["real-time"]:
        raise FileNotFoundError(f"'{dirname}' holds no complete real-time checkpoint")
    results = RealTimeResults.load(os.path.join(dirname, "real-time", "observables"))
    edir = os.path.join(dirname, "real-time", "orbitals")
    occ = ham.load_orbitals(edir, psi, kpin=kpin, first_state=first_state)
    if rho is not None:
        ham.load_density(edir, rho)
    return results, occ
