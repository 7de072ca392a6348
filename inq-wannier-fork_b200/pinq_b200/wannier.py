"""TD-MLWF output as the fork writes it after each real-time step.

real_time::propagate appends to ``mlwf_results.dat`` when the wavefunction
diagnostic is TDMLWF (src/real_time/propagate.hpp:105-111), through
observables::mlwf_properties::calculate (src/observables/mlwf_properties.hpp:28-44):

    Time step: <step + 1>
    MLWFs:
      WF <i + 1>: <x>     <y>     <z>     Spread: <s>

numbers as std::ostream prints doubles by default (6 significant digits, %g).
"""
from __future__ import annotations


def _g(v: float) -> str:
    return format(float(v), "g")


class MLWFProperties:
    """mlwf_properties: rotates the orbitals to the maximally localised gauge (in
    place, as the reference's apply_transform does) and records centres and spreads."""

    def __init__(self, ham, maxsweep: int = 100, tol: float = 1e-8):
        self.ham = ham
        self.maxsweep = maxsweep
        self.tol = tol
        self.last_sweeps = 0

    def calculate(self, out, time_step: int, psi):
        centres, spreads, self.last_sweeps = self.ham.mlwf_step_(psi, self.maxsweep, self.tol)
        if out is not None:
            out.write(f"Time step: {time_step + 1}\n")
            out.write("MLWFs:\n")
            for i, (c, s) in enumerate(zip(centres, spreads)):
                out.write(f"  WF {i + 1}: {_g(c[0])}     {_g(c[1])}     {_g(c[2])}     Spread: {_g(s)}\n")
        return centres, spreads
