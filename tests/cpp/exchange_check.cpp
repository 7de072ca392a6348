// The C++ adapter's exchange seam on the host: INQ's enabled() threshold, and a
// ks_hamiltonian with a nonzero exact-exchange coefficient refused before any device
// work (so this runs without a GPU).
#include <cstdio>
#include <stdexcept>

#include "../../inq-wannier-fork_b200/host/inq_b200.hpp"

int main() {
  using inq::b200::exchange_operator;
  int bad = 0;
  if (exchange_operator::would_enable(0.0) || exchange_operator::would_enable(1e-15)) bad++;
  if (!exchange_operator::would_enable(0.25) || !exchange_operator::would_enable(-1.0)) bad++;
  if (exchange_operator{}.enabled()) bad++;
  const std::array<double, 9> lat = {10, 0, 0, 0, 10, 0, 0, 0, 10};
  for (double c : {0.25, 1.0}) {
    bool threw = false;
    try {
      inq::b200::ks_hamiltonian h(lat, {16, 16, 16}, inq::b200::precision::fp64, 0, c);
    } catch (const std::invalid_argument&) {
      threw = true;
    }
    if (!threw) bad++;
  }
  std::printf("bad=%d\n", bad);
  return bad != 0;
}
