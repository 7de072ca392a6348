// Host side of the library's Broyden density mixer (csrc/broyden_host.h) on the CPU:
// the SPD solve on the reference's least_squares test systems
// (src/solvers/least_squares.hpp:69-129), and the whole mixer, with plain loops in
// place of the device passes (the same arithmetic as the kernels in
// csrc/potential.cu), on the reference's broyden test (src/mixers/broyden.hpp:163-203).
// Prints one line per case; the test reads them.
#include <cmath>
#include <cstdio>
#include <vector>

#include "../../inq-wannier-fork_b200/csrc/broyden_host.h"

using inqb::BroydenRing;

static void solve_case(const char* name, double a00, double a01, double a11, double b0, double b1) {
  std::vector<double> a = {a00, a01, a01, a11}, b = {b0, b1};
  const bool ok = inqb::spd_solve(2, a, b);
  std::printf("%s %d %.12f %.12f\n", name, ok ? 1 : 0, b[0], b[1]);
}

// One mixer call with the ring and vectors held on the host.
struct HostMixer {
  BroydenRing ring;
  long n;
  std::vector<double> df, dv, f_old, vin_old;
  HostMixer(int steps, double mix, long dim) : n(dim), df(steps * dim), dv(steps * dim), f_old(dim), vin_old(dim) {
    ring.max_size = steps;
    ring.mix = mix;
  }
  double dot(const double* a, const double* b) const {
    double s = 0.0;
    for (long i = 0; i < n; i++) s += a[i] * b[i];
    return s;
  }
  bool operator()(std::vector<double>& vin, const std::vector<double>& vout) {
    const int pos = ring.begin();
    double* dfp = pos >= 0 ? &df[pos * n] : nullptr;
    double* dvp = pos >= 0 ? &dv[pos * n] : nullptr;
    for (long i = 0; i < n; i++) {  // k_broyden_diff
      const double x = vin[i], f = vout[i] - x;
      if (dfp) {
        dfp[i] = f - f_old[i];
        dvp[i] = x - vin_old[i];
      }
      f_old[i] = f;
      vin_old[i] = x;
    }
    if (pos >= 0) {
      const double gamma = std::max(1e-8, std::sqrt(dot(dfp, dfp)));
      for (long i = 0; i < n; i++) {  // k_scale2
        dfp[i] *= 1.0 / gamma;
        dvp[i] *= 1.0 / gamma;
      }
      ring.filled(pos);
    }
    const int used = ring.used();
    std::vector<double> c(used > 0 ? used : 1, 0.0);
    if (used > 0) {
      std::vector<double> dots;
      for (int i = 0; i < used; i++)
        for (int j = i + 1; j < used; j++) dots.push_back(dot(&df[i * n], &df[j * n]));
      for (int i = 0; i < used; i++) dots.push_back(dot(&df[i * n], f_old.data()));
      if ((int)dots.size() != inqb::broyden_num_dots(used)) return false;
      if (!inqb::broyden_coefficients(used, dots.data(), c.data())) return false;
    }
    for (long i = 0; i < n; i++) {  // k_broyden_update
      double v = vin[i] + ring.mix * f_old[i];
      for (int k = 0; k < used; k++) v -= c[k] * (ring.mix * df[k * n + i] + dv[k * n + i]);
      vin[i] = v;
    }
    return true;
  }
};

int main() {
  solve_case("lsq_diagonal", 4.0, 0.0, 2.0, 0.0, 1.0);
  solve_case("lsq_symmetric_1", 0.89653, 0.41072, 0.69479, 0.21563, 0.40103);
  solve_case("lsq_symmetric_2", 6432.12, 4502.48, 3151.74, 1.0, 1.0);

  HostMixer m(5, 0.5, 2);
  std::vector<double> vin = {10.0, -20.0};
  bool ok = m(vin, {0.0, 22.2});
  std::printf("broyden_1 %d %.12f %.12f\n", ok ? 1 : 0, vin[0], vin[1]);
  ok = m(vin, {4.0, 5.5});
  std::printf("broyden_2 %d %.12f %.12f\n", ok ? 1 : 0, vin[0], vin[1]);

  // a longer run past the ring's wrap-around (4 slots): a linear map's fixed point
  HostMixer w(4, 0.3, 3);
  std::vector<double> x = {1.0, 0.0, 0.0};
  for (int it = 0; it < 12; it++) {
    const std::vector<double> out = {0.5 * x[1] + 1.0, 0.25 * x[0] - 0.5 * x[2], 0.1 * x[0] + 2.0};
    if (!w(x, out)) ok = false;
  }
  std::printf("broyden_wrap %d %d %.15e %.15e %.15e\n", ok ? 1 : 0, w.ring.calls, x[0], x[1], x[2]);
  return 0;
}
