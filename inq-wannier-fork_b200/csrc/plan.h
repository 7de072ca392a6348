// Launch plan: the compiled kernel set for one (grid, precision) pair.
#pragma once

namespace inqb {

struct LaunchArgs {
  enum Mode { H = 0, FFT_FWD = 1, FFT_BWD = 2, POISSON = 3 };
  int mode = H;
  const void* in = nullptr;
  long ld_in = 0;
  void* out = nullptr;
  long ld_out = 0;
  int M = 0;
  void* tmp = nullptr;              // Fourier workspace, [groups][N][G] rounded up for both tilings
  const void* tw = nullptr;         // twiddles x | y | z
  const void* proj_view = nullptr;  // ProjView<T>*
  const void* V = nullptr;          // [N] local potential (T)
  double rlat[3][3] = {};           // reciprocal vectors (rows)
  double kA_cart[3] = {};           // cartesian k + A
  const void* base = nullptr;       // optional epilogue base (out = alpha H in + beta base)
  long ld_base = 0;
  double alpha[2] = {1.0, 0.0};
  double beta[2] = {0.0, 0.0};
  void* stream = nullptr;
  int fourier_mask = 0;             // zero the kinetic term outside the Fourier sphere
  // optional cudaEvent_t: start, end of the projection kernel, start of the first tile
  // pass, and after each of the three passes
  void* events[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  // launch schedule (0 = the compiled default): CTAs sharing one x-plane in the first
  // pass (a divisor of the y split's Y1), and threads per CTA of the three passes
  int ysplit = 0;
  int threads[3] = {0, 0, 0};
  // optional, H mode: forward 3-D coefficients of `in` (before the kinetic factor) in
  // the tile layout [g][ka][kz][kx][kb][G] (groups padded to G orbitals)
  void* fourier_out = nullptr;
  // H mode: when set (a BatchCellDesc*, batch.h), describe the apply for the
  // persistent batch launch instead of launching it
  void* batch_cell = nullptr;
};

// Candidate values the autotuner tries.
constexpr int kScheduleThreads[2] = {128, 256};

struct Plan {
  int G = 1;       // orbitals per tile of the plain FFT kernels
  int G_tile = 1;  // orbitals per tile of the H kernels
  int y1 = 1;      // tiles per x-plane (the divisors of y1 are the first pass's splits)
  int y2 = 1;      // rows per tile (the y split is NY = y2 * y1)
  int ysplit = 1;  // default split
  int (*launch)(const LaunchArgs&) = nullptr;
};

const Plan* find_plan(int nx, int ny, int nz, int precision);
int launch_phases(int precision, int nent, const float* relpos, const double kA[3], void* phase, void* rec,
                  void* rec_pt, const int* pt_pos, void* adj, const int* atom_pos, void* stream);

}  // namespace inqb
