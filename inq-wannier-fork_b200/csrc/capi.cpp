// extern "C" entry points of libinqb200 (declared in include/inqb200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "batch.h"
#include "inqb_internal.h"
#include "broyden_host.h"
#include "adjoint.h"
#include "checkpoint.h"
#include "observables.h"
#include "potential.h"
#include "propagators.h"
#include "wannier.h"
#include "plan.h"
#include "project.h"

namespace inqb {
const char* last_error();
void twiddle_table(int n, int n1, int n2, std::vector<double>& re, std::vector<double>& im);
int split_of(int n, int* n1, int* n2);
int build_proj_tables(const inqb_ctx& ctx, int nproj, int L, int smax, const int* counts, const int* coords,
                      const float* relpos, const double* beta, const double* coeff, ProjTables& t);
int upload_proj_tables(const inqb_ctx& ctx, ProjTables& t);
int sphere_points(const CellGeom& cell, const int nr[3], const double center[3], double radius, int npts, int* coords,
                  float* dist, float* relpos, int* count_out);
int gaussian_kb_beta(const CellGeom& cell, int npts, const float* dist, const float* relpos, double sigma,
                     double* beta);
constexpr int kMaxL = 4;

namespace {

struct DeviceGuard {
  int prev = -1;
  int status = INQB_OK;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) status = fail(INQB_ERR_CUDA, "cudaSetDevice failed");
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

#define INQB_CHECK_CTX(ctx)                                                   \
  do {                                                                        \
    if (!(ctx)) return ::inqb::fail(INQB_ERR_INVALID, "null context");        \
  } while (0)

#define INQB_GUARD(ctx)                  \
  DeviceGuard guard_((ctx)->device);     \
  if (guard_.status != INQB_OK) return guard_.status

template <typename T>
ProjView<T> proj_view(inqb_ctx* ctx) {
  ProjView<T> v{};
  const ProjTables& t = ctx->proj;
  v.nproj = t.nproj;
  v.L = t.L;
  v.max_plane_atoms = t.max_plane_atoms;
  v.max_tile_ent = t.max_tile_ent;
  v.max_tile_seg = t.max_tile_seg;
  v.pt_stride = t.pt_stride;
  v.ent_rec = t.d_ent_rec.as<EntRec<T>>();
  v.ent_rec_pt = t.d_ent_rec_pt.as<EntRec<T>>();
  v.pt_ptr = t.d_pt_ptr.as<int>();
  v.seg_ptr = t.d_seg_ptr.as<int>();
  v.seg_atom = t.d_seg_atom.as<int>();
  v.seg_ent = t.d_seg_ent.as<int>();
  v.ent_off = t.d_ent_off.as<int>();
  v.ent_atom = t.d_ent_atom.as<int>();
  v.seg_local = t.d_seg_local.as<int>();
  v.plane_ptr = t.d_plane_ptr.as<int>();
  v.plane_atom = t.d_plane_atom.as<int>();
  v.ent_beta = t.d_ent_beta.as<T>();
  v.ent_phase = t.d_ent_phase.ptr;
  v.scale = t.d_scale.as<double>();
  v.proj = ctx->d_projacc.as<double2>();
  v.pc_ptr = t.d_pc_ptr.as<int>();
  v.pc_pt = t.d_pc_pt.as<int>();
  v.pc_table = t.pc_chunks > 0 ? t.d_pc_table.ptr : nullptr;
  v.err = ctx->d_err.as<int>();
  v.proj_mode = ctx->proj_mode;
  v.slots = ctx->d_slots.as<double2>();
  v.aslot_ptr = t.d_aslot_ptr.as<int>();
  v.aslot = t.d_aslot.as<int>();
  return v;
}

int check_block(const inqb_ctx* ctx, const void* a, int M, long ld) {
  if (M <= 0) return fail(INQB_ERR_INVALID, "M must be positive");
  if (ld < M) return fail(INQB_ERR_INVALID, "ld must be >= M");
  if (!a) return fail(INQB_ERR_INVALID, "null orbital pointer");
  if (((uintptr_t)a) % 16 != 0) return fail(INQB_ERR_INVALID, "orbital pointer must be 16-byte aligned");
  (void)ctx;
  return INQB_OK;
}

int reserve(inqb_ctx* ctx, int M) {
  const int G = ctx->plan->G, Gt = ctx->plan->G_tile;
  const size_t padded = std::max((size_t)(M + G - 1) / G * G, (size_t)(M + Gt - 1) / Gt * Gt);
  INQB_TRY(ctx->d_tmp.ensure(padded * (size_t)ctx->N * ctx->elem_bytes()));
  if (ctx->proj.nproj > 0) INQB_TRY(ctx->d_projacc.ensure(sizeof(double2) * (size_t)ctx->proj.nproj * ctx->proj.L * M));
  return INQB_OK;
}

int update_phases(inqb_ctx* ctx, void* stream) {
  if (ctx->proj.nproj == 0 || ctx->proj.nent == 0) return INQB_OK;
  INQB_TRY(launch_phases(ctx->precision, ctx->proj.nent, ctx->proj.d_ent_relpos.as<float>(), ctx->kA_cov,
                         ctx->proj.d_ent_phase.ptr, ctx->proj.d_ent_rec.ptr, ctx->proj.d_ent_rec_pt.ptr,
                         ctx->proj.d_pt_pos.as<int>(), ctx->proj.d_adj_rec.ptr, ctx->proj.d_atom_pos.as<int>(),
                         stream));
  return launch_project_table(ctx->precision, ctx->proj.pc_chunks, ctx->proj.d_pc_relpos.as<float>(),
                              ctx->proj.d_pc_beta.as<double>(), ctx->kA_cov, ctx->proj.d_pc_table.ptr, stream);
}

int set_kA(inqb_ctx* ctx, const double kA[3], void* stream) {
  bool same = true;
  for (int d = 0; d < 3; d++) same = same && (ctx->kA_cov[d] == kA[d]);
  for (int d = 0; d < 3; d++) ctx->kA_cov[d] = kA[d];
  if (same && ctx->proj_phases_valid) return INQB_OK;
  INQB_TRY(update_phases(ctx, stream));
  ctx->proj_phases_valid = true;
  return INQB_OK;
}

// One H application: out = alpha * H in + beta * base.
int apply(inqb_ctx* ctx, int mode, const void* in, long ld_in, void* out, long ld_out, int M, const void* base,
          long ld_base, const double alpha[2], const double beta[2], void* stream, void* fourier_out = nullptr,
          BatchCellDesc* batch_cell = nullptr) {
  INQB_TRY(reserve(ctx, M));
  if (!ctx->proj_phases_valid) {
    INQB_TRY(update_phases(ctx, stream));
    ctx->proj_phases_valid = true;
  }
  LaunchArgs a;
  a.mode = mode;
  a.in = in;
  a.ld_in = ld_in;
  a.out = out;
  a.ld_out = ld_out;
  a.M = M;
  a.tmp = ctx->d_tmp.ptr;
  a.tw = ctx->d_tw.ptr;
  a.V = ctx->d_V.ptr;
  a.base = base;
  a.ld_base = ld_base;
  a.alpha[0] = alpha[0];
  a.alpha[1] = alpha[1];
  a.beta[0] = beta[0];
  a.beta[1] = beta[1];
  a.stream = stream;
  a.fourier_out = fourier_out;
  a.batch_cell = batch_cell;
  a.fourier_mask = ctx->fourier_mask;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) a.rlat[i][j] = ctx->cell.rlat[i][j];
  ctx->cell.cov_to_cart(ctx->kA_cov, a.kA_cart);
  const auto sched = ctx->schedules.find(M);
  if (sched != ctx->schedules.end()) {
    a.ysplit = sched->second[0];
    for (int k = 0; k < 3; k++) a.threads[k] = sched->second[1 + k];
  }
  // the fused projection's partial sums: one [4][M] slot per (plane, atom, half)
  if (mode == LaunchArgs::H && ctx->proj.nproj > 0 && ctx->proj_mode == INQB_PROJECTION_FUSED) {
    const int ys = a.ysplit > 0 ? a.ysplit : ctx->plan->ysplit;
    INQB_TRY(ctx->d_slots.ensure(sizeof(double2) * (size_t)ctx->proj.aslot.size() * ys * 4 * M));
  }
  if (ctx->timing_on && mode == LaunchArgs::H && !batch_cell && ctx->timing_count < ctx->timing_capacity) {
    for (int i = 0; i < 6; i++) a.events[i] = ctx->timing_events[6 * ctx->timing_count + i];
    ctx->timing_count++;
  }
  ProjView<double> v64;
  ProjView<float> v32;
  if (ctx->precision == INQB_FP64) {
    v64 = proj_view<double>(ctx);
    a.proj_view = &v64;
  } else {
    v32 = proj_view<float>(ctx);
    a.proj_view = &v32;
  }
  return ctx->plan->launch(a);
}

// One H application with the four pass events recorded (used by the autotuner).
int apply_events(inqb_ctx* ctx, const void* in, void* out, int M, const double alpha[2], const double beta[2],
                 void* stream, cudaEvent_t ev[6]) {
  INQB_TRY(reserve(ctx, M));
  if (!ctx->proj_phases_valid) {
    INQB_TRY(update_phases(ctx, stream));
    ctx->proj_phases_valid = true;
  }
  const bool on = ctx->timing_on;
  const int cap = ctx->timing_capacity, count = ctx->timing_count;
  std::vector<cudaEvent_t> saved;
  saved.swap(ctx->timing_events);
  ctx->timing_events.assign(ev, ev + 6);
  ctx->timing_on = true;
  ctx->timing_capacity = 1;
  ctx->timing_count = 0;
  const int st = apply(ctx, LaunchArgs::H, in, M, out, M, M, nullptr, 0, alpha, beta, stream);
  ctx->timing_events.swap(saved);
  ctx->timing_on = on;
  ctx->timing_capacity = cap;
  ctx->timing_count = count;
  return st;
}

// psi <- sum_{k <= order} (f H)^k / k! psi by Horner's rule:
// y = psi; for k = order..1: y = psi + (f/k) H y.  (exponential.hpp:21-34)
int exponential(inqb_ctx* ctx, void* psi, int M, long ld, double fre, double fim, int order, void* stream) {
  if (order < 1) return INQB_OK;
  INQB_TRY(ctx->d_work.ensure((size_t)ctx->N * M * ctx->elem_bytes()));
  void* y = ctx->d_work.ptr;
  const double one[2] = {1.0, 0.0};
  for (int k = order; k >= 1; k--) {
    const double alpha[2] = {fre / k, fim / k};
    const void* in = (k == order) ? psi : y;
    const long ldi = (k == order) ? ld : M;
    void* out = (k == 1) ? psi : y;
    const long ldo = (k == 1) ? ld : M;
    INQB_TRY(apply(ctx, LaunchArgs::H, in, ldi, out, ldo, M, psi, ld, alpha, one, stream));
  }
  return INQB_OK;
}

// [N][M] block copy between leading dimensions (device to device)
int copy_block(const void* src, long lds, void* dst, long ldd, int M, long N, size_t esz, void* stream) {
  INQB_CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)ldd * esz, src, (size_t)lds * esz, (size_t)M * esz, (size_t)N,
                                  cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return INQB_OK;
}

// Workspace of the density -> potential step, carved from ctx->d_pot.
struct PotWork {
  void* vh = nullptr;         // [N] complex, context precision (the Poisson field)
  double* rho_old = nullptr;  // [N]
  double* partial = nullptr;  // [kPotBlocks * 4]
  double* sums = nullptr;     // [8]: the four potential sums, then sum |drho|
};

int pot_work(inqb_ctx* ctx, PotWork& w) {
  const size_t N = (size_t)ctx->N;
  const size_t vh = N * ctx->elem_bytes();
  INQB_TRY(ctx->d_pot.ensure(vh + sizeof(double) * (N + (size_t)kPotBlocks * 4 + 8)));
  char* b = static_cast<char*>(ctx->d_pot.ptr);
  w.vh = b;
  w.rho_old = reinterpret_cast<double*>(b + vh);
  w.partial = w.rho_old + N;
  w.sums = w.partial + (size_t)kPotBlocks * 4;
  return INQB_OK;
}

// Workspace of the Broyden density mixer, carved from ctx->d_mix
struct MixWork {
  static constexpr int kRing = 4;  // mixers::broyden(4, 0.3, ...) in crank_nicolson.hpp:68
  double* df = nullptr;       // [kRing][N]
  double* dv = nullptr;       // [kRing][N]
  double* f_old = nullptr;    // [N]: the last vout - vin
  double* vin_old = nullptr;  // [N]
  double* fresh = nullptr;    // [N]: the density of the solved orbitals
  double* partial = nullptr;  // [kPotBlocks * kMaxDots]
  double* dots = nullptr;     // [kMaxDots + 1]: dot products, then the sum for the normalisation
};

int mix_work(inqb_ctx* ctx, MixWork& w) {
  const size_t N = (size_t)ctx->N;
  const size_t n = (2 * MixWork::kRing + 3) * N + (size_t)kPotBlocks * kMaxDots + kMaxDots + 1;
  INQB_TRY(ctx->d_mix.ensure(sizeof(double) * n));
  double* b = ctx->d_mix.as<double>();
  w.df = b;
  w.dv = w.df + MixWork::kRing * N;
  w.f_old = w.dv + MixWork::kRing * N;
  w.vin_old = w.f_old + N;
  w.fresh = w.vin_old + N;
  w.partial = w.fresh + N;
  w.dots = w.partial + (size_t)kPotBlocks * kMaxDots;
  return INQB_OK;
}

// nd dot products of device vectors, read back (synchronises the stream)
int device_dots(const DotList& d, int nd, long n, const MixWork& w, double* out, void* stream) {
  INQB_TRY(launch_dots(d, nd, n, w.partial, w.dots, stream));
  INQB_CUDA_TRY(cudaMemcpyAsync(out, w.dots, sizeof(double) * nd, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return INQB_OK;
}

// One call of mixers::broyden (broyden.hpp:107-160) on the density, vin = rho and
// vout = w.fresh, then observables::density::normalize(rho, nelec)
// (density.hpp:100-111).  The vectors stay on the device; the ring bookkeeping and
// the small solve are on the host (broyden_host.h).  Synchronises three times.
int broyden_mix_density(inqb_ctx* ctx, BroydenRing& ring, double* rho, const MixWork& w, double nelec,
                        void* stream) {
  const long N = ctx->N;
  const int pos = ring.begin();
  double* dfp = pos >= 0 ? w.df + (size_t)pos * N : nullptr;
  double* dvp = pos >= 0 ? w.dv + (size_t)pos * N : nullptr;
  INQB_TRY(launch_broyden_diff(rho, w.fresh, w.f_old, w.vin_old, dfp, dvp, N, stream));
  if (pos >= 0) {
    DotList d{};
    d.a[0] = dfp;
    d.b[0] = dfp;
    double g2 = 0.0;
    INQB_TRY(device_dots(d, 1, N, w, &g2, stream));
    const double gamma = std::max(1e-8, std::sqrt(g2));
    INQB_TRY(launch_scale2(dfp, dvp, 1.0 / gamma, N, stream));
    ring.filled(pos);
  }
  const int used = ring.used();
  BroydenCoef c{};
  if (used > 0) {
    DotList d{};
    int k = 0;
    for (int i = 0; i < used; i++)
      for (int j = i + 1; j < used; j++, k++) {
        d.a[k] = w.df + (size_t)i * N;
        d.b[k] = w.df + (size_t)j * N;
      }
    for (int i = 0; i < used; i++, k++) {
      d.a[k] = w.df + (size_t)i * N;
      d.b[k] = w.f_old;  // ff of this call
    }
    double dots[kMaxDots];
    INQB_TRY(device_dots(d, k, N, w, dots, stream));
    if (!broyden_coefficients(used, dots, c.c))
      return fail(INQB_ERR_NONFINITE, "Broyden mixing: the history system is not finite");
  }
  INQB_TRY(launch_broyden_update(rho, w.f_old, w.df, w.dv, N, used, c, ring.mix, w.partial, w.dots + kMaxDots,
                                 stream));
  double q = 0.0;
  INQB_CUDA_TRY(cudaMemcpyAsync(&q, w.dots + kMaxDots, sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  q *= ctx->dV;
  if (!(std::fabs(q) > 1e-16) || !std::isfinite(q))
    return fail(INQB_ERR_NONFINITE, "density normalisation: the mixed density integrates to zero");
  return launch_scale(rho, nelec / q, N, stream);
}

// update_hamiltonian on the device: V_H by the Poisson passes, then one pass for
// V = vion + V_H + v_xc and the four energy sums (w.sums[0..3], without dV).
int ks_potential_dev(inqb_ctx* ctx, const double* rho, const double* vion, int theory, const PotWork& w,
                     void* stream) {
  if (theory >= INQB_THEORY_HARTREE) {
    const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
    INQB_TRY(launch_pack_density(ctx->precision, rho, w.vh, ctx->N, stream));
    INQB_TRY(apply(ctx, LaunchArgs::POISSON, w.vh, 1, w.vh, 1, 1, nullptr, 0, one, zero, stream));
  }
  return launch_ks_potential(ctx->precision, rho, vion, theory >= INQB_THEORY_HARTREE ? w.vh : nullptr, theory,
                             ctx->N, ctx->d_V.ptr, w.partial, w.sums, stream);
}

// TD-MLWF workspace carved from ctx->d_mlwf
struct MlwfWork {
  double2* a = nullptr;      // [6][M][M]
  double2* u = nullptr;      // [M][M]
  double2* adiag = nullptr;  // [6][M]
  double* sums = nullptr;    // [3 M] band sums
  void* partial = nullptr;   // per-slab Gram partial sums
  int2* pairs = nullptr;     // [2 np - 1][np]
  double* delta = nullptr;   // [2 np - 1][np]
  double* change = nullptr;  // [1]
};

int mlwf_work(inqb_ctx* ctx, int M, bool with_gram, MlwfWork& w) {
  const size_t MM = (size_t)M * M, np = (size_t)(M + 1) / 2, steps = 2 * np - 1;
  const size_t partial_bytes = with_gram ? mlwf_partial_bytes(ctx->N, M) : 0;
  size_t off = 0;
  auto take = [&off](size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) / 256 * 256;
    return at;
  };
  const size_t oa = take(sizeof(double2) * 6 * MM), ou = take(sizeof(double2) * MM),
               od = take(sizeof(double2) * 6 * M), os = take(sizeof(double) * 3 * M),
               op = take(partial_bytes), opr = take(sizeof(int2) * steps * np),
               ode = take(sizeof(double) * steps * np), oc = take(sizeof(double));
  INQB_TRY(ctx->d_mlwf.ensure(off));
  char* b = static_cast<char*>(ctx->d_mlwf.ptr);
  w.a = reinterpret_cast<double2*>(b + oa);
  w.u = reinterpret_cast<double2*>(b + ou);
  w.adiag = reinterpret_cast<double2*>(b + od);
  w.sums = reinterpret_cast<double*>(b + os);
  w.partial = b + op;
  w.pairs = reinterpret_cast<int2*>(b + opr);
  w.delta = reinterpret_cast<double*>(b + ode);
  w.change = reinterpret_cast<double*>(b + oc);
  return INQB_OK;
}

// One JADE sweep (2 np - 1 rotation steps and the trace-change sum) as a CUDA graph:
// captured once per call on a private stream, launched once per sweep (the sweep's
// pair schedule is copied to the same buffer before each launch).
struct SweepGraph {
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int capture(int M, double2* a, double2* u, const MlwfWork& w, int np, int steps) {
    INQB_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    INQB_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int rc = INQB_OK;
    for (int s = 0; s < steps && rc == INQB_OK; s++)
      rc = launch_jade_step(a, u, M, w.pairs + (size_t)s * np, np, w.delta + (size_t)s * np, cap);
    if (rc == INQB_OK) rc = launch_jade_change(w.delta, steps, np, w.change, cap);
    const cudaError_t e = cudaStreamEndCapture(cap, &graph);
    if (rc != INQB_OK) return rc;
    if (e != cudaSuccess) return fail(INQB_ERR_CUDA, std::string("JADE sweep capture: ") + cudaGetErrorString(e));
    INQB_CUDA_TRY(cudaGraphInstantiate(&exec, graph, 0));
    return INQB_OK;
  }
  ~SweepGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cap) cudaStreamDestroy(cap);
  }
};

// jade_complex on device arrays a [6][M][M] (rotated in place), u, adiag.  The pair
// schedule of each sweep is made on the host (the reference's round-robin shift) and
// copied before the sweep; the sweep's trace change is read back once per sweep.
int jade_dev(int M, double2* a, double2* u, double2* adiag, int maxsweep, double tol, const MlwfWork& w, int* sweeps,
             void* stream) {
  const int np = (M + 1) / 2, steps = 2 * np - 1;
  cudaStream_t st = (cudaStream_t)stream;
  INQB_TRY(launch_identity(u, M, stream));
  std::vector<int> top(np), bot(np);
  for (int i = 0; i < np; i++) {
    top[i] = i;
    bot[np - i - 1] = np + i;
  }
  std::vector<int2> sched((size_t)steps * np);
  SweepGraph graph;
  int nsweep = 0;
  for (;;) {
    ++nsweep;
    for (int s = 0; s < steps; s++) {
      for (int i = 0; i < np; i++) sched[(size_t)s * np + i] = make_int2(top[i], bot[i]);
      // the reference's shift: bot[j] <- bot[j+1], top[j+1] <- top[j] as one parallel
      // move, then the ends, then one swap (jade_complex.hpp:296-322)
      const int top_back = top[np - 1], bot_front = bot[0];
      std::vector<int> t2 = top, b2 = bot;
      for (int j = 0; j + 1 < np; j++) {
        b2[j] = bot[j + 1];
        t2[j + 1] = top[j];
      }
      b2[np - 1] = top_back;
      t2[0] = bot_front;
      if (np > 1)
        std::swap(t2[0], t2[1]);
      else
        std::swap(t2[0], b2[0]);
      top.swap(t2);
      bot.swap(b2);
    }
    INQB_CUDA_TRY(cudaMemcpyAsync(w.pairs, sched.data(), sizeof(int2) * sched.size(), cudaMemcpyHostToDevice, st));
    if (!graph.exec) INQB_TRY(graph.capture(M, a, u, w, np, steps));
    INQB_CUDA_TRY(cudaGraphLaunch(graph.exec, st));
    double change = 0.0;
    INQB_CUDA_TRY(cudaMemcpyAsync(&change, w.change, sizeof(double), cudaMemcpyDeviceToHost, st));
    INQB_CUDA_TRY(cudaStreamSynchronize(st));
    if (!std::isfinite(change)) return fail(INQB_ERR_NONFINITE, "TD-MLWF matrices are not finite");
    if (std::fabs(change) < tol || nsweep >= maxsweep) break;
  }
  INQB_TRY(launch_jade_adiag(a, u, M, adiag, stream));
  if (sweeps) *sweeps = nsweep;
  return INQB_OK;
}

// centres and spreads from adiag (tdmlwf_trans::center / spread2, tdmlwf_trans.hpp:196-312)
void mlwf_centres(const inqb_ctx* ctx, int M, const double2* adiag, double* centres, double* spreads) {
  const double (*L)[3] = ctx->cell.lat;
  const double (*B)[3] = ctx->cell.rlat;
  for (int i = 0; i < M; i++) {
    double t[3], s2 = 0.0;
    for (int d = 0; d < 3; d++) {
      const double2 c = adiag[(size_t)(2 * d) * M + i], s = adiag[(size_t)(2 * d + 1) * M + i];
      t[d] = std::atan2(s.x, c.x) / (2.0 * M_PI);
      const double b2 = B[d][0] * B[d][0] + B[d][1] * B[d][1] + B[d][2] * B[d][2];
      s2 += (1.0 - (c.x * c.x + c.y * c.y) - (s.x * s.x + s.y * s.y)) / b2;
    }
    if (centres)
      for (int r = 0; r < 3; r++) centres[3 * i + r] = t[0] * L[r][0] + t[1] * L[r][1] + t[2] * L[r][2];
    if (spreads) spreads[i] = std::sqrt(s2);
  }
}

void energies_from_sums(const inqb_ctx* ctx, const double s[4], double en[4]) {
  en[0] = ctx->dV * s[0];
  en[1] = 0.5 * ctx->dV * s[1];
  en[2] = ctx->dV * s[2];
  en[3] = ctx->dV * s[3];
}

}  // namespace
}  // namespace inqb

// A set of independent cells whose H applications run as one CUDA graph: one
// branch per cell (its three fused kernels), all branches concurrent.
struct inqb_batch {
  std::vector<inqb_ctx*> cells;
  int device = 0;
  std::vector<cudaStream_t> streams;  // capture streams: [0] origin, [1..n] one per cell
  std::vector<cudaEvent_t> events;    // [0] fork, [1..n] joins
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // arguments the instantiated graph or the persistent plan was built with
  std::vector<const void*> psis;
  std::vector<void*> hpsis;
  std::vector<int> Ms, lds;
  // the persistent launch (batch.h)
  int mode = INQB_BATCH_AUTO;
  int tuned = INQB_BATCH_GRAPH;  // the form AUTO runs: GRAPH until inqb_batch_autotune picks
  bool ready = false;        // a graph or a persistent plan matches the recorded arguments
  bool persistent = false;   // the recorded arguments run as one persistent launch
  int precision = INQB_FP64;
  int nitems = 0, ncounters = 0, ctas = 0;
  size_t smem = 0;
  double wait_s = 2.0;
  int unreachable = 0;       // test hook: one stage-C item waits for a count no item reaches
  std::vector<unsigned char> cells_blob;  // the cells' kernel descriptors (kernel parameters)
  size_t cell_bytes = 0;
  inqb::DevBuf d_items, d_ctr, d_err;
};

namespace inqb {
namespace {

void batch_release_graph(inqb_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// The work list and device descriptors of one persistent launch for these arguments;
// INQB_ERR_UNSUPPORTED when a cell cannot run in it (grid not compiled into the
// kernel, projection kernel form, cells of both precisions).
int batch_build_persistent(inqb_batch* b, const void* const* psis, void* const* hpsis, const int* Ms,
                           const int* lds) {
  const int n = (int)b->cells.size();
  const int prec = b->cells[0]->precision;
  if (n > kMaxBatchCells) return fail(INQB_ERR_UNSUPPORTED, "more cells than one persistent launch takes");
  std::vector<BatchCellDesc> descs(n);
  size_t smem = 0;
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  for (int i = 0; i < n; i++) {
    if (b->cells[i]->precision != prec) return fail(INQB_ERR_UNSUPPORTED, "cells of both precisions in one batch");
    INQB_TRY(apply(b->cells[i], LaunchArgs::H, psis[i], lds[i], hpsis[i], lds[i], Ms[i], nullptr, 0, one, zero,
                   nullptr, nullptr, &descs[i]));
    smem = std::max(smem, descs[i].smem);
  }
  int per_sm = 0, sms = 0;
  INQB_TRY(batch_ctas_per_sm(prec, smem, &per_sm));
  INQB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  std::vector<BatchItem> items;
  int nctr = 0;
  INQB_TRY(build_batch_items(descs, per_sm * sms, items, nctr));
  if (b->unreachable)
    for (auto& it : items)
      if (it.stage == kStageC) {
        it.target += 1;
        break;
      }
  const size_t csz = descs[0].bytes.size();
  b->cell_bytes = csz;
  b->cells_blob.assign(csz * n, 0);
  for (int i = 0; i < n; i++) memcpy(b->cells_blob.data() + (size_t)i * csz, descs[i].bytes.data(), csz);
  INQB_TRY(b->d_items.ensure(sizeof(BatchItem) * items.size()));
  INQB_TRY(b->d_ctr.ensure(sizeof(unsigned) * (size_t)nctr));
  INQB_CUDA_TRY(cudaMemcpy(b->d_items.ptr, items.data(), sizeof(BatchItem) * items.size(), cudaMemcpyHostToDevice));
  b->precision = prec;
  b->nitems = (int)items.size();
  b->ncounters = nctr;
  b->smem = smem;
  b->ctas = std::min(per_sm * sms, b->nitems);
  return INQB_OK;
}

int batch_capture(inqb_batch* b, const void* const* psis, void* const* hpsis, const int* Ms, const int* lds) {
  const int n = (int)b->cells.size();
  cudaStream_t s0 = b->streams[0];
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  INQB_CUDA_TRY(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
  int st = INQB_OK;
  if (cudaEventRecord(b->events[0], s0) != cudaSuccess) st = fail(INQB_ERR_CUDA, "fork event");
  for (int i = 0; i < n && st == INQB_OK; i++) {
    cudaStream_t si = b->streams[i + 1];
    if (cudaStreamWaitEvent(si, b->events[0], 0) != cudaSuccess) {
      st = fail(INQB_ERR_CUDA, "fork wait");
      break;
    }
    st = apply(b->cells[i], LaunchArgs::H, psis[i], lds[i], hpsis[i], lds[i], Ms[i], nullptr, 0, one, zero, si);
    if (st == INQB_OK && cudaEventRecord(b->events[i + 1], si) != cudaSuccess) st = fail(INQB_ERR_CUDA, "join event");
    if (st == INQB_OK && cudaStreamWaitEvent(s0, b->events[i + 1], 0) != cudaSuccess) st = fail(INQB_ERR_CUDA, "join");
  }
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(s0, &g);
  if (st != INQB_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (ec != cudaSuccess) return fail(INQB_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(ec));
  batch_release_graph(b);
  b->graph = g;
  INQB_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return INQB_OK;
}

}  // namespace
}  // namespace inqb

using namespace inqb;

extern "C" {

int inqb_version(void) { return 1; }

const char* inqb_status_string(int status) {
  switch (status) {
    case INQB_OK: return "ok";
    case INQB_ERR_INVALID: return "invalid argument";
    case INQB_ERR_UNSUPPORTED: return "unsupported configuration";
    case INQB_ERR_CUDA: return "CUDA error";
    case INQB_ERR_NOMEM: return "out of device memory";
    case INQB_ERR_NONFINITE: return "non-finite input";
    case INQB_ERR_NOT_POSITIVE_DEFINITE: return "matrix not positive definite";
    case INQB_ERR_TIMEOUT: return "device wait timed out";
    case INQB_ERR_IO: return "checkpoint file missing, short or unwritable";
    default: return "unknown status";
  }
}

const char* inqb_last_error(void) { return inqb::last_error(); }

int inqb_grid_supported(int nx, int ny, int nz, int precision) {
  return find_plan(nx, ny, nz, precision) != nullptr ? 1 : 0;
}

int inqb_ctx_create(const double lattice[9], int nx, int ny, int nz, int precision, int device, inqb_ctx** out) {
  if (!out || !lattice) return fail(INQB_ERR_INVALID, "null argument");
  *out = nullptr;
  if (precision != INQB_FP64 && precision != INQB_MIXED) return fail(INQB_ERR_INVALID, "unknown precision");
  const Plan* plan = find_plan(nx, ny, nz, precision);
  if (!plan)
    return fail(INQB_ERR_UNSUPPORTED, "no kernels compiled for grid " + std::to_string(nx) + "x" +
                                          std::to_string(ny) + "x" + std::to_string(nz));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(INQB_ERR_CUDA, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(INQB_ERR_INVALID, "device index out of range");
  DeviceGuard guard(device);
  if (guard.status != INQB_OK) return guard.status;

  auto* ctx = new inqb_ctx();
  ctx->device = device;
  ctx->precision = precision;
  ctx->nr[0] = nx;
  ctx->nr[1] = ny;
  ctx->nr[2] = nz;
  ctx->N = (long)nx * ny * nz;
  ctx->cell.init(lattice);
  if (!(ctx->cell.volume > 1e-10)) {
    delete ctx;
    return fail(INQB_ERR_INVALID, "lattice volume is not positive");
  }
  ctx->dV = ctx->cell.volume / (double)ctx->N;
  ctx->plan = plan;

  // twiddles x | y | z in context precision
  std::vector<double> tw;
  for (int d = 0; d < 3; d++) {
    int n1, n2;
    split_of(ctx->nr[d], &n1, &n2);
    std::vector<double> re, im;
    twiddle_table(ctx->nr[d], n1, n2, re, im);
    for (int i = 0; i < ctx->nr[d]; i++) {
      tw.push_back(re[i]);
      tw.push_back(im[i]);
    }
  }
  int st = INQB_OK;
  if (precision == INQB_FP64) {
    st = ctx->d_tw.ensure(sizeof(double) * tw.size());
    if (st == INQB_OK && cudaMemcpy(ctx->d_tw.ptr, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      st = fail(INQB_ERR_CUDA, "twiddle upload failed");
  } else {
    std::vector<float> twf(tw.begin(), tw.end());
    st = ctx->d_tw.ensure(sizeof(float) * twf.size());
    if (st == INQB_OK && cudaMemcpy(ctx->d_tw.ptr, twf.data(), sizeof(float) * twf.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      st = fail(INQB_ERR_CUDA, "twiddle upload failed");
  }
  if (st == INQB_OK) {
    ctx->V_host.assign(ctx->N, 0.0);
    st = ctx->d_V.ensure(ctx->N * (precision == INQB_FP64 ? sizeof(double) : sizeof(float)));
    if (st == INQB_OK && cudaMemset(ctx->d_V.ptr, 0, ctx->d_V.bytes) != cudaSuccess)
      st = fail(INQB_ERR_CUDA, "potential init failed");
  }
  if (st == INQB_OK) {
    st = ctx->d_err.ensure(sizeof(int));
    if (st == INQB_OK && cudaMemset(ctx->d_err.ptr, 0, sizeof(int)) != cudaSuccess)
      st = fail(INQB_ERR_CUDA, "error word init failed");
  }

  if (st != INQB_OK) {
    delete ctx;
    return st;
  }
  *out = ctx;
  return INQB_OK;
}

int inqb_ctx_clone(const inqb_ctx* src, inqb_ctx** out) {
  if (!src || !out) return fail(INQB_ERR_INVALID, "null argument");
  *out = nullptr;
  double lat[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) lat[3 * i + j] = src->cell.lat[i][j];
  inqb_ctx* c = nullptr;
  INQB_TRY(inqb_ctx_create(lat, src->nr[0], src->nr[1], src->nr[2], src->precision, src->device, &c));
  auto undo = [&c](int st) {
    inqb_ctx_destroy(c);
    return st;
  };
  DeviceGuard guard(src->device);
  if (guard.status != INQB_OK) return undo(guard.status);
  c->V_host = src->V_host;
  if (cudaMemcpy(c->d_V.ptr, src->d_V.ptr, src->d_V.bytes, cudaMemcpyDeviceToDevice) != cudaSuccess)
    return undo(fail(INQB_ERR_CUDA, "potential copy failed"));
  for (int d = 0; d < 3; d++) c->kA_cov[d] = src->kA_cov[d];
  c->fourier_mask = src->fourier_mask;
  c->proj_mode = src->proj_mode;
  c->schedules = src->schedules;
  const auto& ps = src->proj_src;
  if (ps.nproj > 0) {
    const int st = inqb_set_projectors(c, ps.nproj, ps.L, ps.smax, ps.counts.data(), ps.coords.data(),
                                       ps.relpos.data(), ps.beta.data(), ps.coeff.data());
    if (st != INQB_OK) return undo(st);
  }
  *out = c;
  return INQB_OK;
}

int inqb_ctx_destroy(inqb_ctx* ctx) {
  if (!ctx) return INQB_OK;
  DeviceGuard guard(ctx->device);
  cudaDeviceSynchronize();
  for (cudaEvent_t e : ctx->timing_events) cudaEventDestroy(e);
  for (cudaStream_t s : ctx->host_streams)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : ctx->host_events)
    if (e) cudaEventDestroy(e);
  delete ctx;
  return INQB_OK;
}

int inqb_timing_start(inqb_ctx* ctx, int max_applies) {
  INQB_CHECK_CTX(ctx);
  INQB_GUARD(ctx);
  if (max_applies <= 0) return fail(INQB_ERR_INVALID, "max_applies must be positive");
  while ((int)ctx->timing_events.size() < 6 * max_applies) {
    cudaEvent_t e;
    INQB_CUDA_TRY(cudaEventCreate(&e));
    ctx->timing_events.push_back(e);
  }
  ctx->timing_capacity = max_applies;
  ctx->timing_count = 0;
  ctx->timing_on = true;
  return INQB_OK;
}

int inqb_set_projection_mode(inqb_ctx* ctx, int mode) {
  INQB_CHECK_CTX(ctx);
  if (mode != INQB_PROJECTION_FUSED && mode != INQB_PROJECTION_KERNEL)
    return fail(INQB_ERR_INVALID, "unknown projection mode");
  ctx->proj_mode = mode;
  return INQB_OK;
}

int inqb_device_status(inqb_ctx* ctx, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_GUARD(ctx);
  cudaStream_t st = (cudaStream_t)stream;
  int word = 0;
  INQB_CUDA_TRY(cudaMemcpyAsync(&word, ctx->d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  if (word == 0) return INQB_OK;
  INQB_CUDA_TRY(cudaMemsetAsync(ctx->d_err.ptr, 0, sizeof(int), st));
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  return fail(INQB_ERR_TIMEOUT, "a device-side wait of a kernel gave up (its results are not valid)");
}

int inqb_timing_passes(inqb_ctx* ctx, double ms[4], int* napplies) {
  INQB_CHECK_CTX(ctx);
  INQB_GUARD(ctx);
  if (!ms || !napplies) return fail(INQB_ERR_INVALID, "null output");
  ctx->timing_on = false;
  for (int k = 0; k < 4; k++) ms[k] = 0.0;
  *napplies = ctx->timing_count;
  for (int i = 0; i < ctx->timing_count; i++) {
    const cudaEvent_t* e = &ctx->timing_events[6 * i];
    INQB_CUDA_TRY(cudaEventSynchronize(e[5]));
    INQB_CUDA_TRY(cudaEventSynchronize(e[1]));
    // projection: start -> its end (its own stream when concurrent); passes: their events
    const int from[4] = {0, 2, 3, 4}, to[4] = {1, 3, 4, 5};
    for (int k = 0; k < 4; k++) {
      float t = 0.f;
      INQB_CUDA_TRY(cudaEventElapsedTime(&t, e[from[k]], e[to[k]]));
      ms[k] += t;
    }
  }
  ctx->timing_count = 0;
  return INQB_OK;
}

int inqb_timing_stop(inqb_ctx* ctx, double ms_per_pass[3], int* napplies) {
  INQB_CHECK_CTX(ctx);
  INQB_GUARD(ctx);
  if (!ms_per_pass || !napplies) return fail(INQB_ERR_INVALID, "null output");
  ctx->timing_on = false;
  for (int k = 0; k < 3; k++) ms_per_pass[k] = 0.0;
  *napplies = ctx->timing_count;
  for (int i = 0; i < ctx->timing_count; i++) {
    const cudaEvent_t* e = &ctx->timing_events[6 * i];
    INQB_CUDA_TRY(cudaEventSynchronize(e[5]));
    // first pass from the start (it includes a projection kernel run before it), then
    // the second and third passes
    const int from[3] = {0, 3, 4}, to[3] = {3, 4, 5};
    for (int k = 0; k < 3; k++) {
      float t = 0.f;
      INQB_CUDA_TRY(cudaEventElapsedTime(&t, e[from[k]], e[to[k]]));
      ms_per_pass[k] += t;
    }
  }
  ctx->timing_count = 0;
  return INQB_OK;
}

int inqb_ctx_reserve(inqb_ctx* ctx, int M) {
  INQB_CHECK_CTX(ctx);
  INQB_GUARD(ctx);
  if (M <= 0) return fail(INQB_ERR_INVALID, "M must be positive");
  INQB_TRY(reserve(ctx, M));
  INQB_TRY(ctx->d_work.ensure((size_t)ctx->N * M * ctx->elem_bytes()));
  return INQB_OK;
}

double inqb_volume_element(const inqb_ctx* ctx) { return ctx ? ctx->dV : 0.0; }

int inqb_cart_to_cov(const inqb_ctx* ctx, const double cart[3], double cov[3]) {
  INQB_CHECK_CTX(ctx);
  if (!cart || !cov) return fail(INQB_ERR_INVALID, "null vector");
  ctx->cell.cart_to_cov(cart, cov);
  return INQB_OK;
}

int inqb_set_local_potential(inqb_ctx* ctx, const double* V) {
  INQB_CHECK_CTX(ctx);
  if (!V) return fail(INQB_ERR_INVALID, "null potential");
  INQB_GUARD(ctx);
  for (long p = 0; p < ctx->N; p++)
    if (!std::isfinite(V[p])) return fail(INQB_ERR_NONFINITE, "potential has a non-finite value");
  ctx->V_host.assign(V, V + ctx->N);
  if (ctx->precision == INQB_FP64) {
    INQB_CUDA_TRY(cudaMemcpy(ctx->d_V.ptr, V, sizeof(double) * ctx->N, cudaMemcpyHostToDevice));
  } else {
    std::vector<float> vf(V, V + ctx->N);
    INQB_CUDA_TRY(cudaMemcpy(ctx->d_V.ptr, vf.data(), sizeof(float) * ctx->N, cudaMemcpyHostToDevice));
  }
  return INQB_OK;
}

int inqb_set_vector_potential(inqb_ctx* ctx, const double kA_cov[3]) {
  INQB_CHECK_CTX(ctx);
  if (!kA_cov) return fail(INQB_ERR_INVALID, "null vector");
  for (int d = 0; d < 3; d++)
    if (!std::isfinite(kA_cov[d])) return fail(INQB_ERR_NONFINITE, "vector potential is not finite");
  INQB_GUARD(ctx);
  INQB_TRY(set_kA(ctx, kA_cov, nullptr));
  INQB_CUDA_TRY(cudaStreamSynchronize(nullptr));
  return INQB_OK;
}

int inqb_set_fourier_sphere_mask(inqb_ctx* ctx, int enable) {
  INQB_CHECK_CTX(ctx);
  ctx->fourier_mask = enable ? 1 : 0;
  return INQB_OK;
}

int inqb_sphere_size(const double lattice[9], const int nr[3], const double center[3], double radius, int* npts) {
  if (!lattice || !nr || !center || !npts || !(radius >= 0.0)) return fail(INQB_ERR_INVALID, "bad sphere arguments");
  if (nr[0] <= 0 || nr[1] <= 0 || nr[2] <= 0) return fail(INQB_ERR_INVALID, "grid sizes must be positive");
  CellGeom cell;
  cell.init(lattice);
  return sphere_points(cell, nr, center, radius, 0, nullptr, nullptr, nullptr, npts);
}

int inqb_sphere_points(const double lattice[9], const int nr[3], const double center[3], double radius, int npts,
                       int* coords, float* distance, float* relpos) {
  if (!lattice || !nr || !center || !coords || !distance || !relpos || !(radius >= 0.0))
    return fail(INQB_ERR_INVALID, "bad sphere arguments");
  if (nr[0] <= 0 || nr[1] <= 0 || nr[2] <= 0) return fail(INQB_ERR_INVALID, "grid sizes must be positive");
  CellGeom cell;
  cell.init(lattice);
  return sphere_points(cell, nr, center, radius, npts, coords, distance, relpos, nullptr);
}

int inqb_gaussian_kb_beta(const double lattice[9], int npts, const float* distance, const float* relpos, double sigma,
                          double* beta) {
  if (!lattice || npts < 0 || (npts > 0 && (!distance || !relpos || !beta)))
    return fail(INQB_ERR_INVALID, "bad arguments");
  CellGeom cell;
  cell.init(lattice);
  return gaussian_kb_beta(cell, npts, distance, relpos, sigma, beta);
}

int inqb_set_projectors(inqb_ctx* ctx, int nproj, int L, int smax, const int* counts, const int* coords,
                        const float* relpos, const double* beta, const double* coeff) {
  INQB_CHECK_CTX(ctx);
  INQB_GUARD(ctx);
  if (nproj < 0 || smax < 0 || L < 0) return fail(INQB_ERR_INVALID, "negative size");
  if (nproj > 0 && (L == 0 || L > kMaxL))
    return fail(INQB_ERR_UNSUPPORTED, "projectors per atom must be 1.." + std::to_string(kMaxL));
  if (nproj > 0 && (!counts || !coords || !relpos || !beta || !coeff)) return fail(INQB_ERR_INVALID, "null table");
  ProjTables fresh;
  if (nproj > 0) {
    INQB_TRY(build_proj_tables(*ctx, nproj, L, smax, counts, coords, relpos, beta, coeff, fresh));
    for (double b : fresh.ent_beta)
      if (!std::isfinite(b)) return fail(INQB_ERR_NONFINITE, "projector table has a non-finite value");
    INQB_TRY(upload_proj_tables(*ctx, fresh));
  }
  INQB_CUDA_TRY(cudaDeviceSynchronize());
  ctx->proj = std::move(fresh);
  {
    auto& src = ctx->proj_src;
    src.nproj = nproj;
    src.L = L;
    src.smax = smax;
    const size_t ns = (size_t)nproj * smax;
    src.counts.assign(counts, counts + (nproj > 0 ? nproj : 0));
    src.coords.assign(coords, coords + (nproj > 0 ? 3 * ns : 0));
    src.relpos.assign(relpos, relpos + (nproj > 0 ? 3 * ns : 0));
    src.beta.assign(beta, beta + (nproj > 0 ? (size_t)L * ns : 0));
    src.coeff.assign(coeff, coeff + (nproj > 0 ? (size_t)nproj * L : 0));
  }
  ctx->proj_phases_valid = false;
  INQB_TRY(update_phases(ctx, nullptr));
  INQB_CUDA_TRY(cudaStreamSynchronize(nullptr));
  ctx->proj_phases_valid = true;
  return INQB_OK;
}

int inqb_apply_h(inqb_ctx* ctx, const void* psi, void* hpsi, int M, int ld, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  INQB_TRY(check_block(ctx, hpsi, M, ld));
  INQB_GUARD(ctx);
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  return apply(ctx, LaunchArgs::H, psi, ld, hpsi, ld, M, nullptr, 0, one, zero, stream);
}

int inqb_apply_h_host(inqb_ctx* ctx, const void* psi_host, void* hpsi_host, int M) {
  INQB_CHECK_CTX(ctx);
  if (!psi_host || !hpsi_host || M <= 0) return fail(INQB_ERR_INVALID, "bad host buffers");
  INQB_GUARD(ctx);
  const size_t esz = ctx->elem_bytes();
  const size_t bytes = (size_t)ctx->N * M * esz;
  INQB_TRY(ctx->d_work2.ensure(bytes));
  INQB_TRY(ctx->d_work.ensure(bytes));
  // Orbital chunks of at least 32 (rows of >= 256 bytes, up to 4 chunks): the copy-in
  // of chunk c + 1, the H apply of chunk c and the copy-out of chunk c - 1 overlap on
  // three streams, with pitched 2-D copies between the [N][M] host blocks and
  // [N][chunk] device blocks.
  const int G = ctx->plan->G_tile;
  int C = std::max(32, (M + 3) / 4);
  C = (C + G - 1) / G * G;
  const int nchunks = (M + C - 1) / C;
  for (int k = 0; k < 3; k++)
    if (!ctx->host_streams[k]) INQB_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->host_streams[k], cudaStreamNonBlocking));
  for (cudaEvent_t& e : ctx->host_events)
    if (!e) INQB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaStream_t s_in = ctx->host_streams[0], s_comp = ctx->host_streams[1], s_out = ctx->host_streams[2];
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  char* din = static_cast<char*>(ctx->d_work2.ptr);
  char* dout = static_cast<char*>(ctx->d_work.ptr);
  const char* hin = static_cast<const char*>(psi_host);
  char* hout = static_cast<char*>(hpsi_host);
  for (int c = 0; c < nchunks; c++) {
    const int m0 = c * C, mc = std::min(C, M - m0);
    char* di = din + (size_t)ctx->N * m0 * esz;
    char* dq = dout + (size_t)ctx->N * m0 * esz;
    cudaEvent_t ev_in = ctx->host_events[2 * (c % 4)], ev_done = ctx->host_events[2 * (c % 4) + 1];
    INQB_CUDA_TRY(cudaMemcpy2DAsync(di, mc * esz, hin + m0 * esz, (size_t)M * esz, mc * esz, ctx->N,
                                    cudaMemcpyHostToDevice, s_in));
    INQB_CUDA_TRY(cudaEventRecord(ev_in, s_in));
    INQB_CUDA_TRY(cudaStreamWaitEvent(s_comp, ev_in, 0));
    INQB_TRY(apply(ctx, LaunchArgs::H, di, mc, dq, mc, mc, nullptr, 0, one, zero, s_comp));
    INQB_CUDA_TRY(cudaEventRecord(ev_done, s_comp));
    INQB_CUDA_TRY(cudaStreamWaitEvent(s_out, ev_done, 0));
    INQB_CUDA_TRY(cudaMemcpy2DAsync(hout + m0 * esz, (size_t)M * esz, dq, mc * esz, mc * esz, ctx->N,
                                    cudaMemcpyDeviceToHost, s_out));
  }
  INQB_CUDA_TRY(cudaStreamSynchronize(s_out));
  INQB_CUDA_TRY(cudaStreamSynchronize(s_comp));
  INQB_CUDA_TRY(cudaStreamSynchronize(s_in));
  return INQB_OK;
}

int inqb_fft_forward(inqb_ctx* ctx, const void* in, void* out, int M, int ld, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, in, M, ld));
  INQB_TRY(check_block(ctx, out, M, ld));
  INQB_GUARD(ctx);
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  return apply(ctx, LaunchArgs::FFT_FWD, in, ld, out, ld, M, nullptr, 0, one, zero, stream);
}

int inqb_fft_backward(inqb_ctx* ctx, const void* in, void* out, int M, int ld, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, in, M, ld));
  INQB_TRY(check_block(ctx, out, M, ld));
  INQB_GUARD(ctx);
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  return apply(ctx, LaunchArgs::FFT_BWD, in, ld, out, ld, M, nullptr, 0, one, zero, stream);
}

int inqb_exponential(inqb_ctx* ctx, void* psi, int M, int ld, double f_re, double f_im, int order, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (order < 0 || order > 64) return fail(INQB_ERR_INVALID, "order out of range");
  INQB_GUARD(ctx);
  return exponential(ctx, psi, M, ld, f_re, f_im, order, stream);
}

int inqb_etrs_step(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                   const double kA_tdt_cov[3], void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!kA_t_cov || !kA_tdt_cov || !std::isfinite(dt)) return fail(INQB_ERR_INVALID, "bad step arguments");
  INQB_GUARD(ctx);
  INQB_TRY(set_kA(ctx, kA_t_cov, stream));
  INQB_TRY(exponential(ctx, psi, M, ld, 0.0, dt / 2.0, 4, stream));
  INQB_TRY(set_kA(ctx, kA_tdt_cov, stream));
  INQB_TRY(exponential(ctx, psi, M, ld, 0.0, dt / 2.0, 4, stream));
  return INQB_OK;
}

int inqb_kick(inqb_ctx* ctx, void* psi, int M, int ld, const double kick_cart[3], void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!kick_cart) return fail(INQB_ERR_INVALID, "null kick");
  for (int d = 0; d < 3; d++)
    if (!std::isfinite(kick_cart[d])) return fail(INQB_ERR_NONFINITE, "kick is not finite");
  INQB_GUARD(ctx);
  return launch_phase_kick(ctx->precision, *ctx, psi, ld, M, kick_cart, stream);
}

int inqb_poisson(inqb_ctx* ctx, const void* in, void* out, int M, int ld, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, in, M, ld));
  INQB_TRY(check_block(ctx, out, M, ld));
  INQB_GUARD(ctx);
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  return apply(ctx, LaunchArgs::POISSON, in, ld, out, ld, M, nullptr, 0, one, zero, stream);
}

int inqb_ks_potential(inqb_ctx* ctx, const double* rho, const double* vion, int theory, double energies[4],
                      void* stream) {
  INQB_CHECK_CTX(ctx);
  if (!rho) return fail(INQB_ERR_INVALID, "null density");
  if (theory < INQB_THEORY_NONE || theory > INQB_THEORY_LDA) return fail(INQB_ERR_INVALID, "unknown theory");
  INQB_GUARD(ctx);
  PotWork w;
  INQB_TRY(pot_work(ctx, w));
  INQB_TRY(ks_potential_dev(ctx, rho, vion, theory, w, stream));
  if (energies) {
    double s[4];
    INQB_CUDA_TRY(cudaMemcpyAsync(s, w.sums, sizeof(s), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    energies_from_sums(ctx, s, energies);
  }
  return INQB_OK;
}

int inqb_set_density_reduce(inqb_ctx* ctx, inqb_density_reduce_fn fn, void* user) {
  INQB_CHECK_CTX(ctx);
  ctx->density_reduce = fn;
  ctx->density_reduce_user = fn ? user : nullptr;
  return INQB_OK;
}

namespace inqb {
namespace {
// the density of this rank's orbitals, then (when set) the sum over the ranks
int sharded_density(inqb_ctx* ctx, const void* psi, long ld, int M, const double* occ, double* rho, void* stream) {
  INQB_TRY(launch_density(ctx->precision, psi, ld, M, ctx->N, occ, rho, stream));
  if (!ctx->density_reduce) return INQB_OK;
  INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  if (ctx->density_reduce(rho, ctx->N, ctx->density_reduce_user) != 0)
    return fail(INQB_ERR_INVALID, "the density reduction callback failed");
  return INQB_OK;
}
}  // namespace
}  // namespace inqb

int inqb_etrs_scf_step(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                       const double kA_tdt_cov[3], const double* occ, double* rho, const double* vion, int theory,
                       int nscf, double threshold, int* iters, double energies[4], void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!kA_t_cov || !kA_tdt_cov || !occ || !rho || !std::isfinite(dt) || nscf < 1 || !(threshold >= 0.0))
    return fail(INQB_ERR_INVALID, "bad step arguments");
  if (theory < INQB_THEORY_NONE || theory > INQB_THEORY_LDA) return fail(INQB_ERR_INVALID, "unknown theory");
  INQB_GUARD(ctx);
  INQB_TRY(reserve(ctx, M));
  const long N = ctx->N;
  const size_t esz = ctx->elem_bytes();
  const size_t blk = (size_t)N * M * esz;
  INQB_TRY(ctx->d_scf.ensure(2 * blk));
  char* wb = static_cast<char*>(ctx->d_scf.ptr);
  void* save = wb;
  void* y = wb + blk;
  PotWork w;
  INQB_TRY(pot_work(ctx, w));
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};

  // exponential_2_for_1(H(t), i dt/2, i dt): save = T(i dt/2 H) psi, psi = T(i dt H) psi,
  // both from the same H^k psi (summed term by term, as the reference does)
  INQB_TRY(set_kA(ctx, kA_t_cov, stream));
  INQB_TRY(copy_block(psi, ld, save, M, M, N, esz, stream));
  double c1[2] = {1.0, 0.0}, c2[2] = {1.0, 0.0};
  for (int it = 1; it <= 4; it++) {
    INQB_TRY(apply(ctx, LaunchArgs::H, it == 1 ? psi : y, it == 1 ? ld : M, y, M, M, nullptr, 0, one, zero,
                   stream));
    // c *= f / it with f = i dt/2 and i dt
    const double h1 = 0.5 * dt / it, h2 = dt / it;
    const double a1[2] = {-c1[1] * h1, c1[0] * h1}, a2[2] = {-c2[1] * h2, c2[0] * h2};
    c1[0] = a1[0];
    c1[1] = a1[1];
    c2[0] = a2[0];
    c2[1] = a2[1];
    INQB_TRY(launch_shift2(ctx->precision, y, M, save, M, psi, ld, M, N, c1, c2, stream));
  }
  // density of the predicted step; the Hamiltonian moves to t + dt
  INQB_TRY(sharded_density(ctx, psi, ld, M, occ, rho, stream));
  INQB_TRY(set_kA(ctx, kA_tdt_cov, stream));
  INQB_TRY(ks_potential_dev(ctx, rho, vion, theory, w, stream));

  // the second half step with H(t + dt), self-consistently
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int done_iters = 0;
  for (int iscf = 0; iscf < nscf; iscf++) {
    INQB_TRY(copy_block(save, M, psi, ld, M, N, esz, stream));
    INQB_TRY(exponential(ctx, psi, M, ld, 0.0, 0.5 * dt, 4, stream));
    INQB_CUDA_TRY(cudaMemcpyAsync(w.rho_old, rho, sizeof(double) * N, cudaMemcpyDeviceToDevice,
                                  (cudaStream_t)stream));
    INQB_TRY(sharded_density(ctx, psi, ld, M, occ, rho, stream));
    INQB_TRY(launch_absdiff(w.rho_old, rho, N, w.partial, w.sums + 4, stream));
    INQB_TRY(ks_potential_dev(ctx, rho, vion, theory, w, stream));
    INQB_CUDA_TRY(cudaMemcpyAsync(s, w.sums, sizeof(s), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    done_iters = iscf + 1;
    if (ctx->dV * s[4] < threshold) break;
  }
  if (iters) *iters = done_iters;
  if (energies) energies_from_sums(ctx, s, energies);
  return INQB_OK;
}

int inqb_save_orbitals(inqb_ctx* ctx, const char* dirname, int kpin, const void* psi, int M, int ld,
                       int first_state, const double* occ, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!dirname || kpin < 0 || first_state < 0) return fail(INQB_ERR_INVALID, "bad checkpoint arguments");
  INQB_GUARD(ctx);
  INQB_TRY(ctx->d_io.ensure(checkpoint_staging_bytes(ctx->N, M)));
  return save_states(ctx->precision, dirname, kpin, psi, ld, M, ctx->N, first_state, occ, ctx->d_io.ptr, stream);
}

int inqb_load_orbitals(inqb_ctx* ctx, const char* dirname, int kpin, void* psi, int M, int ld, int first_state,
                       double* occ, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!dirname || kpin < 0 || first_state < 0) return fail(INQB_ERR_INVALID, "bad checkpoint arguments");
  INQB_GUARD(ctx);
  INQB_TRY(ctx->d_io.ensure(checkpoint_staging_bytes(ctx->N, M)));
  return load_states(ctx->precision, dirname, kpin, psi, ld, M, ctx->N, first_state, occ, ctx->d_io.ptr, stream);
}

int inqb_save_density(inqb_ctx* ctx, const char* dirname, const double* rho, void* stream) {
  INQB_CHECK_CTX(ctx);
  if (!dirname || !rho) return fail(INQB_ERR_INVALID, "bad checkpoint arguments");
  INQB_GUARD(ctx);
  return save_density(dirname, rho, ctx->N, stream);
}

int inqb_load_density(inqb_ctx* ctx, const char* dirname, double* rho, void* stream) {
  INQB_CHECK_CTX(ctx);
  if (!dirname || !rho) return fail(INQB_ERR_INVALID, "bad checkpoint arguments");
  INQB_GUARD(ctx);
  return load_density(dirname, rho, ctx->N, stream);
}

int inqb_mlwf_matrices(inqb_ctx* ctx, const void* psi, int M, int ld, void* a, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!a) return fail(INQB_ERR_INVALID, "null matrix buffer");
  INQB_GUARD(ctx);
  MlwfWork w;
  INQB_TRY(mlwf_work(ctx, M, true, w));
  INQB_TRY(launch_band_sums(ctx->precision, psi, psi, ld, M, ctx->N, w.sums, stream));
  return launch_mlwf_gram(ctx->precision, psi, ld, M, ctx->N, ctx->nr, ctx->cell.lat, w.sums, w.partial,
                          static_cast<double2*>(a), stream);
}

int inqb_mlwf_gram_block(inqb_ctx* ctx, const void* a, int Ma, int lda, const void* b, int Mb, int ldb, void* Z,
                         void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, a, Ma, lda));
  INQB_TRY(check_block(ctx, b, Mb, ldb));
  if (!Z) return fail(INQB_ERR_INVALID, "null matrix buffer");
  INQB_GUARD(ctx);
  INQB_TRY(ctx->d_mlwf.ensure(mlwf_partial_bytes(ctx->N, Ma, Mb)));
  return launch_mlwf_gram_block(ctx->precision, a, lda, Ma, b, ldb, Mb, ctx->N, ctx->nr, ctx->cell.lat,
                                ctx->d_mlwf.ptr, static_cast<double2*>(Z), stream);
}

int inqb_mlwf_finish(inqb_ctx* ctx, int M, const void* Z, const double* norms, void* a, void* stream) {
  INQB_CHECK_CTX(ctx);
  if (M <= 0 || !Z || !norms || !a) return fail(INQB_ERR_INVALID, "bad arguments");
  INQB_GUARD(ctx);
  return launch_mlwf_finish(static_cast<const double2*>(Z), M, norms, 1, static_cast<double2*>(a), stream);
}

int inqb_orbital_norms(inqb_ctx* ctx, const void* psi, int M, int ld, double* norms, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!norms) return fail(INQB_ERR_INVALID, "null output");
  INQB_GUARD(ctx);
  DevBuf acc;
  INQB_TRY(acc.ensure(sizeof(double) * 3 * (size_t)M));
  INQB_TRY(launch_band_sums(ctx->precision, psi, psi, ld, M, ctx->N, acc.as<double>(), stream));
  INQB_CUDA_TRY(cudaMemcpy2DAsync(norms, sizeof(double), acc.as<double>() + 2, 3 * sizeof(double), sizeof(double),
                                  M, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return INQB_OK;
}

int inqb_mlwf_centres(inqb_ctx* ctx, int M, const double* adiag, double* centres, double* spreads) {
  INQB_CHECK_CTX(ctx);
  if (M <= 0 || !adiag) return fail(INQB_ERR_INVALID, "bad arguments");
  mlwf_centres(ctx, M, reinterpret_cast<const double2*>(adiag), centres, spreads);
  return INQB_OK;
}

int inqb_jade(inqb_ctx* ctx, int M, void* a, void* u, void* adiag, int maxsweep, double tol, int* sweeps,
              void* stream) {
  INQB_CHECK_CTX(ctx);
  if (M < 1 || !a || !u || !adiag || maxsweep < 1 || !(tol > 0.0)) return fail(INQB_ERR_INVALID, "bad jade arguments");
  INQB_GUARD(ctx);
  MlwfWork w;
  INQB_TRY(mlwf_work(ctx, M, false, w));
  return jade_dev(M, static_cast<double2*>(a), static_cast<double2*>(u), static_cast<double2*>(adiag), maxsweep, tol,
                  w, sweeps, stream);
}

int inqb_mlwf_rotate(inqb_ctx* ctx, void* psi, int M, int ld, const void* u, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!u) return fail(INQB_ERR_INVALID, "null rotation");
  INQB_GUARD(ctx);
  const size_t esz = ctx->elem_bytes();
  INQB_TRY(ctx->d_work.ensure((size_t)ctx->N * M * esz));
  INQB_TRY(launch_mlwf_rotate(ctx->precision, psi, ld, M, ctx->N, static_cast<const double2*>(u), ctx->d_work.ptr, M,
                              stream));
  return copy_block(ctx->d_work.ptr, M, psi, ld, M, ctx->N, esz, stream);
}

int inqb_mlwf_step(inqb_ctx* ctx, void* psi, int M, int ld, int maxsweep, double tol, int* sweeps, double* centres,
                   double* spreads, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (maxsweep < 1 || !(tol > 0.0)) return fail(INQB_ERR_INVALID, "bad jade arguments");
  INQB_GUARD(ctx);
  MlwfWork w;
  INQB_TRY(mlwf_work(ctx, M, true, w));
  INQB_TRY(launch_band_sums(ctx->precision, psi, psi, ld, M, ctx->N, w.sums, stream));
  INQB_TRY(launch_mlwf_gram(ctx->precision, psi, ld, M, ctx->N, ctx->nr, ctx->cell.lat, w.sums, w.partial, w.a,
                            stream));
  INQB_TRY(jade_dev(M, w.a, w.u, w.adiag, maxsweep, tol, w, sweeps, stream));
  const size_t esz = ctx->elem_bytes();
  INQB_TRY(ctx->d_work.ensure((size_t)ctx->N * M * esz));
  INQB_TRY(launch_mlwf_rotate(ctx->precision, psi, ld, M, ctx->N, w.u, ctx->d_work.ptr, M, stream));
  INQB_TRY(copy_block(ctx->d_work.ptr, M, psi, ld, M, ctx->N, esz, stream));
  if (centres || spreads) {
    std::vector<double2> h((size_t)6 * M);
    INQB_CUDA_TRY(cudaMemcpyAsync(h.data(), w.adiag, sizeof(double2) * h.size(), cudaMemcpyDeviceToHost,
                                  (cudaStream_t)stream));
    INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    mlwf_centres(ctx, M, h.data(), centres, spreads);
  }
  return INQB_OK;
}

int inqb_crank_nicolson_step(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                             const double kA_tdt_cov[3], int max_sweeps, double tol, int* sweeps, double* residual,
                             void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!kA_t_cov || !kA_tdt_cov || !std::isfinite(dt) || max_sweeps < 1 || !(tol >= 0.0))
    return fail(INQB_ERR_INVALID, "bad step arguments");
  INQB_GUARD(ctx);
  INQB_TRY(reserve(ctx, M));
  const size_t blk = (size_t)ctx->N * M * ctx->elem_bytes();
  INQB_TRY(ctx->d_cn.ensure(3 * blk));
  INQB_TRY(ctx->d_cnred.ensure(sizeof(double) * 5 * (size_t)M));
  char* w = static_cast<char*>(ctx->d_cn.ptr);
  void* rhs = w;
  void* r = w + blk;
  void* hsd = w + 2 * blk;
  double* acc = ctx->d_cnred.as<double>();
  double* normres = acc + 4 * (size_t)M;
  const long Mi = M;
  cudaStream_t st = (cudaStream_t)stream;
  // rhs = (1 - i dt/2 H(t)) psi  (op_rhs, crank_nicolson.hpp:49-55)
  INQB_TRY(set_kA(ctx, kA_t_cov, stream));
  const double one[2] = {1.0, 0.0};
  const double fr[2] = {0.0, -0.5 * dt}, fl[2] = {0.0, 0.5 * dt};
  INQB_TRY(apply(ctx, LaunchArgs::H, psi, ld, rhs, Mi, M, psi, ld, fr, one, stream));
  INQB_TRY(set_kA(ctx, kA_tdt_cov, stream));
  std::vector<double> hres(M);
  double res = 0.0;
  int k = 0;
  while (k < max_sweeps) {
    // steepest_descent (steepest_descent.hpp:22-80): five steps, no preconditioner
    for (int step = 0; step < 5; step++) {
      // r = (1 + i dt/2 H) phi - rhs
      INQB_TRY(apply(ctx, LaunchArgs::H, psi, ld, r, Mi, M, psi, ld, fl, one, stream));
      {
        const double a[2][2] = {{1.0, 0.0}, {-1.0, 0.0}};
        const void* x[2] = {r, rhs};
        const long ldx[2] = {Mi, Mi};
        INQB_TRY(launch_lincomb(ctx->precision, ctx->N, M, 2, a, x, ldx, r, Mi, stream));
      }
      // hsd = (1 + i dt/2 H) r
      INQB_TRY(apply(ctx, LaunchArgs::H, r, Mi, hsd, Mi, M, r, Mi, fl, one, stream));
      INQB_TRY(launch_sd_sums(ctx->precision, r, hsd, Mi, M, ctx->N, acc, stream));
      INQB_TRY(launch_sd_update(ctx->precision, psi, ld, r, Mi, M, ctx->N, acc, ctx->dV, normres, stream));
    }
    k++;
    INQB_CUDA_TRY(cudaMemcpyAsync(hres.data(), normres, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
    INQB_CUDA_TRY(cudaStreamSynchronize(st));
    res = 0.0;
    for (double v : hres) res = std::max(res, v);
    if (!std::isfinite(res)) return fail(INQB_ERR_NONFINITE, "Crank-Nicolson residual is not finite");
    if (res < tol) break;
  }
  if (sweeps) *sweeps = k;
  if (residual) *residual = res;
  return INQB_OK;
}

int inqb_crank_nicolson_scf_step(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                                 const double kA_tdt_cov[3], const double* occ, double num_electrons, double* rho,
                                 const double* vion, int theory, int max_iter, double dens_tol, int* iters,
                                 double* residual, double energies[4], void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!kA_t_cov || !kA_tdt_cov || !occ || !rho || !std::isfinite(dt) || max_iter < 1 || !(dens_tol >= 0.0) ||
      !(num_electrons > 0.0) || !std::isfinite(num_electrons))
    return fail(INQB_ERR_INVALID, "bad step arguments");
  if (theory < INQB_THEORY_NONE || theory > INQB_THEORY_LDA) return fail(INQB_ERR_INVALID, "unknown theory");
  INQB_GUARD(ctx);
  INQB_TRY(reserve(ctx, M));
  const long N = ctx->N;
  const size_t blk = (size_t)N * M * ctx->elem_bytes();
  INQB_TRY(ctx->d_cn.ensure(3 * blk));
  INQB_TRY(ctx->d_cnred.ensure(sizeof(double) * 5 * (size_t)M));
  char* wb = static_cast<char*>(ctx->d_cn.ptr);
  void* rhs = wb;
  void* r = wb + blk;
  void* hsd = wb + 2 * blk;
  double* acc = ctx->d_cnred.as<double>();
  double* normres = acc + 4 * (size_t)M;
  PotWork pw;
  INQB_TRY(pot_work(ctx, pw));
  MixWork mw;
  INQB_TRY(mix_work(ctx, mw));
  const long Mi = M;
  cudaStream_t st = (cudaStream_t)stream;
  const double one[2] = {1.0, 0.0};
  const double fr[2] = {0.0, -0.5 * dt}, fl[2] = {0.0, 0.5 * dt};

  // rhs = (1 - i dt/2 H(t)) psi with the potential of rho at t (crank_nicolson.hpp:47-56)
  INQB_TRY(set_kA(ctx, kA_t_cov, stream));
  INQB_TRY(apply(ctx, LaunchArgs::H, psi, ld, rhs, Mi, M, psi, ld, fr, one, stream));
  INQB_TRY(set_kA(ctx, kA_tdt_cov, stream));

  BroydenRing ring;  // mixers::broyden(4, 0.3, ...)
  std::vector<double> hres(M);
  double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  double res = 0.0;
  int done_iters = 0;
  for (int istep = 0; istep < max_iter; istep++) {
    // update_hamiltonian(rho) at t + dt, then steepest_descent (five steps, as in
    // inqb_crank_nicolson_step) from the current psi
    INQB_TRY(ks_potential_dev(ctx, rho, vion, theory, pw, stream));
    for (int step = 0; step < 5; step++) {
      INQB_TRY(apply(ctx, LaunchArgs::H, psi, ld, r, Mi, M, psi, ld, fl, one, stream));
      {
        const double a[2][2] = {{1.0, 0.0}, {-1.0, 0.0}};
        const void* x[2] = {r, rhs};
        const long ldx[2] = {Mi, Mi};
        INQB_TRY(launch_lincomb(ctx->precision, N, M, 2, a, x, ldx, r, Mi, stream));
      }
      INQB_TRY(apply(ctx, LaunchArgs::H, r, Mi, hsd, Mi, M, r, Mi, fl, one, stream));
      INQB_TRY(launch_sd_sums(ctx->precision, r, hsd, Mi, M, N, acc, stream));
      INQB_TRY(launch_sd_update(ctx->precision, psi, ld, r, Mi, M, N, acc, ctx->dV, normres, stream));
    }
    // the new density and dV sum |rho - new| / nelec (crank_nicolson.hpp:98-99)
    INQB_TRY(sharded_density(ctx, psi, ld, M, occ, mw.fresh, stream));
    INQB_TRY(launch_absdiff(rho, mw.fresh, N, pw.partial, pw.sums + 4, stream));
    INQB_CUDA_TRY(cudaMemcpyAsync(hres.data(), normres, sizeof(double) * M, cudaMemcpyDeviceToHost, st));
    INQB_CUDA_TRY(cudaMemcpyAsync(s, pw.sums, sizeof(s), cudaMemcpyDeviceToHost, st));
    INQB_CUDA_TRY(cudaStreamSynchronize(st));
    res = 0.0;
    for (double v : hres) res = std::max(res, v);
    if (!std::isfinite(res)) return fail(INQB_ERR_NONFINITE, "Crank-Nicolson residual is not finite");
    done_iters = istep + 1;
    if (ctx->dV * s[4] / num_electrons < dens_tol) break;
    // mixer(rho, new) and normalize(rho, nelec) (crank_nicolson.hpp:107-108)
    INQB_TRY(broyden_mix_density(ctx, ring, rho, mw, num_electrons, stream));
  }
  // rho = density(psi), update_hamiltonian(rho) (crank_nicolson.hpp:111-112)
  INQB_TRY(sharded_density(ctx, psi, ld, M, occ, rho, stream));
  INQB_TRY(ks_potential_dev(ctx, rho, vion, theory, pw, stream));
  INQB_CUDA_TRY(cudaMemcpyAsync(s, pw.sums, sizeof(double) * 4, cudaMemcpyDeviceToHost, st));
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  if (iters) *iters = done_iters;
  if (residual) *residual = res;
  if (energies) energies_from_sums(ctx, s, energies);
  return INQB_OK;
}

int inqb_density(inqb_ctx* ctx, const void* psi, int M, int ld, const double* occ, double* rho, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!occ || !rho) return fail(INQB_ERR_INVALID, "null occupation or density");
  INQB_GUARD(ctx);
  return launch_density(ctx->precision, psi, ld, M, ctx->N, occ, rho, stream);
}

int inqb_dipole(inqb_ctx* ctx, const double* rho, double out[3], void* stream) {
  INQB_CHECK_CTX(ctx);
  if (!rho || !out) return fail(INQB_ERR_INVALID, "null argument");
  INQB_GUARD(ctx);
  INQB_TRY(ctx->d_red.ensure(256));
  double* d = ctx->d_red.as<double>();
  INQB_TRY(launch_dipole(rho, ctx->N, ctx->cell.lat, ctx->nr, d, stream));
  double h[3];
  INQB_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  for (int k = 0; k < 3; k++) out[k] = ctx->dV * h[k];
  return INQB_OK;
}

int inqb_band_energies(inqb_ctx* ctx, const void* psi, const void* hpsi, int M, int ld, double* eps,
                       void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  INQB_TRY(check_block(ctx, hpsi, M, ld));
  if (!eps) return fail(INQB_ERR_INVALID, "null output");
  INQB_GUARD(ctx);
  INQB_TRY(ctx->d_band.ensure(sizeof(double) * 3 * (size_t)M));
  double* d = ctx->d_band.as<double>();
  INQB_TRY(launch_band_sums(ctx->precision, psi, hpsi, ld, M, ctx->N, d, stream));
  std::vector<double> h(3 * (size_t)M);
  INQB_CUDA_TRY(cudaMemcpyAsync(h.data(), d, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  for (int m = 0; m < M; m++) eps[m] = h[3 * m] / h[3 * m + 2];
  return INQB_OK;
}

int inqb_orthonormalize(inqb_ctx* ctx, void* psi, int M, int ld, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  INQB_GUARD(ctx);
  DevBuf S, X, info;
  INQB_TRY(S.ensure(sizeof(double2) * (size_t)M * M));
  INQB_TRY(X.ensure(sizeof(double2) * (size_t)M * M));
  INQB_TRY(info.ensure(sizeof(int)));
  return launch_orthonormalize(ctx->precision, psi, ld, M, ctx->N, ctx->dV, S.as<double2>(), X.as<double2>(),
                               info.as<int>(), stream);
}

int inqb_overlap_block(inqb_ctx* ctx, const void* a, int Ma, int lda, const void* b, int Mb, int ldb, double* S,
                       int lds, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, a, Ma, lda));
  INQB_TRY(check_block(ctx, b, Mb, ldb));
  if (!S || lds < Mb) return fail(INQB_ERR_INVALID, "overlap block: need S and lds >= Mb");
  INQB_GUARD(ctx);
  return launch_overlap_block(ctx->precision, a, lda, Ma, b, ldb, Mb, ctx->N, ctx->dV,
                              reinterpret_cast<double2*>(S), lds, stream);
}

int inqb_cholesky_inverse(inqb_ctx* ctx, double* S, int M, int lds, void* stream) {
  INQB_CHECK_CTX(ctx);
  if (!S || M <= 0 || lds < M) return fail(INQB_ERR_INVALID, "cholesky inverse: need S, M > 0 and lds >= M");
  if (((uintptr_t)S) % 16 != 0) return fail(INQB_ERR_INVALID, "cholesky inverse: S must be 16-byte aligned");
  INQB_GUARD(ctx);
  DevBuf X, info;
  INQB_TRY(X.ensure(sizeof(double2) * (size_t)M * M));
  INQB_TRY(info.ensure(sizeof(int)));
  return launch_cholesky_inverse(reinterpret_cast<double2*>(S), M, lds, X.as<double2>(), info.as<int>(), stream);
}

int inqb_rotate_block(inqb_ctx* ctx, const void* a, int Ma, int lda, const double* R, int ldr, int Mo, void* out,
                      int ldo, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, a, Ma, lda));
  INQB_TRY(check_block(ctx, out, Mo, ldo));
  if (!R || ldr < Mo) return fail(INQB_ERR_INVALID, "rotate block: need R and ldr >= Mo");
  if (((uintptr_t)R) % 16 != 0) return fail(INQB_ERR_INVALID, "rotate block: R must be 16-byte aligned");
  const size_t esz = ctx->elem_bytes();
  const char* a0 = static_cast<const char*>(a);
  const char* o0 = static_cast<const char*>(out);
  const size_t span_a = ((size_t)(ctx->N - 1) * lda + Ma) * esz, span_o = ((size_t)(ctx->N - 1) * ldo + Mo) * esz;
  if (o0 < a0 + span_a && a0 < o0 + span_o) return fail(INQB_ERR_INVALID, "rotate block: out overlaps a");
  INQB_GUARD(ctx);
  return launch_rotate_block(ctx->precision, a, lda, Ma, reinterpret_cast<const double2*>(R), ldr, Mo, out, ldo,
                             ctx->N, stream);
}

int inqb_batch_create(inqb_ctx* const* cells, int ncells, inqb_batch** out) {
  if (!cells || !out || ncells <= 0) return fail(INQB_ERR_INVALID, "bad batch arguments");
  *out = nullptr;
  for (int i = 0; i < ncells; i++) {
    if (!cells[i]) return fail(INQB_ERR_INVALID, "null cell context");
    if (cells[i]->device != cells[0]->device) return fail(INQB_ERR_INVALID, "cells on different devices");
  }
  DeviceGuard guard(cells[0]->device);
  if (guard.status != INQB_OK) return guard.status;
  auto* b = new inqb_batch();
  b->cells.assign(cells, cells + ncells);
  b->device = cells[0]->device;
  if (b->d_err.ensure(sizeof(int)) != INQB_OK || cudaMemset(b->d_err.ptr, 0, sizeof(int)) != cudaSuccess) {
    delete b;
    return fail(INQB_ERR_NOMEM, "batch error word");
  }
  for (int i = 0; i <= ncells; i++) {
    cudaStream_t s;
    cudaEvent_t e;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      for (auto x : b->streams) cudaStreamDestroy(x);
      for (auto x : b->events) cudaEventDestroy(x);
      delete b;
      return fail(INQB_ERR_CUDA, "stream or event creation failed");
    }
    b->streams.push_back(s);
    b->events.push_back(e);
  }
  *out = b;
  return INQB_OK;
}

int inqb_batch_destroy(inqb_batch* b) {
  if (!b) return INQB_OK;
  DeviceGuard guard(b->device);
  cudaDeviceSynchronize();
  batch_release_graph(b);
  for (auto x : b->streams) cudaStreamDestroy(x);
  for (auto x : b->events) cudaEventDestroy(x);
  delete b;
  return INQB_OK;
}

int inqb_batch_apply_h(inqb_batch* b, const void* const* psis, void* const* hpsis, const int* Ms, const int* lds,
                       void* stream) {
  if (!b || !psis || !hpsis || !Ms || !lds) return fail(INQB_ERR_INVALID, "null batch argument");
  const int n = (int)b->cells.size();
  for (int i = 0; i < n; i++) {
    INQB_TRY(check_block(b->cells[i], psis[i], Ms[i], lds[i]));
    INQB_TRY(check_block(b->cells[i], hpsis[i], Ms[i], lds[i]));
  }
  DeviceGuard guard(b->device);
  if (guard.status != INQB_OK) return guard.status;
  bool same = b->ready;
  for (int i = 0; i < n && same; i++)
    same = b->psis[i] == psis[i] && b->hpsis[i] == hpsis[i] && b->Ms[i] == Ms[i] && b->lds[i] == lds[i];
  if (!same) {
    b->ready = false;
    b->persistent = false;
    // workspace, attributes and phases are set up outside the capture
    for (int i = 0; i < n; i++) {
      INQB_TRY(reserve(b->cells[i], Ms[i]));
      if (!b->cells[i]->proj_phases_valid) {
        INQB_TRY(update_phases(b->cells[i], nullptr));
        b->cells[i]->proj_phases_valid = true;
      }
      const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
      INQB_TRY(apply(b->cells[i], LaunchArgs::H, psis[i], lds[i], hpsis[i], lds[i], Ms[i], nullptr, 0, one, zero,
                     nullptr));
    }
    INQB_CUDA_TRY(cudaDeviceSynchronize());
    batch_release_graph(b);
    const int form = b->mode == INQB_BATCH_AUTO ? b->tuned : b->mode;
    if (form == INQB_BATCH_PERSISTENT) {
      const int st = batch_build_persistent(b, psis, hpsis, Ms, lds);
      if (st == INQB_OK)
        b->persistent = true;
      else if (b->mode == INQB_BATCH_PERSISTENT || st != INQB_ERR_UNSUPPORTED)
        return st;  // AUTO falls back to the graph where the cells do not fit the kernel
    }
    if (!b->persistent) INQB_TRY(batch_capture(b, psis, hpsis, Ms, lds));
    b->psis.assign(psis, psis + n);
    b->hpsis.assign(hpsis, hpsis + n);
    b->Ms.assign(Ms, Ms + n);
    b->lds.assign(lds, lds + n);
    b->ready = true;
  }
  if (b->persistent)
    return launch_batch(b->precision, b->cells_blob.data(), n, b->cell_bytes, b->d_items.as<BatchItem>(), b->nitems,
                        b->d_ctr.as<unsigned>(), b->ncounters, b->d_err.as<int>(), (long long)(b->wait_s * 1e9),
                        b->ctas, b->smem, stream);
  INQB_CUDA_TRY(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return INQB_OK;
}

int inqb_batch_set_mode(inqb_batch* b, int mode) {
  if (!b) return fail(INQB_ERR_INVALID, "null batch");
  if (mode != INQB_BATCH_AUTO && mode != INQB_BATCH_GRAPH && mode != INQB_BATCH_PERSISTENT)
    return fail(INQB_ERR_INVALID, "unknown batch mode");
  b->mode = mode;
  b->ready = false;
  return INQB_OK;
}

int inqb_batch_autotune(inqb_batch* b, const void* const* psis, void* const* hpsis, const int* Ms, const int* lds,
                        void* stream, int* form, double* ms) {
  if (!b) return fail(INQB_ERR_INVALID, "null batch");
  DeviceGuard guard(b->device);
  if (guard.status != INQB_OK) return guard.status;
  cudaStream_t st = (cudaStream_t)stream;
  const int saved = b->mode;
  double t[2] = {-1.0, -1.0};
  cudaEvent_t e0, e1;
  INQB_CUDA_TRY(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(INQB_ERR_CUDA, "event creation failed");
  }
  int rc = INQB_OK;
  const int forms[2] = {INQB_BATCH_GRAPH, INQB_BATCH_PERSISTENT};
  for (int k = 0; k < 2 && rc == INQB_OK; k++) {
    b->mode = forms[k];
    b->ready = false;
    int r = inqb_batch_apply_h(b, psis, hpsis, Ms, lds, stream);  // builds the form
    if (r == INQB_ERR_UNSUPPORTED && forms[k] == INQB_BATCH_PERSISTENT) continue;
    if (r != INQB_OK) {
      rc = r;
      break;
    }
    constexpr int kWarm = 2, kTimed = 5;
    for (int i = 0; i < kWarm && r == INQB_OK; i++) r = inqb_batch_apply_h(b, psis, hpsis, Ms, lds, stream);
    if (r == INQB_OK && cudaEventRecord(e0, st) != cudaSuccess) r = fail(INQB_ERR_CUDA, "event record");
    for (int i = 0; i < kTimed && r == INQB_OK; i++) r = inqb_batch_apply_h(b, psis, hpsis, Ms, lds, stream);
    if (r == INQB_OK && cudaEventRecord(e1, st) != cudaSuccess) r = fail(INQB_ERR_CUDA, "event record");
    if (r == INQB_OK && cudaEventSynchronize(e1) != cudaSuccess) r = fail(INQB_ERR_CUDA, "event sync");
    float el = 0.f;
    if (r == INQB_OK && cudaEventElapsedTime(&el, e0, e1) != cudaSuccess) r = fail(INQB_ERR_CUDA, "elapsed time");
    if (r == INQB_OK && forms[k] == INQB_BATCH_PERSISTENT) r = inqb_batch_status(b, stream);
    if (r != INQB_OK) {
      rc = r;
      break;
    }
    t[k] = el / kTimed;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->mode = saved;
  b->ready = false;
  if (rc != INQB_OK) return rc;
  b->tuned = (t[1] > 0.0 && t[1] < t[0]) ? INQB_BATCH_PERSISTENT : INQB_BATCH_GRAPH;
  if (form) *form = b->tuned;
  if (ms) {
    ms[0] = t[0];
    ms[1] = t[1];
  }
  return INQB_OK;
}

int inqb_batch_info(inqb_batch* b, int* form, int* nitems, int* ctas) {
  if (!b) return fail(INQB_ERR_INVALID, "null batch");
  if (form) *form = !b->ready ? 0 : (b->persistent ? INQB_BATCH_PERSISTENT : INQB_BATCH_GRAPH);
  if (nitems) *nitems = b->persistent ? b->nitems : 0;
  if (ctas) *ctas = b->persistent ? b->ctas : 0;
  return INQB_OK;
}

int inqb_batch_status(inqb_batch* b, void* stream) {
  if (!b) return fail(INQB_ERR_INVALID, "null batch");
  DeviceGuard guard(b->device);
  if (guard.status != INQB_OK) return guard.status;
  cudaStream_t st = (cudaStream_t)stream;
  int word = 0;
  INQB_CUDA_TRY(cudaMemcpyAsync(&word, b->d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  if (word == 0) return INQB_OK;
  INQB_CUDA_TRY(cudaMemsetAsync(b->d_err.ptr, 0, sizeof(int), st));
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  return fail(INQB_ERR_TIMEOUT, "a device-side wait of the persistent batch launch gave up (its results are not valid)");
}

int inqb_batch_set_wait_limit(inqb_batch* b, double seconds) {
  if (!b) return fail(INQB_ERR_INVALID, "null batch");
  if (!(seconds > 0.0) || seconds > 60.0) return fail(INQB_ERR_INVALID, "wait limit must be in (0, 60] seconds");
  b->wait_s = seconds;
  return INQB_OK;
}

int inqb_batch_test_unreachable_wait(inqb_batch* b, int on) {
  if (!b) return fail(INQB_ERR_INVALID, "null batch");
  b->unreachable = on ? 1 : 0;
  b->ready = false;
  return INQB_OK;
}

int inqb_axpby(inqb_ctx* ctx, int M, double a_re, double a_im, const void* x, int ldx, double b_re, double b_im,
               void* y, int ldy, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, x, M, ldx));
  INQB_TRY(check_block(ctx, y, M, ldy));
  INQB_GUARD(ctx);
  const double a[2] = {a_re, a_im}, b[2] = {b_re, b_im};
  return launch_axpby(ctx->precision, ctx->N, M, a, x, ldx, b, y, ldy, stream);
}

int inqb_position_scale(inqb_ctx* ctx, const void* psi, int ld, void* out, int ldo, int M, int dir,
                        const double* occ, double scale, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  INQB_TRY(check_block(ctx, out, M, ldo));
  if (dir < 0 || dir > 2 || !occ) return fail(INQB_ERR_INVALID, "bad direction or occupations");
  INQB_GUARD(ctx);
  return launch_position_scale(ctx->precision, *ctx, psi, ld, out, ldo, M, dir, occ, scale, stream);
}

int inqb_accum_potential_gradient(inqb_ctx* ctx, const void* u, const void* w, int M, int ld, double c_re,
                                  double c_im, double* gV, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, u, M, ld));
  INQB_TRY(check_block(ctx, w, M, ld));
  if (!gV) return fail(INQB_ERR_INVALID, "null gradient");
  INQB_GUARD(ctx);
  return launch_vgrad(ctx->precision, ctx->N, M, u, w, ld, c_re, c_im, gV, stream);
}

int inqb_accum_vector_potential_gradient(inqb_ctx* ctx, const void* u, const void* w, int M, int ld, double c_re,
                                         double c_im, double* gA, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, u, M, ld));
  INQB_TRY(check_block(ctx, w, M, ld));
  if (!gA) return fail(INQB_ERR_INVALID, "null gradient");
  INQB_GUARD(ctx);
  const size_t bytes = (size_t)ctx->N * M * ctx->elem_bytes();
  INQB_TRY(ctx->d_adjU.ensure(bytes));
  INQB_TRY(ctx->d_adjW.ensure(bytes));
  INQB_TRY(ctx->d_red.ensure(256));
  INQB_TRY(ctx->d_nlpart.ensure(std::max<size_t>(
      (size_t)ctx->proj.chunk_atom.size() * ctx->proj.L * 16 * M * sizeof(double), 16)));
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  INQB_TRY(apply(ctx, LaunchArgs::FFT_FWD, u, ld, ctx->d_adjU.ptr, M, M, nullptr, 0, one, zero, stream));
  INQB_TRY(apply(ctx, LaunchArgs::FFT_FWD, w, ld, ctx->d_adjW.ptr, M, M, nullptr, 0, one, zero, stream));
  return launch_agrad(*ctx, ctx->d_adjU.ptr, ctx->d_adjW.ptr, u, w, ld, M, ctx->d_red.as<double>(), c_re, c_im, gA,
                      stream);
}

// ---------------------------------------------------------------- native ETRS adjoint step
namespace inqb {
namespace {

// c_k = (i dt/2)^k / k!, k = 0..4: the Taylor coefficients of one ETRS half step
void taylor_coeffs(double dt, double c[5][2]) {
  double re = 1.0, im = 0.0;
  c[0][0] = 1.0;
  c[0][1] = 0.0;
  for (int k = 1; k <= 4; k++) {
    const double f = 0.5 * dt / k;  // (i f) * (re + i im)
    const double nre = -f * im, nim = f * re;
    re = nre;
    im = nim;
    c[k][0] = re;
    c[k][1] = im;
  }
}

// Elements of one block of forward coefficients in the tile layout (orbital groups
// padded to the tile's G).
size_t fourier_elems(const inqb_ctx* ctx, int M) {
  const size_t G = (size_t)ctx->plan->G_tile;
  return (M + G - 1) / G * G * (size_t)ctx->N;
}

// One half step psi -> sum_k c_k H^k psi at the current k + A, keeping
// P[0..3] = H^k psi (P[0] a copy of the input) and F[0..3] = their forward
// coefficients (tile layout, written by the H applications); `out` receives the result.
// One half step term by term: P[k] = H^k in (k < 4), out = sum_k c_k H^k in.  With
// keep, P[0] receives a copy of in and F[k] the forward coefficients of P[k]; without,
// P[0] is in itself and no coefficients are written (the same arithmetic).
int half_step_powers(inqb_ctx* ctx, const void* in, long ld_in, void* const P[4], void* const F[4], void* out,
                     long ld_out, int M, const double c[5][2], void* stream, bool keep = true) {
  const long Mi = M;
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  void* H4 = ctx->d_adjL.ptr;
  const void* p0 = in;
  long ld0 = ld_in;
  if (keep) {
    const double a[1][2] = {{1.0, 0.0}};
    const void* x[1] = {in};
    const long ldx[1] = {ld_in};
    INQB_TRY(launch_lincomb(ctx->precision, ctx->N, M, 1, a, x, ldx, P[0], Mi, stream));
    p0 = P[0];
    ld0 = Mi;
  }
  const void* src = p0;
  long lds = ld0;
  for (int k = 1; k < 4; k++) {
    INQB_TRY(apply(ctx, LaunchArgs::H, src, lds, P[k], Mi, M, nullptr, 0, one, zero, stream,
                   keep ? F[k - 1] : nullptr));
    src = P[k];
    lds = Mi;
  }
  INQB_TRY(apply(ctx, LaunchArgs::H, P[3], Mi, H4, Mi, M, nullptr, 0, one, zero, stream, keep ? F[3] : nullptr));
  const void* x[5] = {p0, P[1], P[2], P[3], H4};
  const long ldx[5] = {ld0, Mi, Mi, Mi, Mi};
  return launch_lincomb(ctx->precision, ctx->N, M, 5, c, x, ldx, out, ld_out, stream);
}

// Reverse of one half step at the current k + A: with Lambda_j = H^j lam,
//   Xi_i = sum_j conj(c_{i+j+1}) Lambda_j,   gV += 2 Re conj(Xi_i) Phi_i,
//   gA += 2 Re <Xi_i| dH/dA |Phi_i>,          lam <- sum_k conj(c_k) Lambda_k.
// The kinetic part of dH/dA reads forward coefficients: those of Phi_i were kept by
// the forward step (FPhi), those of Xi_i are the same combination of the Lambda_j's,
// which the H applications below emit.
int half_back(inqb_ctx* ctx, void* lam, long ld, int M, const double c[5][2], const void* const Phi[4],
              const void* const FPhi[4], double* gV, double* gA, void* stream) {
  const long Mi = M;
  const size_t blk = (size_t)ctx->N * M * ctx->elem_bytes();
  const size_t nF = fourier_elems(ctx, M);
  const size_t fblk = nF * ctx->elem_bytes();
  char* w = static_cast<char*>(ctx->d_adjL.ptr);
  void* Lam[5] = {lam, w + blk, w + 2 * blk, w + 3 * blk, w + 4 * blk};
  char* wf = w + 6 * blk;
  void* FL[4] = {wf, wf + fblk, wf + 2 * fblk, wf + 3 * fblk};
  const long ldL[5] = {ld, Mi, Mi, Mi, Mi};
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  for (int j = 1; j <= 4; j++)
    INQB_TRY(apply(ctx, LaunchArgs::H, Lam[j - 1], ldL[j - 1], Lam[j], Mi, M, nullptr, 0, one, zero, stream,
                   FL[j - 1]));
  double cc[5][2];
  for (int k = 0; k < 5; k++) {
    cc[k][0] = c[k][0];
    cc[k][1] = -c[k][1];
  }
  // gradients of the four (Xi_i, Phi_i) pairs in one pass over the eight blocks
  double wgt[4][4][2] = {};
  for (int i = 0; i < 4; i++)
    for (int j = 0; j + i <= 3; j++) {
      wgt[i][j][0] = cc[i + j + 1][0];
      wgt[i][j][1] = cc[i + j + 1][1];
    }
  {
    const void* L4[4] = {Lam[0], Lam[1], Lam[2], Lam[3]};
    const long ld4[4] = {ldL[0], ldL[1], ldL[2], ldL[3]};
    const void* F4[4] = {FL[0], FL[1], FL[2], FL[3]};
    INQB_TRY(launch_half_grad(*ctx, L4, ld4, Phi, Mi, F4, FPhi, wgt, M, gV, gA, stream));
  }
  const void* x[5] = {Lam[0], Lam[1], Lam[2], Lam[3], Lam[4]};
  return launch_lincomb(ctx->precision, ctx->N, M, 5, cc, x, ldL, lam, ld, stream);
}

// Bytes of one step's powers: 8 orbital blocks [N][M] then 8 coefficient blocks.
size_t powers_bytes(const inqb_ctx* ctx, int M) {
  return 8 * ((size_t)ctx->N * M + fourier_elems(ctx, M)) * ctx->elem_bytes();
}

int adjoint_workspace(inqb_ctx* ctx, int M) {
  const size_t blk = (size_t)ctx->N * M * ctx->elem_bytes();
  const size_t fblk = fourier_elems(ctx, M) * ctx->elem_bytes();
  INQB_TRY(ctx->d_adjL.ensure(6 * blk + 5 * fblk));
  INQB_TRY(ctx->d_red.ensure(256));
  // per-chunk moments of four pairs of blocks
  INQB_TRY(ctx->d_nlpart.ensure(std::max<size_t>(
      (size_t)ctx->proj.chunk_atom.size() * 4 * ctx->proj.L * 16 * M * sizeof(double), 16)));
  return reserve(ctx, M);
}

}  // namespace
}  // namespace inqb

int inqb_etrs_powers_size(inqb_ctx* ctx, int M, size_t* bytes) {
  INQB_CHECK_CTX(ctx);
  if (M <= 0 || !bytes) return fail(INQB_ERR_INVALID, "M must be positive and bytes not null");
  *bytes = powers_bytes(ctx, M);
  return INQB_OK;
}

int inqb_etrs_step_powers(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                          const double kA_tdt_cov[3], void* powers, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!powers || (uintptr_t)powers % 16 != 0) return fail(INQB_ERR_INVALID, "powers must be 16-byte aligned");
  if (!kA_t_cov || !kA_tdt_cov || !std::isfinite(dt)) return fail(INQB_ERR_INVALID, "bad step arguments");
  INQB_GUARD(ctx);
  INQB_TRY(adjoint_workspace(ctx, M));
  double c[5][2];
  taylor_coeffs(dt, c);
  const size_t blk = (size_t)ctx->N * M * ctx->elem_bytes();
  const size_t fblk = fourier_elems(ctx, M) * ctx->elem_bytes();
  char* P = static_cast<char*>(powers);
  char* F = P + 8 * blk;
  void* P1[4] = {P, P + blk, P + 2 * blk, P + 3 * blk};
  void* P2[4] = {P + 4 * blk, P + 5 * blk, P + 6 * blk, P + 7 * blk};
  void* F1[4] = {F, F + fblk, F + 2 * fblk, F + 3 * fblk};
  void* F2[4] = {F + 4 * fblk, F + 5 * fblk, F + 6 * fblk, F + 7 * fblk};
  INQB_TRY(set_kA(ctx, kA_t_cov, stream));
  // phi = the first half step, written straight into P2[0]
  INQB_TRY(half_step_powers(ctx, psi, ld, P1, F1, P2[0], M, M, c, stream));
  INQB_TRY(set_kA(ctx, kA_tdt_cov, stream));
  return half_step_powers(ctx, P2[0], M, P2, F2, psi, ld, M, c, stream);
}

int inqb_etrs_step_terms(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                         const double kA_tdt_cov[3], void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  if (!kA_t_cov || !kA_tdt_cov || !std::isfinite(dt)) return fail(INQB_ERR_INVALID, "bad step arguments");
  INQB_GUARD(ctx);
  INQB_TRY(adjoint_workspace(ctx, M));
  double c[5][2];
  taylor_coeffs(dt, c);
  // the adjoint workspace: block 0 takes H^4, blocks 1-3 the powers, block 4 phi
  const size_t blk = (size_t)ctx->N * M * ctx->elem_bytes();
  char* w = static_cast<char*>(ctx->d_adjL.ptr);
  void* P[4] = {nullptr, w + blk, w + 2 * blk, w + 3 * blk};
  void* const F[4] = {nullptr, nullptr, nullptr, nullptr};
  void* phi = w + 4 * blk;
  INQB_TRY(set_kA(ctx, kA_t_cov, stream));
  INQB_TRY(half_step_powers(ctx, psi, ld, P, F, phi, M, M, c, stream, false));
  INQB_TRY(set_kA(ctx, kA_tdt_cov, stream));
  return half_step_powers(ctx, phi, M, P, F, psi, ld, M, c, stream, false);
}

int inqb_etrs_adjoint_step(inqb_ctx* ctx, void* lambda, int M, int ld, double dt, const double kA_t_cov[3],
                           const double kA_tdt_cov[3], const void* powers, double* gV, double* gA_t,
                           double* gA_tdt, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, lambda, M, ld));
  if (!powers || (uintptr_t)powers % 16 != 0) return fail(INQB_ERR_INVALID, "powers must be 16-byte aligned");
  if (!kA_t_cov || !kA_tdt_cov || !std::isfinite(dt)) return fail(INQB_ERR_INVALID, "bad step arguments");
  if (!gV || !gA_t || !gA_tdt) return fail(INQB_ERR_INVALID, "null gradient");
  INQB_GUARD(ctx);
  INQB_TRY(adjoint_workspace(ctx, M));
  double c[5][2];
  taylor_coeffs(dt, c);
  const size_t blk = (size_t)ctx->N * M * ctx->elem_bytes();
  const size_t fblk = fourier_elems(ctx, M) * ctx->elem_bytes();
  const char* P = static_cast<const char*>(powers);
  const char* F = P + 8 * blk;
  const void* P1[4] = {P, P + blk, P + 2 * blk, P + 3 * blk};
  const void* P2[4] = {P + 4 * blk, P + 5 * blk, P + 6 * blk, P + 7 * blk};
  const void* F1[4] = {F, F + fblk, F + 2 * fblk, F + 3 * fblk};
  const void* F2[4] = {F + 4 * fblk, F + 5 * fblk, F + 6 * fblk, F + 7 * fblk};
  INQB_TRY(set_kA(ctx, kA_tdt_cov, stream));
  INQB_TRY(half_back(ctx, lambda, ld, M, c, P2, F2, gV, gA_tdt, stream));
  INQB_TRY(set_kA(ctx, kA_t_cov, stream));
  return half_back(ctx, lambda, ld, M, c, P1, F1, gV, gA_t, stream);
}

int inqb_set_schedule(inqb_ctx* ctx, int M, const int schedule[4]) {
  INQB_CHECK_CTX(ctx);
  if (M <= 0) return fail(INQB_ERR_INVALID, "M must be positive");
  if (!schedule) {
    ctx->schedules.erase(M);
    return INQB_OK;
  }
  if (schedule[0] < 1 || ctx->plan->y1 % schedule[0] != 0)
    return fail(INQB_ERR_INVALID, "schedule: ysplit must divide " + std::to_string(ctx->plan->y1));
  for (int k = 1; k < 4; k++)
    if (schedule[k] < 64 || schedule[k] > 256 || schedule[k] % 32 != 0)
      return fail(INQB_ERR_INVALID, "schedule: threads per CTA must be a multiple of 32 in [64, 256]");
  ctx->schedules[M] = {schedule[0], schedule[1], schedule[2], schedule[3]};
  return INQB_OK;
}

int inqb_autotune(inqb_ctx* ctx, int M, void* stream, int schedule[4]) {
  INQB_CHECK_CTX(ctx);
  if (M <= 0) return fail(INQB_ERR_INVALID, "M must be positive");
  INQB_GUARD(ctx);
  INQB_TRY(reserve(ctx, M));
  // the timings do not depend on the values: zeroed blocks
  DevBuf in, out;
  const size_t bytes = (size_t)ctx->N * M * ctx->elem_bytes();
  INQB_TRY(in.ensure(bytes));
  INQB_TRY(out.ensure(bytes));
  cudaStream_t st = (cudaStream_t)stream;
  INQB_CUDA_TRY(cudaMemsetAsync(in.ptr, 0, bytes, st));
  cudaEvent_t ev[6];
  for (auto& e : ev) INQB_CUDA_TRY(cudaEventCreate(&e));
  const double one[2] = {1.0, 0.0}, zero[2] = {0.0, 0.0};
  const bool saved_timing = ctx->timing_on;
  ctx->timing_on = false;
  std::array<int, 4> best = {ctx->plan->ysplit, 256, 256, 256};
  // pass times (ms) of one schedule: the best of three applications after a warm-up
  auto pass_ms = [&](const std::array<int, 4>& s, float out_ms[3]) -> int {
    ctx->schedules[M] = s;
    for (int k = 0; k < 3; k++) out_ms[k] = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
      INQB_TRY(apply_events(ctx, in.ptr, out.ptr, M, one, zero, stream, ev));
      INQB_CUDA_TRY(cudaEventSynchronize(ev[5]));
      if (rep == 0) continue;
      // the three tile passes (the projection kernel is not scheduled)
      for (int k = 0; k < 3; k++) {
        float t = 0.f;
        INQB_CUDA_TRY(cudaEventElapsedTime(&t, ev[k + 2], ev[k + 3]));
        out_ms[k] = std::min(out_ms[k], t);
      }
    }
    return INQB_OK;
  };
  int status = INQB_OK;
  float t[3], best_t[3] = {1e30f, 1e30f, 1e30f};
  // pass A: every divisor of Y1 times every thread count; passes B and C: thread counts
  for (int ys = 1; ys <= ctx->plan->y1 && status == INQB_OK; ys++) {
    if (ctx->plan->y1 % ys != 0) continue;
    for (int thr : kScheduleThreads) {
      std::array<int, 4> s = best;
      s[0] = ys;
      s[1] = thr;
      if ((status = pass_ms(s, t)) != INQB_OK) break;
      if (t[0] < best_t[0]) {
        best_t[0] = t[0];
        best[0] = ys;
        best[1] = thr;
      }
    }
  }
  for (int k = 1; k < 3 && status == INQB_OK; k++)
    for (int thr : kScheduleThreads) {
      std::array<int, 4> s = best;
      s[1 + k] = thr;
      if ((status = pass_ms(s, t)) != INQB_OK) break;
      if (t[k] < best_t[k]) {
        best_t[k] = t[k];
        best[1 + k] = thr;
      }
    }
  for (auto& e : ev) cudaEventDestroy(e);
  ctx->timing_on = saved_timing;
  if (status != INQB_OK) {
    ctx->schedules.erase(M);
    return status;
  }
  ctx->schedules[M] = best;
  if (schedule)
    for (int k = 0; k < 4; k++) schedule[k] = best[k];
  return INQB_OK;
}

int inqb_orthonormalize_noalloc(inqb_ctx* ctx, void* psi, int M, int ld, void* stream) {
  INQB_CHECK_CTX(ctx);
  INQB_TRY(check_block(ctx, psi, M, ld));
  INQB_GUARD(ctx);
  return orthonormalize_noalloc(ctx->precision, ctx->device, psi, ld, M, ctx->N, ctx->dV, stream);
}

}  // extern "C"
