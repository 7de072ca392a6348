// The launcher of the tile kernels (tiles.cuh) for one compiled grid: the shared
// kernel parameters, the projection finish kernel and launch_h_impl<T, NX, NY, NZ>.
// Included by the grid translation units (grids_*.cu), each of which instantiates
// the plans of a group of grids.
//
// H|psi> (src/hamiltonian/ks_hamiltonian.hpp:132-152): k_tile_fwd (z FFT, inner
// y stage, KB projection) -> k_tile_x (outer y stage, x FFT, kinetic, inverse) ->
// k_tile_inv (inverse stages, epilogue with V psi and the nonlocal term).
// to_fourier: k_tile_fwd without projection -> k_tile_x_fft<0>.
// to_real: k_tile_x_fft<1> -> k_tile_inv<MODE_H = 0> with the 1/N.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "batch.h"
#include "fft_tile.cuh"
#include "inqb_internal.h"
#include "plan.h"
#include "project.h"
#include "sizes.h"

namespace inqb {

constexpr int LMAX = 4;  // KB projectors per atom handled by the fused kernels

// ---------------------------------------------------------------- sizes
template <int N>
struct Split;
#define INQB_SPLIT(N, A, B)              \
  template <>                            \
  struct Split<N> {                      \
    static constexpr int N1 = A, N2 = B; \
  };
INQB_FFT_SIZES(INQB_SPLIT)
#undef INQB_SPLIT

// ---------------------------------------------------------------- kernel params
template <typename T>
struct KinParams {
  T b[3][3];  // reciprocal vectors: G_cart = sum_d n_d b[d]
  T kA[3];    // cartesian k + A
  T scale;    // 1/N folded into the kinetic factor
  int mask;   // zero the Laplacian term outside the Fourier sphere (|n/N|^2 > 1/4)
  int nr[3];
  T shift;    // 1/2 |k+A|^2 / N, moved to the epilogue when the mask is on
  // Poisson mode when nonzero (k + A = 0, scale 1, so the quadratic is 1/2 |G|^2):
  // the factor becomes pois / (1/2 |G|^2) = 4 pi / (N |G|^2), 0 where |G|^2 < 1e-6
  // (solvers::poisson's periodic kernel, src/solvers/poisson.hpp:29-35,66-83)
  T pois;
};

// INQ's fourier_space::outside_sphere (src/basis/fourier_space.hpp:87-93) in exact
// integer arithmetic: sum_d (n_d / N_d)^2 > 1/4.
__device__ __forceinline__ bool outside_sphere(const int nr[3], int n0, int n1, int n2) {
  const long long a = (long long)nr[1] * nr[2], b = (long long)nr[0] * nr[2], c = (long long)nr[0] * nr[1];
  const long long lhs = 4 * ((long long)n0 * n0 * a * a + (long long)n1 * n1 * b * b + (long long)n2 * n2 * c * c);
  const long long tot = (long long)nr[0] * nr[1] * nr[2];
  return lhs > tot * tot;
}

__device__ __forceinline__ int sym_freq(int k, int n) { return (k >= (n + 1) / 2) ? k - n : k; }

template <typename T>
struct EpiParams {
  const T* V;               // [N] local potential
  T vshift;                 // added to V (1/2 |k+A|^2 when the Fourier mask is on)
  const cplx<T>* base;      // optional [N][ld_base]
  long ld_base;
  cplx<T> alpha, beta;      // out = alpha * H in + beta * base
};

// One cell of the persistent batch launch (batch.h): every argument the three tile
// passes of its H apply take, as launch_h_impl derives them.
template <typename T>
struct BatchCell {
  const cplx<T>* in;
  long ld_in;
  cplx<T>* out;
  long ld_out;
  int M, ysplit, acc_cap, rec_cap_a, rec_cap_inv, seg_cap, vin, vio;
  cplx<T>* tmp;
  const cplx<T>* tw;  // x | y | z twiddles
  ProjView<T> pj;
  KinParams<T> kp;
  EpiParams<T> ep;
};

}  // namespace inqb

#include "tiles.cuh"

namespace inqb {

// ---------------------------------------------------------------- launch
inline bool aligned16(const void* p, long ld, size_t esz) {
  return ((uintptr_t)p % 16 == 0) && ((ld * (long)esz) % 16 == 0);
}

template <typename T, int NX, int NY, int NZ>
int launch_h_impl(const LaunchArgs& a) {
  using TG = TileGeom<T, NX, NY, NZ>;
  constexpr int GT = TG::G;
  // the kernels' shared-memory limits, set once per device (contexts on several host
  // threads may launch for the first time together)
  static std::once_flag attr_once[64];
  int dev = 0;
  INQB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 64) return fail(INQB_ERR_UNSUPPORTED, "device index above 63");
  int attr_rc = INQB_OK;
  std::call_once(attr_once[dev], [&attr_rc] {
    attr_rc = [] {
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_fwd<T, NX, NY, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)std::min(TG::smem_fwd(kAccAtomsMax, kRecCapMax), TG::SMEM_MAX)));
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_x<T, NX, NY, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)TG::SMEM_X));
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_x_fft<T, NX, NY, NZ, 0>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TG::SMEM_X));
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_x_fft<T, NX, NY, NZ, 1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TG::SMEM_X));
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_inv<T, NX, NY, NZ, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)std::min(TG::smem_inv(kRecCapMax, kAccAtomsMax), TG::SMEM_MAX)));
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_inv<T, NX, NY, NZ, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)TG::smem_inv(0, 0)));
      return (int)INQB_OK;
    }();
  });
  if (attr_rc != INQB_OK) return attr_rc;
  const cplx<T>* tw = reinterpret_cast<const cplx<T>*>(a.tw);
  const cplx<T>* twx = tw;
  const cplx<T>* twy = tw + NX;
  const cplx<T>* twz = tw + NX + NY;
  cplx<T>* tmp = reinterpret_cast<cplx<T>*>(a.tmp);
  cudaStream_t st = (cudaStream_t)a.stream;
  const size_t esz = sizeof(cplx<T>);
  const int tgroups = (a.M + GT - 1) / GT;
  // 16-byte vectors of G orbitals: full groups, aligned pointers and leading dimensions
  const int vin = aligned16(a.in, a.ld_in, esz);
  const int vout = aligned16(a.out, a.ld_out, esz);
  int ysplit = a.ysplit > 0 ? a.ysplit : TG::YSPLIT;
  if (TG::Y1 % ysplit != 0) return fail(INQB_ERR_INVALID, "schedule: ysplit must divide the tiles per plane");
  // compiled defaults: 256 threads per CTA, except the x-line pass in FP64, which the
  // autotuner measured faster with 128 (64^3: 295 -> 258 us)
  const int thr_default[3] = {TG::THREADS, sizeof(T) == 8 ? 128 : TG::THREADS, TG::THREADS};
  int thr[3];
  for (int k = 0; k < 3; k++) {
    thr[k] = a.threads[k] > 0 ? a.threads[k] : thr_default[k];
    if (thr[k] % 32 != 0 || thr[k] < 64 || thr[k] > TG::THREADS)
      return fail(INQB_ERR_INVALID, "schedule: threads per CTA must be a multiple of 32 in [64, 256]");
  }
  const dim3 gfwd(tgroups, NX * ysplit), gx(TG::Y2 * NZ, tgroups), ginv(tgroups, NX * TG::Y1);

  ProjView<T> pj = *reinterpret_cast<const ProjView<T>*>(a.proj_view);
  KinParams<T> kp;
  for (int d = 0; d < 3; d++) {
    for (int c = 0; c < 3; c++) kp.b[d][c] = (T)a.rlat[d][c];
    kp.kA[d] = (T)a.kA_cart[d];
  }
  kp.scale = (T)(1.0 / ((double)NX * NY * NZ));
  kp.mask = a.fourier_mask;
  const double kA2 = a.kA_cart[0] * a.kA_cart[0] + a.kA_cart[1] * a.kA_cart[1] + a.kA_cart[2] * a.kA_cart[2];
  kp.shift = (T)(0.5 * kA2 / ((double)NX * NY * NZ));
  kp.nr[0] = NX;
  kp.nr[1] = NY;
  kp.nr[2] = NZ;
  kp.pois = (T)0;

  if (a.mode == LaunchArgs::H) {
    // the KB projection: its own deterministic kernel (project.cu) where the tables and
    // the block's alignment allow, else fused into the first tile pass with FP64 atomics
    const bool sep = pj.nproj > 0 && pj.proj_mode == 1 && pj.pc_table != nullptr &&
                     project_supported(sizeof(T) == 8 ? INQB_FP64 : INQB_MIXED, a.in, a.ld_in);
    ProjView<T> pjA = pj;
    if (sep) pjA.nproj = 0;
    const int acc_cap = pjA.nproj > 0 ? std::min(pj.max_plane_atoms, kAccAtomsMax) : 0;
    const int seg_cap = pj.nproj > 0 ? std::min(pj.max_tile_seg, kAccAtomsMax) : 0;
    // stage a tile's records only when all of them fit beside the tile (the kernel
    // reads them from global memory otherwise)
    int rec_cap = (pj.nproj > 0 && pj.max_tile_ent <= kRecCapMax) ? pj.max_tile_ent : 0;
    const int rec_cap_fwd = pjA.nproj > 0 ? rec_cap : 0;
    if (TG::smem_fwd(acc_cap, rec_cap) > TG::SMEM_MAX) rec_cap = 0;
    const int rec_cap_a = (TG::smem_fwd(acc_cap, rec_cap_fwd) > TG::SMEM_MAX) ? 0 : rec_cap_fwd;
    if (pj.nproj > 0 && pj.pt_stride != TG::PSTRIDE)
      return fail(INQB_ERR_INVALID, "projector tables were built for another tiling of this grid");
    EpiParams<T> ep;
    ep.V = (const T*)a.V;
    ep.vshift = a.fourier_mask ? (T)(0.5 * kA2) : (T)0;
    ep.base = (const cplx<T>*)a.base;
    ep.ld_base = a.ld_base;
    ep.alpha = mk<T>((T)a.alpha[0], (T)a.alpha[1]);
    ep.beta = mk<T>((T)a.beta[0], (T)a.beta[1]);
    // pass C stages the records in shared memory only in FP64 (where the orbital
    // prefetch already limits it to two CTAs per SM); in FP32 the smem is worth more
    // as a fourth CTA per SM, and the epilogue prefetches records into registers
    int rec_cap_inv = TG::PREFETCH ? rec_cap : 0;
    if (TG::smem_inv(rec_cap_inv, seg_cap) > TG::SMEM_MAX) rec_cap_inv = 0;
    if (TG::smem_inv(rec_cap_inv, seg_cap) > TG::SMEM_MAX)
      return fail(INQB_ERR_UNSUPPORTED, "tile of this grid does not fit in shared memory");
    if (a.batch_cell) {
      // describe the apply for the persistent batch launch instead of launching it
      auto* d = reinterpret_cast<BatchCellDesc*>(a.batch_cell);
      d->kind = batch_kind(NX, NY, NZ);
      if (d->kind < 0) return fail(INQB_ERR_UNSUPPORTED, "grid not compiled into the persistent batch kernel");
      if (sep || (pj.nproj > 0 && pj.slots == nullptr) || a.fourier_out || a.base)
        return fail(INQB_ERR_UNSUPPORTED, "the persistent batch launch runs the fused projection only");
      BatchCell<T> c;
      c.in = (const cplx<T>*)a.in;
      c.ld_in = a.ld_in;
      c.out = (cplx<T>*)a.out;
      c.ld_out = a.ld_out;
      c.M = a.M;
      c.ysplit = ysplit;
      c.acc_cap = acc_cap;
      c.rec_cap_a = rec_cap_a;
      c.rec_cap_inv = rec_cap_inv;
      c.seg_cap = seg_cap;
      c.vin = vin;
      c.vio = vin && vout;
      c.tmp = tmp;
      c.tw = tw;
      c.pj = pj;
      c.kp = kp;
      c.ep = ep;
      d->groups = tgroups;
      d->a_per = NX * ysplit;
      d->b_per = TG::Y2 * NZ;
      d->c_per = NX * TG::Y1;
      d->finish = pj.nproj > 0 ? 1 : 0;
      d->smem = std::max({TG::smem_fwd(acc_cap, rec_cap_a), TG::SMEM_X, TG::smem_inv(rec_cap_inv, seg_cap)});
      d->bytes.resize(sizeof(c));
      memcpy(d->bytes.data(), &c, sizeof(c));
      return INQB_OK;
    }
    if (a.events[0]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[0], st));
    if (sep) {
      INQB_TRY(launch_project(sizeof(T) == 8 ? INQB_FP64 : INQB_MIXED, a.in, a.ld_in, a.M, pj.nproj, pj.L,
                              pj.pc_ptr, pj.pc_pt, pj.pc_table, pj.scale, pj.proj, pj.err, st));
    } else if (pj.nproj > 0 && pj.slots == nullptr) {
      INQB_CUDA_TRY(cudaMemsetAsync(pj.proj, 0, sizeof(double2) * (size_t)pj.nproj * pj.L * a.M, st));
    }
    if (a.events[1]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[1], st));
    if (a.events[2]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[2], st));
    k_tile_fwd<T, NX, NY, NZ><<<gfwd, thr[0], TG::smem_fwd(acc_cap, rec_cap_a), st>>>(
        (const cplx<T>*)a.in, a.ld_in, a.M, tmp, twy, twz, pjA, acc_cap, rec_cap_a, ysplit, vin);
    if (a.events[3]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[3], st));
    // the second pass also adds the fused projection's partial sums per atom, in a
    // fixed order (its first CTAs; the third pass reads the result)
    ProjView<T> fin = pj;
    if (sep || pj.nproj == 0) fin.slots = nullptr;
    k_tile_x<T, NX, NY, NZ><<<gx, thr[1], TG::SMEM_X, st>>>(tmp, twx, kp, (cplx<T>*)a.fourier_out, fin, a.M,
                                                             ysplit);
    if (a.events[4]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[4], st));
    k_tile_inv<T, NX, NY, NZ, 1><<<ginv, thr[2], TG::smem_inv(rec_cap_inv, seg_cap), st>>>(
        tmp, (const cplx<T>*)a.in, a.ld_in, (cplx<T>*)a.out, a.ld_out, a.M, twy, twz, pj, ep, rec_cap_inv, seg_cap,
        vin && vout);
    if (a.events[5]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[5], st));
  } else if (a.mode == LaunchArgs::POISSON) {
    // solvers::poisson on M complex fields: forward z and inner y, then the outer y
    // and x transforms with the 4 pi / (N |G|^2) factor, then the inverse (no 1/N:
    // the factor holds it)
    ProjView<T> none = pj;
    none.nproj = 0;
    k_tile_fwd<T, NX, NY, NZ><<<gfwd, thr[0], TG::smem_fwd(0, 0), st>>>(
        (const cplx<T>*)a.in, a.ld_in, a.M, tmp, twy, twz, none, 0, 0, ysplit, vin);
    KinParams<T> kq = kp;
    for (int d = 0; d < 3; d++) kq.kA[d] = (T)0;
    kq.scale = (T)1;
    kq.mask = 0;
    kq.shift = (T)0;
    kq.pois = (T)(2.0 * M_PI / ((double)NX * NY * NZ));
    ProjView<T> nofin = pj;
    nofin.slots = nullptr;
    k_tile_x<T, NX, NY, NZ><<<gx, thr[1], TG::SMEM_X, st>>>(tmp, twx, kq, nullptr, nofin, 0, 1);
    EpiParams<T> ep{};
    ep.alpha = mk<T>((T)1, (T)0);
    k_tile_inv<T, NX, NY, NZ, 0><<<ginv, thr[2], TG::smem_inv(0, 0), st>>>(
        tmp, nullptr, 0, (cplx<T>*)a.out, a.ld_out, a.M, twy, twz, none, ep, 0, 0, vout);
  } else if (a.mode == LaunchArgs::FFT_FWD) {
    ProjView<T> none = pj;
    none.nproj = 0;
    k_tile_fwd<T, NX, NY, NZ><<<gfwd, thr[0], TG::smem_fwd(0, 0), st>>>(
        (const cplx<T>*)a.in, a.ld_in, a.M, tmp, twy, twz, none, 0, 0, ysplit, vin);
    k_tile_x_fft<T, NX, NY, NZ, 0><<<gx, thr[1], TG::SMEM_X, st>>>(tmp, nullptr, (cplx<T>*)a.out, a.ld_out,
                                                                       a.M, twx, vout);
  } else {
    k_tile_x_fft<T, NX, NY, NZ, 1><<<gx, thr[1], TG::SMEM_X, st>>>(tmp, (const cplx<T>*)a.in, nullptr, a.ld_in,
                                                                       a.M, twx, vin);
    EpiParams<T> ep{};
    ep.alpha = mk<T>(kp.scale, (T)0);
    ProjView<T> none = pj;
    none.nproj = 0;
    k_tile_inv<T, NX, NY, NZ, 0><<<ginv, thr[2], TG::smem_inv(0, 0), st>>>(
        tmp, nullptr, 0, (cplx<T>*)a.out, a.ld_out, a.M, twy, twz, none, ep, 0, 0, vout);
  }
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

// ---------------------------------------------------------------- registry
template <typename T, int NX, int NY, int NZ>
inline Plan make_plan() {
  Plan p;
  p.G = TileGeom<T, NX, NY, NZ>::G;
  p.G_tile = TileGeom<T, NX, NY, NZ>::G;
  p.y1 = TileGeom<T, NX, NY, NZ>::Y1;
  p.y2 = TileGeom<T, NX, NY, NZ>::Y2;
  p.ysplit = TileGeom<T, NX, NY, NZ>::YSPLIT;
  p.launch = &launch_h_impl<T, NX, NY, NZ>;
  return p;
}

#define INQB_CUBIC(N) {std::make_tuple(N, N, N, 0), make_plan<double, N, N, N>()}, \
                      {std::make_tuple(N, N, N, 1), make_plan<float, N, N, N>()},
#define INQB_GRID(X, Y, Z) {std::make_tuple(X, Y, Z, 0), make_plan<double, X, Y, Z>()}, \
                           {std::make_tuple(X, Y, Z, 1), make_plan<float, X, Y, Z>()},

using GridRegistry = std::map<std::tuple<int, int, int, int>, Plan>;

}  // namespace inqb
