// Observables and FP64 orbital linear algebra on the device:
//   density   rho[p] = sum_m occ[m] |psi[p][m]|^2       (src/observables/density.hpp:23-33)
//   dipole    dV sum_p r_p rho[p]                         (src/observables/dipole.hpp:23-40)
//   overlap   S = dV psi^H psi, FP64 accumulation         (src/operations/overlap.hpp:41)
//   cholesky  S = U^H U, U upper                          (src/matrix/cholesky.hpp:28-89)
//   rotate    psi <- psi U^-1                             (src/operations/rotate.hpp:147-157)
// Input orbitals may be complex64 (mixed) or complex128; every sum is FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "dft.cuh"
#include "inqb_internal.h"
#include "observables.h"

namespace inqb {

template <typename T>
__global__ void k_density(const cplx<T>* __restrict__ psi, long ld, int M, long N, const double* __restrict__ occ,
                          double* __restrict__ rho) {
  const int lane = threadIdx.x & 31;
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
  for (long p = warp; p < N; p += nwarps) {
    double acc = 0.0;
    for (int m = lane; m < M; m += 32) {
      const cplx<T> v = psi[p * ld + m];
      acc += occ[m] * ((double)v.x * (double)v.x + (double)v.y * (double)v.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) rho[p] = acc;
  }
}

struct LatticeView {
  double lat[3][3];
  int nr[3];
};

__device__ __forceinline__ void rvector(const LatticeView& g, long p, double r[3]) {
  const int nyz = g.nr[1] * g.nr[2];
  int ii[3] = {(int)(p / nyz), (int)((p / g.nr[2]) % g.nr[1]), (int)(p % g.nr[2])};
  double c[3];
  for (int d = 0; d < 3; d++) {
    int s = (ii[d] >= (g.nr[d] + 1) / 2) ? ii[d] - g.nr[d] : ii[d];
    c[d] = s * (1.0 / g.nr[d]);
  }
  for (int k = 0; k < 3; k++) r[k] = g.lat[0][k] * c[0] + g.lat[1][k] * c[1] + g.lat[2][k] * c[2];
}

__global__ void k_dipole(const double* __restrict__ rho, long N, LatticeView g, double* __restrict__ out) {
  double acc[3] = {0, 0, 0};
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long)gridDim.x * blockDim.x) {
    double r[3];
    rvector(g, p, r);
    const double d = rho[p];
    for (int k = 0; k < 3; k++) acc[k] += r[k] * d;
  }
  __shared__ double red[3][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < 3; k++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    if (lane == 0) red[k][warp] = acc[k];
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    for (int k = 0; k < 3; k++) {
      double v = lane < nw ? red[k][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) atomicAdd(&out[k], v);
    }
  }
}

// S[i][j] += dV sum_{p in chunk} conj(a[p][i]) b[p][j] ; 32x32 tile per CTA.  The
// square overlap passes the same block twice; an orbital-sharded caller passes two
// blocks (one block of operations::overlap's set-parallel branch).
template <typename T>
__global__ void __launch_bounds__(1024) k_overlap(const cplx<T>* __restrict__ pa, long lda, int Ma,
                                                  const cplx<T>* __restrict__ pb_, long ldb, int Mb, long N,
                                                  long chunk, double dV, double2* __restrict__ S, long lds) {
  constexpr int TP = 32;  // points staged per round
  __shared__ double2 a[TP][33], b[TP][33];
  const int ti = threadIdx.y, tj = threadIdx.x;
  const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
  const long p0 = (long)blockIdx.z * chunk, p1 = min(N, p0 + chunk);
  double re = 0.0, im = 0.0;
  for (long pb = p0; pb < p1; pb += TP) {
    // thread (ti, tj) loads point pb+ti, orbital i0+tj of a / j0+tj of b
    const long p = pb + ti;
    double2 va = make_double2(0, 0), vb = make_double2(0, 0);
    if (p < p1) {
      if (i0 + tj < Ma) {
        cplx<T> v = pa[p * lda + i0 + tj];
        va = make_double2(v.x, v.y);
      }
      if (j0 + tj < Mb) {
        cplx<T> v = pb_[p * ldb + j0 + tj];
        vb = make_double2(v.x, v.y);
      }
    }
    a[ti][tj] = va;
    b[ti][tj] = vb;
    __syncthreads();
#pragma unroll 8
    for (int q = 0; q < TP; q++) {
      const double2 x = a[q][ti], y = b[q][tj];
      re += x.x * y.x + x.y * y.y;
      im += x.x * y.y - x.y * y.x;
    }
    __syncthreads();
  }
  if (i0 + ti < Ma && j0 + tj < Mb) {
    atomicAdd(&S[(long)(i0 + ti) * lds + j0 + tj].x, dV * re);
    atomicAdd(&S[(long)(i0 + ti) * lds + j0 + tj].y, dV * im);
  }
}

// In-place Cholesky of the Hermitian S (upper triangle used): on exit the upper
// triangle holds U with S = U^H U.  One CTA; info[0] = first failing pivot + 1.
__global__ void __launch_bounds__(1024) k_cholesky(double2* __restrict__ S, int M, long lds, int* __restrict__ info) {
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int k = 0; k < M; k++) {
    __syncthreads();
    const double d = S[(long)k * lds + k].x;
    if (!(d > 0.0)) {
      if (threadIdx.x == 0) {
        bad = 1;
        info[0] = k + 1;
      }
      __syncthreads();
      return;
    }
    const double u = sqrt(d);
    __syncthreads();
    for (int j = k + threadIdx.x; j < M; j += blockDim.x) {
      double2 v = S[(long)k * lds + j];
      S[(long)k * lds + j] = j == k ? make_double2(u, 0.0) : make_double2(v.x / u, v.y / u);
    }
    __syncthreads();
    // trailing update: S[i][j] -= conj(U[k][i]) U[k][j], k < i <= j
    const int n = M - k - 1;
    for (long t = threadIdx.x; t < (long)n * n; t += blockDim.x) {
      const int i = k + 1 + (int)(t / n), j = k + 1 + (int)(t % n);
      if (j < i) continue;
      const double2 ui = S[(long)k * lds + i], uj = S[(long)k * lds + j];
      double2 s = S[(long)i * lds + j];
      s.x -= ui.x * uj.x + ui.y * uj.y;
      s.y -= ui.x * uj.y - ui.y * uj.x;
      S[(long)i * lds + j] = s;
    }
  }
  (void)bad;
}

// X = U^-1 (upper triangular), one thread per column j, back substitution.
__global__ void k_triangular_inverse(const double2* __restrict__ U, int M, long ldu, double2* __restrict__ X) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  for (int i = 0; i < M; i++) X[(long)i * M + j] = make_double2(0, 0);
  for (int i = j; i >= 0; i--) {
    double2 s = make_double2(i == j ? 1.0 : 0.0, 0.0);
    for (int k = i + 1; k <= j; k++) {
      const double2 u = U[(long)i * ldu + k], x = X[(long)k * M + j];
      s.x -= u.x * x.x - u.y * x.y;
      s.y -= u.x * x.y + u.y * x.x;
    }
    const double uii = U[(long)i * ldu + i].x;
    X[(long)i * M + j] = make_double2(s.x / uii, s.y / uii);
  }
}

// psi[p][:] <- psi[p][:] X  (X upper triangular), FP64 arithmetic, in place.
template <typename T>
__global__ void k_rotate_upper(cplx<T>* __restrict__ psi, long ld, int M, long N, const double2* __restrict__ X) {
  extern __shared__ double2 row[];
  for (long p = blockIdx.x; p < N; p += gridDim.x) {
    __syncthreads();
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
      const cplx<T> v = psi[p * ld + m];
      row[m] = make_double2(v.x, v.y);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
      double re = 0.0, im = 0.0;
      for (int i = 0; i <= j; i++) {
        const double2 a = row[i], x = X[(long)i * M + j];
        re += a.x * x.x - a.y * x.y;
        im += a.x * x.y + a.y * x.x;
      }
      psi[p * ld + j] = mk<T>((T)re, (T)im);
    }
  }
}

// out[p][j] = sum_{i < Ma} a[p][i] R[i][j], j < Mo: one block of operations::rotate's
// set-parallel branch (src/operations/rotate.hpp:100-125), FP64 arithmetic, a row of a
// staged in shared memory per point.
template <typename T>
__global__ void k_rotate_block(const cplx<T>* __restrict__ a, long lda, int Ma, const double2* __restrict__ R,
                               long ldr, int Mo, cplx<T>* __restrict__ out, long ldo, long N) {
  extern __shared__ double2 row[];
  for (long p = blockIdx.x; p < N; p += gridDim.x) {
    __syncthreads();
    for (int m = threadIdx.x; m < Ma; m += blockDim.x) {
      const cplx<T> v = a[p * lda + m];
      row[m] = make_double2(v.x, v.y);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < Mo; j += blockDim.x) {
      double re = 0.0, im = 0.0;
      for (int i = 0; i < Ma; i++) {
        const double2 x = row[i], r = R[(long)i * ldr + j];
        re += x.x * r.x - x.y * r.y;
        im += x.x * r.y + x.y * r.x;
      }
      out[p * ldo + j] = mk<T>((T)re, (T)im);
    }
  }
}

// ---------------------------------------------------------------- launchers
template <typename T>
static int density_impl(const void* psi, long ld, int M, long N, const double* occ, double* rho, cudaStream_t st) {
  const int blocks = (int)std::min<long>((N * 32 + 255) / 256, 148L * 16);
  k_density<T><<<blocks, 256, 0, st>>>((const cplx<T>*)psi, ld, M, N, occ, rho);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_density(int precision, const void* psi, long ld, int M, long N, const double* occ, double* rho,
                   void* stream) {
  return precision == INQB_FP64 ? density_impl<double>(psi, ld, M, N, occ, rho, (cudaStream_t)stream)
                                : density_impl<float>(psi, ld, M, N, occ, rho, (cudaStream_t)stream);
}

// acc[3 m .. 3 m + 2] += (Re, Im) sum_p conj(hpsi) psi and sum_p |psi|^2 over this
// block's points (overlap_diagonal.hpp:118-127).  Block: 32 orbitals (lanes) x 8
// point lanes, reduced in shared memory before one FP64 atomic per orbital and sum.
template <typename T>
__global__ void __launch_bounds__(256)
    k_band_sums(const cplx<T>* __restrict__ psi, const cplx<T>* __restrict__ hpsi, long ld, int M, long N,
                long pts_per_block, double* __restrict__ acc) {
  __shared__ double red[8][32][3];
  const int tm = threadIdx.x & 31, tp = threadIdx.x >> 5;
  const int m = blockIdx.y * 32 + tm;
  const long p0 = (long)blockIdx.x * pts_per_block, p1 = min(N, p0 + pts_per_block);
  double vr = 0.0, vi = 0.0, nn = 0.0;
  if (m < M) {
    for (long p = p0 + tp; p < p1; p += 8) {
      const cplx<T> a = hpsi[p * ld + m], b = psi[p * ld + m];
      const double ax = a.x, ay = a.y, bx = b.x, by = b.y;
      vr += ax * bx + ay * by;
      vi += ax * by - ay * bx;
      nn += bx * bx + by * by;
    }
  }
  red[tp][tm][0] = vr;
  red[tp][tm][1] = vi;
  red[tp][tm][2] = nn;
  __syncthreads();
  if (tp < 3 && m < M) {
    double v = 0.0;
    for (int k = 0; k < 8; k++) v += red[k][tm][tp];
    atomicAdd(&acc[3 * m + tp], v);
  }
}

template <typename T>
static int band_sums_impl(const void* psi, const void* hpsi, long ld, int M, long N, double* acc, cudaStream_t st) {
  INQB_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * 3 * (size_t)M, st));
  const int ym = (M + 31) / 32;
  // about 8 blocks per SM over the points
  const long nblk = std::max<long>(1, std::min<long>(N / 64 + 1, 148L * 8 / ym + 1));
  const long per = (N + nblk - 1) / nblk;
  k_band_sums<T><<<dim3((unsigned)((N + per - 1) / per), ym), 256, 0, st>>>(
      (const cplx<T>*)psi, (const cplx<T>*)hpsi, ld, M, N, per, acc);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_band_sums(int precision, const void* psi, const void* hpsi, long ld, int M, long N, double* acc,
                     void* stream) {
  return precision == INQB_FP64 ? band_sums_impl<double>(psi, hpsi, ld, M, N, acc, (cudaStream_t)stream)
                                : band_sums_impl<float>(psi, hpsi, ld, M, N, acc, (cudaStream_t)stream);
}

int launch_dipole(const double* rho, long N, const double lat[3][3], const int nr[3], double* out_dev,
                  void* stream) {
  LatticeView g;
  for (int i = 0; i < 3; i++) {
    g.nr[i] = nr[i];
    for (int j = 0; j < 3; j++) g.lat[i][j] = lat[i][j];
  }
  cudaStream_t st = (cudaStream_t)stream;
  INQB_CUDA_TRY(cudaMemsetAsync(out_dev, 0, 3 * sizeof(double), st));
  const int blocks = (int)std::min<long>((N + 255) / 256, 148L * 4);
  k_dipole<<<blocks, 256, 0, st>>>(rho, N, g, out_dev);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

template <typename T>
static int orthonormalize_impl(void* psi, long ld, int M, long N, double dV, double2* S, double2* X, int* info,
                               cudaStream_t st) {
  INQB_CUDA_TRY(cudaMemsetAsync(S, 0, sizeof(double2) * (size_t)M * M, st));
  INQB_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int), st));
  const int tiles = (M + 31) / 32;
  long nchunks = std::max<long>(1, std::min<long>(N / 1024, (148L * 8) / (tiles * tiles) + 1));
  const long chunk = (N + nchunks - 1) / nchunks;
  nchunks = (N + chunk - 1) / chunk;
  k_overlap<T><<<dim3(tiles, tiles, (unsigned)nchunks), dim3(32, 32), 0, st>>>(
      (const cplx<T>*)psi, ld, M, (const cplx<T>*)psi, ld, M, N, chunk, dV, S, M);
  INQB_CUDA_TRY(cudaGetLastError());
  k_cholesky<<<1, 1024, 0, st>>>(S, M, M, info);
  INQB_CUDA_TRY(cudaGetLastError());
  int h_info = 0;
  INQB_CUDA_TRY(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_info != 0)
    return fail(INQB_ERR_NOT_POSITIVE_DEFINITE,
                "overlap matrix is not positive definite at pivot " + std::to_string(h_info - 1));
  k_triangular_inverse<<<(M + 127) / 128, 128, 0, st>>>(S, M, M, X);
  INQB_CUDA_TRY(cudaGetLastError());
  const int blocks = (int)std::min<long>(N, 148L * 16);
  k_rotate_upper<T><<<blocks, 128, sizeof(double2) * M, st>>>((cplx<T>*)psi, ld, M, N, X);
  INQB_CUDA_TRY(cudaGetLastError());
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  return INQB_OK;
}

int launch_orthonormalize(int precision, void* psi, long ld, int M, long N, double dV, double2* S, double2* X,
                          int* info, void* stream) {
  return precision == INQB_FP64
             ? orthonormalize_impl<double>(psi, ld, M, N, dV, S, X, info, (cudaStream_t)stream)
             : orthonormalize_impl<float>(psi, ld, M, N, dV, S, X, info, (cudaStream_t)stream);
}

// ---------------------------------------------------------------- orbital-sharded orthonormalisation
// The pieces of operations::orthogonalize over a states communicator: blocks of the
// overlap, the Cholesky factor's inverse of the summed matrix, and blocks of the
// rotation.  The caller moves the blocks between ranks.
template <typename T>
static int overlap_block_impl(const void* a, long lda, int Ma, const void* b, long ldb, int Mb, long N, double dV,
                              double2* S, long lds, cudaStream_t st) {
  INQB_CUDA_TRY(cudaMemset2DAsync(S, sizeof(double2) * lds, 0, sizeof(double2) * Mb, Ma, st));
  const int ti = (Ma + 31) / 32, tj = (Mb + 31) / 32;
  long nchunks = std::max<long>(1, std::min<long>(N / 1024, (148L * 8) / (ti * tj) + 1));
  const long chunk = (N + nchunks - 1) / nchunks;
  nchunks = (N + chunk - 1) / chunk;
  k_overlap<T><<<dim3(tj, ti, (unsigned)nchunks), dim3(32, 32), 0, st>>>((const cplx<T>*)a, lda, Ma,
                                                                          (const cplx<T>*)b, ldb, Mb, N, chunk, dV,
                                                                          S, lds);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_overlap_block(int precision, const void* a, long lda, int Ma, const void* b, long ldb, int Mb, long N,
                         double dV, double2* S, long lds, void* stream) {
  return precision == INQB_FP64
             ? overlap_block_impl<double>(a, lda, Ma, b, ldb, Mb, N, dV, S, lds, (cudaStream_t)stream)
             : overlap_block_impl<float>(a, lda, Ma, b, ldb, Mb, N, dV, S, lds, (cudaStream_t)stream);
}

int launch_cholesky_inverse(double2* S, int M, long lds, double2* X, int* info, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  INQB_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int), st));
  k_cholesky<<<1, 1024, 0, st>>>(S, M, lds, info);
  INQB_CUDA_TRY(cudaGetLastError());
  int h_info = 0;
  INQB_CUDA_TRY(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_info != 0)
    return fail(INQB_ERR_NOT_POSITIVE_DEFINITE,
                "overlap matrix is not positive definite at pivot " + std::to_string(h_info - 1));
  k_triangular_inverse<<<(M + 127) / 128, 128, 0, st>>>(S, M, lds, X);
  INQB_CUDA_TRY(cudaGetLastError());
  INQB_CUDA_TRY(cudaMemcpy2DAsync(S, sizeof(double2) * lds, X, sizeof(double2) * M, sizeof(double2) * M, M,
                                  cudaMemcpyDeviceToDevice, st));
  INQB_CUDA_TRY(cudaStreamSynchronize(st));
  return INQB_OK;
}

template <typename T>
static int rotate_block_impl(const void* a, long lda, int Ma, const double2* R, long ldr, int Mo, void* out,
                             long ldo, long N, cudaStream_t st) {
  const int blocks = (int)std::min<long>(N, 148L * 16);
  k_rotate_block<T><<<blocks, 128, sizeof(double2) * Ma, st>>>((const cplx<T>*)a, lda, Ma, R, ldr, Mo,
                                                               (cplx<T>*)out, ldo, N);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_rotate_block(int precision, const void* a, long lda, int Ma, const double2* R, long ldr, int Mo,
                        void* out, long ldo, long N, void* stream) {
  return precision == INQB_FP64
             ? rotate_block_impl<double>(a, lda, Ma, R, ldr, Mo, out, ldo, N, (cudaStream_t)stream)
             : rotate_block_impl<float>(a, lda, Ma, R, ldr, Mo, out, ldo, N, (cudaStream_t)stream);
}

// ---------------------------------------------------------------- orthonormalisation without allocation
// The same kernels as launch_orthonormalize, with their scratch (overlap S, inverse
// factor X, pivot status) taken from a fixed array in device memory rather than from
// cudaMalloc, for callers that may not allocate device memory.
namespace {
constexpr size_t kNoAllocMat = (size_t)kOrthoNoAllocMaxStates * kOrthoNoAllocMaxStates;
// S (M x M) | X (M x M) | status: 2 MiB plus a little, held by every GPU that loads
// the library until the process exits.  All calls on a device share it.
static __device__ __align__(256) double2 g_orth_scratch[2 * kNoAllocMat + 16];
std::mutex g_orth_scratch_mutex;
double2* g_orth_scratch_ptr[64] = {};
}  // namespace

int orthonormalize_noalloc(int precision, int device, void* psi, long ld, int M, long N, double dV, void* stream) {
  if (M > kOrthoNoAllocMaxStates)
    return fail(INQB_ERR_UNSUPPORTED, "allocation-free orthonormalisation takes at most " +
                                          std::to_string(kOrthoNoAllocMaxStates) + " orbitals, got " +
                                          std::to_string(M));
  if (device < 0 || device >= 64) return fail(INQB_ERR_INVALID, "device index out of range");
  double2* base = nullptr;
  {
    // once per device, with that device current: the device address of the array
    std::lock_guard<std::mutex> lock(g_orth_scratch_mutex);
    if (!g_orth_scratch_ptr[device]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_orth_scratch);
      if (e != cudaSuccess)
        return fail(INQB_ERR_CUDA, std::string("cudaGetSymbolAddress of the orthonormalisation scratch: ") +
                                       cudaGetErrorString(e));
      g_orth_scratch_ptr[device] = static_cast<double2*>(p);
    }
    base = g_orth_scratch_ptr[device];
  }
  // launch_orthonormalize zeroes S and the status before accumulating into them
  return launch_orthonormalize(precision, psi, ld, M, N, dV, base, base + kNoAllocMat,
                               reinterpret_cast<int*>(base + 2 * kNoAllocMat), stream);
}

}  // namespace inqb
