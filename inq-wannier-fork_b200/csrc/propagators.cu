// Kernels of the Crank-Nicolson step (src/real_time/crank_nicolson.hpp:22-114):
// the per-orbital reductions and the update of solvers::steepest_descent
// (src/solvers/steepest_descent.hpp:22-80) without preconditioner.
//
//   sums     acc[4m..4m+3] = dV sum_p (|hsd|^2, conj(r) hsd (re, im), |r|^2)
//   update   lambda_m = cc / qq from those sums, phi += lambda_m r, normres[m] = |cc|
//
// Both run on the device, so a sweep of five steps needs no host round trip.
#include <cuda_runtime.h>

#include <algorithm>

#include "dft.cuh"
#include "inqb_internal.h"
#include "propagators.h"

namespace inqb {

// Block: 32 orbitals (lanes) x 8 point lanes; the point lanes' partial sums meet in
// shared memory, then one FP64 atomic per orbital and sum.
template <typename T>
__global__ void __launch_bounds__(256)
    k_sd_sums(const cplx<T>* __restrict__ r, const cplx<T>* __restrict__ hsd, long ld, int M, long N,
              long pts_per_block, double* __restrict__ acc) {
  __shared__ double red[8][32][5];
  const int tm = threadIdx.x & 31, tp = threadIdx.x >> 5;
  const int m = blockIdx.y * 32 + tm;
  const long p0 = (long)blockIdx.x * pts_per_block, p1 = min(N, p0 + pts_per_block);
  double hh = 0.0, rhr = 0.0, rhi = 0.0, rr = 0.0;
  if (m < M) {
    for (long p = p0 + tp; p < p1; p += 8) {
      const cplx<T> a = r[p * ld + m], b = hsd[p * ld + m];
      const double ax = a.x, ay = a.y, bx = b.x, by = b.y;
      hh += bx * bx + by * by;
      rhr += ax * bx + ay * by;
      rhi += ax * by - ay * bx;
      rr += ax * ax + ay * ay;
    }
  }
  red[tp][tm][0] = hh;
  red[tp][tm][1] = rhr;
  red[tp][tm][2] = rhi;
  red[tp][tm][3] = rr;
  __syncthreads();
  if (tp < 4 && m < M) {
    double v = 0.0;
    for (int k = 0; k < 8; k++) v += red[k][tm][tp];
    atomicAdd(&acc[4 * m + tp], v);
  }
}

// The step length of steepest_descent.hpp:48-58 in complex FP64: ca = <hsd|hsd>,
// cb = 4 Re <r|hsd>, cc = <r|r> (all times dV); qq = -(cb + sign sqrt(cb^2 - 4 ca cc)) / 2
// with the sign of Re(conj(cb) (cb^2 - 4 ca cc)); lambda = cc / qq.
__device__ __forceinline__ double2 sd_lambda(const double* a, double dV, double* normres) {
  const double ca = dV * a[0];
  const double cb = 4.0 * dV * a[1];
  const double cc = dV * a[3];
  *normres = fabs(cc);
  // ca and cc are exact norms, so in the reference's complex arithmetic the
  // discriminant cb^2 - 4 ca cc is real with imaginary part -0 (a real minus a
  // complex with +0 imaginary part); its principal square root is sqrt(disc) or,
  // below zero, -i sqrt(-disc) (C99 csqrt takes the sign of the imaginary zero)
  const double disc = cb * cb - 4.0 * ca * cc;
  const double signb = (cb * disc >= 0.0) ? 1.0 : -1.0;
  double qr, qi;
  if (disc >= 0.0) {
    qr = -0.5 * (cb + signb * sqrt(disc));
    qi = 0.0;
  } else {
    qr = -0.5 * cb;
    qi = 0.5 * signb * sqrt(-disc);
  }
  const double den = qr * qr + qi * qi;
  return make_double2(cc * qr / den, -cc * qi / den);
}

template <typename T>
__global__ void k_sd_update(cplx<T>* __restrict__ phi, long ldp, const cplx<T>* __restrict__ r, long ldr, int M,
                            long N, const double* __restrict__ acc, double dV, double* __restrict__ normres) {
  const long total = N * M;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long p = i / M;
    const int m = (int)(i - p * M);
    double nr;
    const double2 lam = sd_lambda(acc + 4 * m, dV, &nr);
    if (p == 0) normres[m] = nr;
    const cplx<T> rv = r[p * ldr + m];
    cplx<T>& d = phi[p * ldp + m];
    d.x = (T)((double)d.x + lam.x * rv.x - lam.y * rv.y);
    d.y = (T)((double)d.y + lam.x * rv.y + lam.y * rv.x);
  }
}

template <typename T>
static int sd_sums_impl(const void* r, const void* hsd, long ld, int M, long N, double* acc, cudaStream_t st) {
  INQB_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * 4 * (size_t)M, st));
  const int ym = (M + 31) / 32;
  const long nblk = std::max<long>(1, std::min<long>(N / 64 + 1, 148L * 8 / ym + 1));
  const long per = (N + nblk - 1) / nblk;
  k_sd_sums<T><<<dim3((unsigned)((N + per - 1) / per), ym), 256, 0, st>>>(
      (const cplx<T>*)r, (const cplx<T>*)hsd, ld, M, N, per, acc);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_sd_sums(int precision, const void* r, const void* hsd, long ld, int M, long N, double* acc,
                   void* stream) {
  return precision == INQB_FP64 ? sd_sums_impl<double>(r, hsd, ld, M, N, acc, (cudaStream_t)stream)
                                : sd_sums_impl<float>(r, hsd, ld, M, N, acc, (cudaStream_t)stream);
}

template <typename T>
static int sd_update_impl(void* phi, long ldp, const void* r, long ldr, int M, long N, const double* acc, double dV,
                          double* normres, cudaStream_t st) {
  const long total = N * M;
  const int blocks = (int)std::min<long>((total + 255) / 256, 148L * 32);
  k_sd_update<T><<<blocks, 256, 0, st>>>((cplx<T>*)phi, ldp, (const cplx<T>*)r, ldr, M, N, acc, dV, normres);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_sd_update(int precision, void* phi, long ldp, const void* r, long ldr, int M, long N, const double* acc,
                     double dV, double* normres, void* stream) {
  return precision == INQB_FP64
             ? sd_update_impl<double>(phi, ldp, r, ldr, M, N, acc, dV, normres, (cudaStream_t)stream)
             : sd_update_impl<float>(phi, ldp, r, ldr, M, N, acc, dV, normres, (cudaStream_t)stream);
}

}  // namespace inqb
