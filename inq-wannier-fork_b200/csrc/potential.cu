// Kernels of the density -> potential step (src/hamiltonian/self_consistency.hpp:89-160)
// and of the ETRS step with self-consistency (src/real_time/etrs.hpp:22-82):
//
//   pack      rho (FP64) -> complex field of the context precision, the Poisson input
//   ks        V = vion + Re V_H + v_xc[max(rho, 0)] into the context's potential, with
//             per-block FP64 partial sums of rho vion, rho V_H, e_xc n and rho v_xc
//   absdiff   per-block partial sums of |a - b| (operations::integral_sum_absdiff,
//             src/operations/integral.hpp:113-126)
//   finish    one block adds the partials in a fixed order, so every sum is
//             deterministic
//   shift2    a1 += c1 y, a2 += c2 y: the two accumulators of
//             operations::exponential_2_for_1 (src/operations/exponential.hpp:50-69)
//   broyden   the vector passes of mixers::broyden (src/mixers/broyden.hpp:107-160),
//             the density mixer of the self-consistent Crank-Nicolson step: the
//             differences, up to 16 dot products in a fixed order, the update with
//             the sum for observables::density::normalize, and scalings
//
// The exchange-correlation functional is evaluated in FP64 in both precisions (it is
// one pass over N points).  libxc, which the reference calls for it
// (src/hamiltonian/xc_term.hpp:276-287), is not part of the reference snapshot; the
// two LDA functionals are restated from their publications:
//   XC_LDA_X     Dirac-Slater exchange: e_x = -(3/4) (3/pi)^(1/3) n^(1/3),
//                v_x = -(3 n / pi)^(1/3) for an unpolarised density;
//   XC_LDA_C_PZ  Perdew and Zunger, Phys. Rev. B 23, 5048 (1981), the unpolarised
//                Ceperley-Alder fit: rs >= 1: e_c = g / (1 + b1 sqrt(rs) + b2 rs),
//                rs < 1: e_c = A ln rs + B + C rs ln rs + D rs, v_c = e_c - rs/3 de_c/drs.
// Densities below 1e-15 give e = v = 0.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "dft.cuh"
#include "inqb_internal.h"
#include "potential.h"

namespace inqb {

namespace {

constexpr int kThreads = 256;
constexpr double kDensThreshold = 1e-15;
// Perdew-Zunger unpolarised parameters (their Table XII)
constexpr double kPZg = -0.1423, kPZb1 = 1.0529, kPZb2 = 0.3334;
constexpr double kPZa = 0.0311, kPZb = -0.048, kPZc = 0.0020, kPZd = -0.0116;

__device__ __forceinline__ void lda_unpolarised(double n, double& e, double& v) {
  e = 0.0;
  v = 0.0;
  if (!(n >= kDensThreshold)) return;
  // exchange, with spin densities n / 2: e = -(3/4) (6/pi)^(1/3) (n/2)^(1/3)
  const double cx = cbrt(6.0 / M_PI);
  const double ns13 = cbrt(0.5 * n);
  e = -0.75 * cx * ns13;
  v = -cx * ns13;
  // correlation
  const double rs = cbrt(3.0 / (4.0 * M_PI * n));
  double ec, dec;
  if (rs >= 1.0) {
    const double sr = sqrt(rs), den = 1.0 + kPZb1 * sr + kPZb2 * rs;
    ec = kPZg / den;
    dec = -kPZg * (0.5 * kPZb1 / sr + kPZb2) / (den * den);
  } else {
    const double lr = log(rs);
    ec = kPZa * lr + kPZb + kPZc * rs * lr + kPZd * rs;
    dec = kPZa / rs + kPZc * (lr + 1.0) + kPZd;
  }
  e += ec;
  v += ec - rs / 3.0 * dec;
}

// Sums NS values over the block (warp shuffles, then the warps in shared memory)
// and writes them to out[0..NS) from thread 0.
template <int NS>
__device__ __forceinline__ void block_sum_store(double (&v)[NS], double* out) {
  __shared__ double red[kThreads / 32][NS];
#pragma unroll
  for (int k = 0; k < NS; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NS; ++k) red[w][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double s = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i][k];
      out[k] = s;
    }
  }
}

template <typename T>
__global__ void k_pack_density(const double* __restrict__ rho, cplx<T>* __restrict__ out, long N) {
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long)gridDim.x * blockDim.x)
    out[p] = mk<T>((T)rho[p], (T)0);
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
    k_ks_potential(const double* __restrict__ rho, const double* __restrict__ vion, const cplx<T>* __restrict__ vh,
                   int theory, long N, T* __restrict__ V, double* __restrict__ partial) {
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long)gridDim.x * blockDim.x) {
    const double r = rho[p];
    const double vi = vion ? vion[p] : 0.0;
    double v = vi;
    s[0] += r * vi;
    if (theory >= 1 && vh) {
      const double h = (double)vh[p].x;
      v += h;
      s[1] += r * h;
    }
    if (theory >= 2) {
      double e, vx;
      const double n = fmax(r, 0.0);
      lda_unpolarised(n, e, vx);
      v += vx;
      s[2] += e * n;
      s[3] += r * vx;
    }
    V[p] = (T)v;
  }
  block_sum_store<4>(s, partial + 4 * (long)blockIdx.x);
}

__global__ void __launch_bounds__(kThreads)
    k_absdiff(const double* __restrict__ a, const double* __restrict__ b, long N, double* __restrict__ partial) {
  double s[1] = {0.0};
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long)gridDim.x * blockDim.x)
    s[0] += fabs(a[i] - b[i]);
  block_sum_store<1>(s, partial + blockIdx.x);
}

// out[k] = sum_b partial[b * ns + k], one block, fixed order
__global__ void __launch_bounds__(kThreads) k_finish(const double* __restrict__ partial, int nblk, int ns,
                                                     double* __restrict__ out) {
  for (int k = 0; k < ns; ++k) {
    double s[1] = {0.0};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) s[0] += partial[(long)b * ns + k];
    block_sum_store<1>(s, out + k);
    __syncthreads();
  }
}

template <typename T>
__global__ void k_shift2(const cplx<T>* __restrict__ y, long ldy, cplx<T>* __restrict__ a1, long ld1,
                         cplx<T>* __restrict__ a2, long ld2, int M, long N, double c1r, double c1i, double c2r,
                         double c2i) {
  const long total = N * M;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long p = i / M;
    const int m = (int)(i - p * M);
    const cplx<T> v = y[p * ldy + m];
    const double vx = v.x, vy = v.y;
    cplx<T>& u = a1[p * ld1 + m];
    u.x = (T)((double)u.x + c1r * vx - c1i * vy);
    u.y = (T)((double)u.y + c1r * vy + c1i * vx);
    cplx<T>& w = a2[p * ld2 + m];
    w.x = (T)((double)w.x + c2r * vx - c2i * vy);
    w.y = (T)((double)w.y + c2r * vy + c2i * vx);
  }
}

// ---- Broyden density mixer (src/mixers/broyden.hpp:107-160), FP64 vectors of n values

// ff = vout - vin, kept in f_old (the reference sets f_old = ff after using the old
// value); with a ring slot, df = ff - f_old and dv = vin - vin_old first; vin_old = vin.
__global__ void __launch_bounds__(kThreads)
    k_broyden_diff(const double* __restrict__ vin, const double* __restrict__ vout, double* __restrict__ f_old,
                   double* __restrict__ vin_old, double* __restrict__ df, double* __restrict__ dv, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double x = vin[i], f = vout[i] - x;
    if (df) {
      df[i] = f - f_old[i];
      dv[i] = x - vin_old[i];
    }
    f_old[i] = f;
    vin_old[i] = x;
  }
}

// per-block partial sums of a_k . b_k for k < nd
__global__ void __launch_bounds__(kThreads) k_dots(DotList d, int nd, long n, double* __restrict__ partial) {
  double s[kMaxDots];
#pragma unroll
  for (int k = 0; k < kMaxDots; ++k) s[k] = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < kMaxDots; ++k)
      if (k < nd) s[k] += d.a[k][i] * d.b[k][i];
  }
  block_sum_store<kMaxDots>(s, partial + (long)kMaxDots * blockIdx.x);
}

__global__ void k_scale2(double* __restrict__ x, double* __restrict__ y, double s, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    x[i] *= s;
    y[i] *= s;
  }
}

// vin += mix ff - sum_k c_k (mix df_k + dv_k) (broyden_extrapolation, broyden.hpp:95-101),
// with per-block partial sums of the new vin
__global__ void __launch_bounds__(kThreads)
    k_broyden_update(double* __restrict__ vin, const double* __restrict__ ff, const double* __restrict__ df,
                     const double* __restrict__ dv, long n, int used, BroydenCoef c, double mix,
                     double* __restrict__ partial) {
  double s[1] = {0.0};
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double v = vin[i] + mix * ff[i];
#pragma unroll
    for (int k = 0; k < kMaxBroyden; ++k)
      if (k < used) v -= c.c[k] * (mix * df[(long)k * n + i] + dv[(long)k * n + i]);
    vin[i] = v;
    s[0] += v;
  }
  block_sum_store<1>(s, partial + blockIdx.x);
}

__global__ void k_scale(double* __restrict__ x, double s, long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] *= s;
}

int grid_for(long n) { return (int)std::max<long>(1, std::min<long>((n + kThreads - 1) / kThreads, kPotBlocks)); }

}  // namespace

int launch_pack_density(int precision, const double* rho, void* out, long N, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == INQB_FP64)
    k_pack_density<double><<<grid_for(N), kThreads, 0, st>>>(rho, (cplx<double>*)out, N);
  else
    k_pack_density<float><<<grid_for(N), kThreads, 0, st>>>(rho, (cplx<float>*)out, N);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_ks_potential(int precision, const double* rho, const double* vion, const void* vh, int theory, long N,
                        void* V, double* partial, double* sums, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = grid_for(N);
  if (precision == INQB_FP64)
    k_ks_potential<double><<<nb, kThreads, 0, st>>>(rho, vion, (const cplx<double>*)vh, theory, N, (double*)V,
                                                     partial);
  else
    k_ks_potential<float><<<nb, kThreads, 0, st>>>(rho, vion, (const cplx<float>*)vh, theory, N, (float*)V,
                                                    partial);
  INQB_CUDA_TRY(cudaGetLastError());
  k_finish<<<1, kThreads, 0, st>>>(partial, nb, 4, sums);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_absdiff(const double* a, const double* b, long N, double* partial, double* sum, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = grid_for(N);
  k_absdiff<<<nb, kThreads, 0, st>>>(a, b, N, partial);
  INQB_CUDA_TRY(cudaGetLastError());
  k_finish<<<1, kThreads, 0, st>>>(partial, nb, 1, sum);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_shift2(int precision, const void* y, long ldy, void* a1, long ld1, void* a2, long ld2, int M, long N,
                  const double c1[2], const double c2[2], void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const long total = N * M;
  const int nb = (int)std::max<long>(1, std::min<long>((total + kThreads - 1) / kThreads, 148L * 32));
  if (precision == INQB_FP64)
    k_shift2<double><<<nb, kThreads, 0, st>>>((const cplx<double>*)y, ldy, (cplx<double>*)a1, ld1,
                                               (cplx<double>*)a2, ld2, M, N, c1[0], c1[1], c2[0], c2[1]);
  else
    k_shift2<float><<<nb, kThreads, 0, st>>>((const cplx<float>*)y, ldy, (cplx<float>*)a1, ld1,
                                              (cplx<float>*)a2, ld2, M, N, c1[0], c1[1], c2[0], c2[1]);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_broyden_diff(const double* vin, const double* vout, double* f_old, double* vin_old, double* df,
                        double* dv, long n, void* stream) {
  if ((df == nullptr) != (dv == nullptr)) return fail(INQB_ERR_INVALID, "Broyden ring slot: df and dv together");
  k_broyden_diff<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(vin, vout, f_old, vin_old, df, dv, n);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_dots(const DotList& d, int nd, long n, double* partial, double* out, void* stream) {
  if (nd < 1 || nd > kMaxDots) return fail(INQB_ERR_INVALID, "launch_dots: 1 to 16 products");
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = grid_for(n);
  k_dots<<<nb, kThreads, 0, st>>>(d, nd, n, partial);
  INQB_CUDA_TRY(cudaGetLastError());
  k_finish<<<1, kThreads, 0, st>>>(partial, nb, kMaxDots, out);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_scale2(double* x, double* y, double s, long n, void* stream) {
  k_scale2<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(x, y, s, n);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_broyden_update(double* vin, const double* ff, const double* df, const double* dv, long n, int used,
                          const BroydenCoef& c, double mix, double* partial, double* sum, void* stream) {
  if (used < 0 || used > kMaxBroyden) return fail(INQB_ERR_INVALID, "Broyden update: 0 to 8 ring slots");
  cudaStream_t st = (cudaStream_t)stream;
  const int nb = grid_for(n);
  k_broyden_update<<<nb, kThreads, 0, st>>>(vin, ff, df, dv, n, used, c, mix, partial);
  INQB_CUDA_TRY(cudaGetLastError());
  k_finish<<<1, kThreads, 0, st>>>(partial, nb, 1, sum);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_scale(double* x, double s, long n, void* stream) {
  k_scale<<<grid_for(n), kThreads, 0, (cudaStream_t)stream>>>(x, s, n);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

}  // namespace inqb
