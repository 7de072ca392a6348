// Building blocks of the discrete adjoint of the ETRS propagator.
//
//   axpby        y <- a x + b y on orbital blocks
//   position     lambda <- s occ[m] r_d(p) psi      (d dipole / d psi*, dipole.hpp:23-40)
//   V gradient   gV[p] += Re(c sum_m conj(u) w)      (<u| dH/dV(p) |w>, H's local term)
//   A gradient   gA[d] += Re(c <u| dH/dA_d |w>)      kinetic (G + k + A)_d in Fourier space
//                plus the nonlocal position commutator i S [conj(p_u) r_w - conj(r_u) p_w]
//                (the structure of projector_all::position_commutator,
//                src/hamiltonian/projector_all.hpp:319-403).
// All sums are FP64 whatever the orbital precision.
#include <cuda_runtime.h>

#include "adjoint.h"
#include "dft.cuh"
#include "inqb_internal.h"

namespace inqb {

template <typename T>
__global__ void k_axpby(long N, int M, cplx<T> a, const cplx<T>* __restrict__ x, long ldx, cplx<T> b,
                        cplx<T>* __restrict__ y, long ldy) {
  const long total = N * M;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long p = i / M;
    const int m = (int)(i - p * M);
    cplx<T>& dst = y[p * ldy + m];
    const cplx<T> xv = x[p * ldx + m];
    dst = a * xv + b * dst;
  }
}

struct Lat {
  double lat[3][3];
  int nr[3];
};

__device__ __forceinline__ double rcomp(const Lat& g, long p, int d) {
  const int nyz = g.nr[1] * g.nr[2];
  const int ii[3] = {(int)(p / nyz), (int)((p / g.nr[2]) % g.nr[1]), (int)(p % g.nr[2])};
  double c[3];
  for (int k = 0; k < 3; k++) {
    const int s = (ii[k] >= (g.nr[k] + 1) / 2) ? ii[k] - g.nr[k] : ii[k];
    c[k] = s * (1.0 / g.nr[k]);
  }
  return g.lat[0][d] * c[0] + g.lat[1][d] * c[1] + g.lat[2][d] * c[2];
}

template <typename T>
__global__ void k_position_scale(long N, int M, const cplx<T>* __restrict__ psi, long ld, cplx<T>* __restrict__ out,
                                 long ldo, Lat g, int d, const double* __restrict__ occ, double s) {
  const long total = N * M;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long p = i / M;
    const int m = (int)(i - p * M);
    const double f = s * occ[m] * rcomp(g, p, d);
    const cplx<T> v = psi[p * ld + m];
    out[p * ldo + m] = mk<T>((T)(f * (double)v.x), (T)(f * (double)v.y));
  }
}

// gV[p] += Re(c sum_m conj(u) w), one warp per grid point.
template <typename T>
__global__ void k_vgrad(long N, int M, const cplx<T>* __restrict__ u, const cplx<T>* __restrict__ w, long ld,
                        double cre, double cim, double* __restrict__ gV) {
  const int lane = threadIdx.x & 31;
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
  for (long p = warp; p < N; p += nwarps) {
    double re = 0.0, im = 0.0;
    for (int m = lane; m < M; m += 32) {
      const cplx<T> a = u[p * ld + m], b = w[p * ld + m];
      re += (double)a.x * b.x + (double)a.y * b.y;
      im += (double)a.x * b.y - (double)a.y * b.x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      re += __shfl_xor_sync(0xffffffffu, re, o);
      im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) gV[p] += cre * re - cim * im;
  }
}

struct Recip {
  double b[3][3];
  double kA[3];
  int nr[3];
  int mask;
};

// acc[2d..2d+1] += sum_{G,m} conj(U) (G + kA)_d W   (U, W forward FFTs, natural order)
template <typename T>
__global__ void k_velocity_dot(long N, int M, const cplx<T>* __restrict__ U, const cplx<T>* __restrict__ W, long ld,
                               Recip r, double* __restrict__ acc) {
  double s[6] = {0, 0, 0, 0, 0, 0};
  const int nyz = r.nr[1] * r.nr[2];
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N * M; i += (long)gridDim.x * blockDim.x) {
    const long p = i / M;
    const int m = (int)(i - p * M);
    const int k[3] = {(int)(p / nyz), (int)((p / r.nr[2]) % r.nr[1]), (int)(p % r.nr[2])};
    double n[3];
    for (int c = 0; c < 3; c++) n[c] = (k[c] >= (r.nr[c] + 1) / 2) ? k[c] - r.nr[c] : k[c];
    // with the mask, the Laplacian term P(1/2 g^2 + kA.G)P drops its G outside the sphere
    // while the 1/2|kA|^2 shift stays: the derivative there is kA alone
    double gf = 1.0;
    if (r.mask) {
      const long long a0 = (long long)r.nr[1] * r.nr[2], a1 = (long long)r.nr[0] * r.nr[2],
                      a2 = (long long)r.nr[0] * r.nr[1];
      const long long tot = (long long)r.nr[0] * r.nr[1] * r.nr[2];
      const long long i0 = (long long)n[0], i1 = (long long)n[1], i2 = (long long)n[2];
      if (4 * (i0 * i0 * a0 * a0 + i1 * i1 * a1 * a1 + i2 * i2 * a2 * a2) > tot * tot) gf = 0.0;
    }
    const cplx<T> a = U[p * ld + m], b = W[p * ld + m];
    const double re = (double)a.x * b.x + (double)a.y * b.y;
    const double im = (double)a.x * b.y - (double)a.y * b.x;
    for (int d = 0; d < 3; d++) {
      const double v = gf * (n[0] * r.b[0][d] + n[1] * r.b[1][d] + n[2] * r.b[2][d]) + r.kA[d];
      s[2 * d] += v * re;
      s[2 * d + 1] += v * im;
    }
  }
  __shared__ double red[6][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = 0; q < 6; q++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
    if (lane == 0) red[q][warp] = s[q];
  }
  __syncthreads();
  if (warp == 0) {
    for (int q = 0; q < 6; q++) {
      double v = lane < (int)(blockDim.x >> 5) ? red[q][lane] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) atomicAdd(&acc[q], v);
    }
  }
}

// Nonlocal part of <u| dH/dA_d |w> per atom: one thread per orbital walks the
// atom's sphere entries; acc[6 + 2d..] += sum_l S_l i [conj(p_u) r_w,d - conj(r_u,d) p_w].
template <typename T>
__global__ void k_nl_dA(int nproj, int L, int M, const cplx<T>* __restrict__ u, const cplx<T>* __restrict__ w,
                        long ld, const int* __restrict__ atom_ptr, const int* __restrict__ atom_ent,
                        const int* __restrict__ ent_pt, const double* __restrict__ ent_xyz,
                        const T* __restrict__ ent_beta, const cplx<T>* __restrict__ phase,
                        const double* __restrict__ scale, double* __restrict__ acc) {
  constexpr int LM = 4;
  const int a = blockIdx.x;
  const int m = blockIdx.y * blockDim.x + threadIdx.x;
  double out[6] = {0, 0, 0, 0, 0, 0};
  if (m < M) {
    double pu[LM][2] = {}, pw[LM][2] = {}, ru[LM][3][2] = {}, rw[LM][3][2] = {};
    for (int i = atom_ptr[a]; i < atom_ptr[a + 1]; i++) {
      const int e = atom_ent[i];
      const long pt = ent_pt[e];
      const cplx<T> ph = phase[e];
      const cplx<T> uu = u[pt * ld + m], ww = w[pt * ld + m];
      // phase * value in FP64
      const double ur = (double)ph.x * uu.x - (double)ph.y * uu.y, ui = (double)ph.x * uu.y + (double)ph.y * uu.x;
      const double wr = (double)ph.x * ww.x - (double)ph.y * ww.y, wi = (double)ph.x * ww.y + (double)ph.y * ww.x;
      const double x[3] = {ent_xyz[3 * e], ent_xyz[3 * e + 1], ent_xyz[3 * e + 2]};
      for (int l = 0; l < L && l < LM; l++) {
        const double b = (double)ent_beta[(long)e * L + l];
        pu[l][0] += b * ur;
        pu[l][1] += b * ui;
        pw[l][0] += b * wr;
        pw[l][1] += b * wi;
        for (int d = 0; d < 3; d++) {
          ru[l][d][0] += b * x[d] * ur;
          ru[l][d][1] += b * x[d] * ui;
          rw[l][d][0] += b * x[d] * wr;
          rw[l][d][1] += b * x[d] * wi;
        }
      }
    }
    for (int l = 0; l < L && l < LM; l++) {
      const double S = scale[a * L + l];
      for (int d = 0; d < 3; d++) {
        // z1 = conj(pu) rw, z2 = conj(ru) pw, result += S i (z1 - z2)
        const double z1r = pu[l][0] * rw[l][d][0] + pu[l][1] * rw[l][d][1];
        const double z1i = pu[l][0] * rw[l][d][1] - pu[l][1] * rw[l][d][0];
        const double z2r = ru[l][d][0] * pw[l][0] + ru[l][d][1] * pw[l][1];
        const double z2i = ru[l][d][0] * pw[l][1] - ru[l][d][1] * pw[l][0];
        out[2 * d] += -S * (z1i - z2i);
        out[2 * d + 1] += S * (z1r - z2r);
      }
    }
  }
  for (int q = 0; q < 6; q++) {
    double v = out[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&acc[6 + q], v);
  }
}

// gA[d] += Re(c (kin[d] / N + nl[d]))
__global__ void k_finish_dA(const double* __restrict__ acc, double invN, double cre, double cim,
                            double* __restrict__ gA) {
  const int d = threadIdx.x;
  if (d < 3) {
    const double re = acc[2 * d] * invN + acc[6 + 2 * d];
    const double im = acc[2 * d + 1] * invN + acc[6 + 2 * d + 1];
    gA[d] += cre * re - cim * im;
  }
}

// ---------------------------------------------------------------- launchers
static int grid_for(long n, int threads) { return (int)std::min<long>((n + threads - 1) / threads, 148L * 32); }

template <typename T>
static int axpby_impl(long N, int M, const double a[2], const void* x, long ldx, const double b[2], void* y, long ldy,
                      cudaStream_t st) {
  k_axpby<T><<<grid_for(N * M, 256), 256, 0, st>>>(N, M, mk<T>((T)a[0], (T)a[1]), (const cplx<T>*)x, ldx,
                                                   mk<T>((T)b[0], (T)b[1]), (cplx<T>*)y, ldy);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_axpby(int precision, long N, int M, const double a[2], const void* x, long ldx, const double b[2], void* y,
                 long ldy, void* stream) {
  return precision == INQB_FP64 ? axpby_impl<double>(N, M, a, x, ldx, b, y, ldy, (cudaStream_t)stream)
                                : axpby_impl<float>(N, M, a, x, ldx, b, y, ldy, (cudaStream_t)stream);
}

int launch_position_scale(int precision, const inqb_ctx& ctx, const void* psi, long ld, void* out, long ldo, int M,
                          int dir, const double* occ, double s, void* stream) {
  Lat g;
  for (int i = 0; i < 3; i++) {
    g.nr[i] = ctx.nr[i];
    for (int j = 0; j < 3; j++) g.lat[i][j] = ctx.cell.lat[i][j];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long n = ctx.N * M;
  if (precision == INQB_FP64)
    k_position_scale<double><<<grid_for(n, 256), 256, 0, st>>>(ctx.N, M, (const cplx<double>*)psi, ld,
                                                               (cplx<double>*)out, ldo, g, dir, occ, s);
  else
    k_position_scale<float><<<grid_for(n, 256), 256, 0, st>>>(ctx.N, M, (const cplx<float>*)psi, ld,
                                                              (cplx<float>*)out, ldo, g, dir, occ, s);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_vgrad(int precision, long N, int M, const void* u, const void* w, long ld, double cre, double cim,
                 double* gV, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const int blocks = (int)std::min<long>((N * 32 + 255) / 256, 148L * 16);
  if (precision == INQB_FP64)
    k_vgrad<double><<<blocks, 256, 0, st>>>(N, M, (const cplx<double>*)u, (const cplx<double>*)w, ld, cre, cim, gV);
  else
    k_vgrad<float><<<blocks, 256, 0, st>>>(N, M, (const cplx<float>*)u, (const cplx<float>*)w, ld, cre, cim, gV);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

template <typename T>
static int agrad_impl(const inqb_ctx& ctx, const void* U, const void* W, const void* u, const void* w, long ld, int M,
                      double* acc, double cre, double cim, double* gA, cudaStream_t st) {
  Recip r;
  for (int i = 0; i < 3; i++) {
    r.nr[i] = ctx.nr[i];
    for (int j = 0; j < 3; j++) r.b[i][j] = ctx.cell.rlat[i][j];
  }
  ctx.cell.cov_to_cart(ctx.kA_cov, r.kA);
  r.mask = ctx.fourier_mask;
  INQB_CUDA_TRY(cudaMemsetAsync(acc, 0, 12 * sizeof(double), st));
  k_velocity_dot<T><<<grid_for(ctx.N * M, 256), 256, 0, st>>>(ctx.N, M, (const cplx<T>*)U, (const cplx<T>*)W, M, r,
                                                             acc);
  INQB_CUDA_TRY(cudaGetLastError());
  const ProjTables& t = ctx.proj;
  if (t.nproj > 0) {
    dim3 grid(t.nproj, (M + 31) / 32);
    k_nl_dA<T><<<grid, 32, 0, st>>>(t.nproj, t.L, M, (const cplx<T>*)u, (const cplx<T>*)w, ld,
                                    t.d_atom_ptr.as<int>(), t.d_atom_ent.as<int>(), t.d_ent_pt.as<int>(),
                                    t.d_ent_xyz.as<double>(), t.d_ent_beta.as<T>(),
                                    (const cplx<T>*)t.d_ent_phase.ptr, t.d_scale.as<double>(), acc);
    INQB_CUDA_TRY(cudaGetLastError());
  }
  k_finish_dA<<<1, 32, 0, st>>>(acc, 1.0 / (double)ctx.N, cre, cim, gA);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_agrad(const inqb_ctx& ctx, const void* U, const void* W, const void* u, const void* w, long ld, int M,
                 double* acc, double cre, double cim, double* gA, void* stream) {
  return ctx.precision == INQB_FP64
             ? agrad_impl<double>(ctx, U, W, u, w, ld, M, acc, cre, cim, gA, (cudaStream_t)stream)
             : agrad_impl<float>(ctx, U, W, u, w, ld, M, acc, cre, cim, gA, (cudaStream_t)stream);
}

}  // namespace inqb
