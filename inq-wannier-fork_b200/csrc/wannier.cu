// TD-MLWF: the Wannier transformation applied after each real-time step
// (src/observables/mlwf_properties.hpp:28-44, src/wannier/tdmlwf_trans.hpp,
// src/wannier/jade_complex.hpp).
//
//   gram     split over points: Z_d[m][n] = sum_p conj(psi_m) e^{i theta_d} psi_n for the
//            three directions (theta_d = 2 pi r_d / |a_d|), one partial per slab of points
//            (FP64 slabs in FP64; FP32 slabs of 1024 points in the mixed precision)
//   finish   sum of the slabs, normalisation 1/(|psi_m| |psi_n|), and the six matrices
//            of tdmlwf_trans::update: cos = (Z + Z^H)/2, sin = (Z - Z^H)/(2i)
//   jade     one CTA per pair and rotation step: the 18 pair elements, the 3 x 3
//            Jacobi eigenproblem, the plane rotation of the pair's rows of the six
//            matrices and of u, and the step's change of the traces.  The reference
//            multiplies dense M x M rotation matrices (7 GEMMs per step); the pairs are
//            disjoint, so rotating two rows per pair is the same product in O(M) per pair.
//   adiag    adiag[k][i] = sum_j conj(a_k[i][j]) u[i][j]
//   rotate   psi <- psi u^H (operations::rotate), tiled through shared memory
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "dft.cuh"
#include "inqb_internal.h"
#include "wannier.h"

namespace inqb {

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// ------------------------------------------------------------------ gram
// 256 threads as 16 x 16; thread (tm, tn) holds outputs m = m0 + tm + 16 a (a < TMX),
// n = n0 + tn + 16 b (b < TNX) for the three directions; CTA tile (16 TMX) x (16 TNX).
// FP64 contexts accumulate in FP64 over the CTA's slab (few slabs).  The mixed context
// accumulates FP32 products in FP32 over a slab of at most kSlabF32 points and keeps one
// FP32 partial per slab; the finish kernel adds the slabs in FP64 (the FP32 rounding of
// a slab sum is about 6e-8 sqrt(kSlabF32) of its size, about 1e-7 of the total after the
// FP64 sum over slabs).  Freeing the FP64 registers lets the FP32 tile be 4 x 2.
constexpr long kSlabF32 = 1024;    // points per slab in the mixed precision

struct GramGeom {
  int nr[3];
  double frac_to_theta[3][3];  // theta_d / pi = sum_j f_j frac_to_theta[d][j]
};

template <typename T>
struct GramCfg;
template <>
struct GramCfg<double> {
  static constexpr int TMX = 2, TNX = 2, GP = 16, MINB = 2;  // GP: points per staged chunk
  using P = double2;                                         // partial type
};
template <>
struct GramCfg<float> {
  static constexpr int TMX = 4, TNX = 2, GP = 32, MINB = 3;
  using P = float2;
};

__device__ __forceinline__ void store_partial(double2* p, double x, double y) { *p = make_double2(x, y); }
__device__ __forceinline__ void store_partial(float2* p, float x, float y) { *p = make_float2(x, y); }

// grid (tiles_m * tiles_n, nslab)
template <typename T>
__global__ void __launch_bounds__(256, GramCfg<T>::MINB)
    k_mlwf_gram(const cplx<T>* __restrict__ pa, long lda, int Ma, const cplx<T>* __restrict__ pb, long ldb, int Mb,
                long N, GramGeom geo, long pts_per_slab, typename GramCfg<T>::P* __restrict__ partial) {
  using R = T;
  constexpr int TMX = GramCfg<T>::TMX, TNX = GramCfg<T>::TNX, kGP = GramCfg<T>::GP;
  constexpr int TILE_M = 16 * TMX, TILE_N = 16 * TNX;
  __shared__ cplx<R> sA[kGP][TILE_M];
  __shared__ cplx<R> sB[3][kGP][TILE_N];
  __shared__ cplx<R> sW[3][kGP];
  const int tiles_m = (Ma + TILE_M - 1) / TILE_M;
  const int m0 = (blockIdx.x % tiles_m) * TILE_M, n0 = (blockIdx.x / tiles_m) * TILE_N;
  const long p_beg = (long)blockIdx.y * pts_per_slab, p_end = min(N, p_beg + pts_per_slab);
  const int tm = threadIdx.x % 16, tn = threadIdx.x / 16;
  R acc[3][TMX][TNX][2];
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int a = 0; a < TMX; ++a)
#pragma unroll
      for (int b = 0; b < TNX; ++b) acc[d][a][b][0] = acc[d][a][b][1] = (R)0;
  for (long pc = p_beg; pc < p_end; pc += kGP) {
    // weights of the chunk's points, e^{i theta_d}
    if (threadIdx.x < kGP) {
      const long p = pc + threadIdx.x;
      cplx<R> w[3] = {mk<R>(0, 0), mk<R>(0, 0), mk<R>(0, 0)};
      if (p < p_end) {
        const int iz = (int)(p % geo.nr[2]), iy = (int)((p / geo.nr[2]) % geo.nr[1]),
                  ix = (int)(p / ((long)geo.nr[1] * geo.nr[2]));
        const int id[3] = {ix, iy, iz};
        double f[3];
        for (int j = 0; j < 3; ++j) {
          const int sy = (id[j] >= (geo.nr[j] + 1) / 2) ? id[j] - geo.nr[j] : id[j];
          f[j] = (double)sy / geo.nr[j];
        }
        for (int d = 0; d < 3; ++d) {
          const double th = geo.frac_to_theta[d][0] * f[0] + geo.frac_to_theta[d][1] * f[1] +
                            geo.frac_to_theta[d][2] * f[2];
          double sn, cs;
          sincospi(th, &sn, &cs);
          w[d] = mk<R>((R)cs, (R)sn);
        }
      }
      for (int d = 0; d < 3; ++d) sW[d][threadIdx.x] = w[d];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kGP * TILE_M; i += blockDim.x) {
      const int q = i / TILE_M, j = i % TILE_M;
      const long p = pc + q;
      sA[q][j] = (p < p_end && m0 + j < Ma) ? pa[p * lda + m0 + j] : mk<R>(0, 0);
    }
    for (int i = threadIdx.x; i < kGP * TILE_N; i += blockDim.x) {
      const int q = i / TILE_N, j = i % TILE_N;
      const long p = pc + q;
      const cplx<R> vb = (p < p_end && n0 + j < Mb) ? pb[p * ldb + n0 + j] : mk<R>(0, 0);
#pragma unroll
      for (int d = 0; d < 3; ++d) sB[d][q][j] = sW[d][q] * vb;
    }
    __syncthreads();
#pragma unroll 2
    for (int q = 0; q < kGP; ++q) {
      cplx<R> av[TMX];
#pragma unroll
      for (int a = 0; a < TMX; ++a) av[a] = sA[q][tm + 16 * a];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        cplx<R> bv[TNX];
#pragma unroll
        for (int b = 0; b < TNX; ++b) bv[b] = sB[d][q][tn + 16 * b];
#pragma unroll
        for (int a = 0; a < TMX; ++a)
#pragma unroll
          for (int b = 0; b < TNX; ++b) {
            // conj(a) * b
            acc[d][a][b][0] = fma(av[a].x, bv[b].x, fma(av[a].y, bv[b].y, acc[d][a][b][0]));
            acc[d][a][b][1] = fma(av[a].x, bv[b].y, fma(-av[a].y, bv[b].x, acc[d][a][b][1]));
          }
      }
    }
    __syncthreads();
  }
  // partial[slab][d][m][n], m < Ma, n < Mb
  const size_t MM = (size_t)Ma * Mb;
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int a = 0; a < TMX; ++a)
#pragma unroll
      for (int b = 0; b < TNX; ++b) {
        const int m = m0 + tm + 16 * a, n = n0 + tn + 16 * b;
        if (m < Ma && n < Mb)
          store_partial(&partial[((size_t)blockIdx.y * 3 + d) * MM + (size_t)m * Mb + n], acc[d][a][b][0],
                        acc[d][a][b][1]);
      }
}

// Z[e] = sum over the slabs of partial[slab][e] in FP64, e = (d, m, n): the slabs' sums
// in slab order, reads coalesced along e, eight slabs in flight per thread.
template <typename P>
__global__ void k_mlwf_slab_sum(const P* __restrict__ partial, int nslab, long n, double2* __restrict__ Z) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    double zx = 0.0, zy = 0.0;
    for (int s0 = 0; s0 < nslab; s0 += 8) {
      P v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = (s0 + u < nslab) ? partial[(size_t)(s0 + u) * n + e] : P{0, 0};
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        zx += (double)v[u].x;
        zy += (double)v[u].y;
      }
    }
    Z[e] = make_double2(zx, zy);
  }
}

// a[2d][m][n] = (Z + Z^H)/2, a[2d+1][m][n] = (Z - Z^H)/(2i), Z the slab sum (FP64) divided
// by |psi_m| |psi_n|: norms[ns m + ns - 1] = sum_p |psi_m|^2 (ns = 3: the band sums; 1: plain)
__global__ void k_mlwf_finish(const double2* __restrict__ Z, int M, const double* __restrict__ norms, int ns,
                              double2* __restrict__ a) {
  const size_t MM = (size_t)M * M;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < 3 * (long)MM; e += (long)gridDim.x * blockDim.x) {
    const int d = (int)(e / MM);
    const int m = (int)((e % MM) / M), n = (int)(e % M);
    const double2 x = Z[(size_t)d * MM + (size_t)m * M + n];
    const double2 y = Z[(size_t)d * MM + (size_t)n * M + m];
    const double zx = x.x, zy = x.y, tx = y.x, ty = y.y;
    const double sc = 1.0 / sqrt(norms[ns * m + ns - 1] * norms[ns * n + ns - 1]);
    // conj(Z[n][m]) = (tx, -ty)
    a[(2 * d) * MM + (size_t)m * M + n] = make_double2(0.5 * sc * (zx + tx), 0.5 * sc * (zy - ty));
    // (Z - conj(Z[n][m])) / (2i) = (v - i u) / 2 with u + i v = Z - conj(Z[n][m])
    const double ur = zx - tx, vi = zy + ty;
    a[(2 * d + 1) * MM + (size_t)m * M + n] = make_double2(0.5 * sc * vi, -0.5 * sc * ur);
  }
}

// ------------------------------------------------------------------ jade
// Symmetric 3x3 eigenproblem by cyclic Jacobi rotations (the method of
// wannier/jacobi_eigenvalue.hpp; the oracle restates the same steps); returns the
// eigenvector of the largest eigenvalue with the sign the iteration leaves.
__device__ void jacobi3_top(double S[3][3], double out[3]) {
  double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  double d[3] = {S[0][0], S[1][1], S[2][2]};
  double base[3] = {d[0], d[1], d[2]};
  double inc[3] = {0, 0, 0};
  for (int pass = 1; pass <= 10000; pass++) {
    double off = 0.0;
#pragma unroll
    for (int q = 0; q < 3; q++)
#pragma unroll
      for (int p = 0; p < q; p++) off += S[p][q] * S[p][q];
    const double thresh = sqrt(off) / 12.0;
    if (!(thresh > 0.0)) break;  // converged, or a non-finite matrix (reported by the sweep's change)
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int q = p + 1; q < 3; q++) {
        const double big = 10.0 * fabs(S[p][q]);
        if (pass > 4 && big + fabs(d[p]) == fabs(d[p]) && big + fabs(d[q]) == fabs(d[q])) {
          S[p][q] = 0.0;
          continue;
        }
        if (fabs(S[p][q]) < thresh) continue;
        double h = d[q] - d[p];
        double t;
        if (fabs(h) + big == fabs(h)) {
          t = S[p][q] / h;
        } else {
          const double theta = 0.5 * h / S[p][q];
          t = 1.0 / (fabs(theta) + sqrt(1.0 + theta * theta));
          if (theta < 0.0) t = -t;
        }
        const double c = 1.0 / sqrt(1.0 + t * t), s = t * c, tau = s / (1.0 + c);
        h = t * S[p][q];
        inc[p] -= h;
        inc[q] += h;
        d[p] -= h;
        d[q] += h;
        S[p][q] = 0.0;
#define INQB_JROT(x, y)                   \
  {                                       \
    const double g_ = (x), h_ = (y);      \
    (x) = g_ - s * (h_ + g_ * tau);       \
    (y) = h_ + s * (g_ - h_ * tau);       \
  }
#pragma unroll
        for (int j = 0; j < p; j++) INQB_JROT(S[j][p], S[j][q])
#pragma unroll
        for (int j = p + 1; j < q; j++) INQB_JROT(S[p][j], S[j][q])
#pragma unroll
        for (int j = q + 1; j < 3; j++) INQB_JROT(S[p][j], S[q][j])
#pragma unroll
        for (int j = 0; j < 3; j++) INQB_JROT(V[j][p], V[j][q])
#undef INQB_JROT
      }
    for (int i = 0; i < 3; i++) {
      base[i] += inc[i];
      d[i] = base[i];
      inc[i] = 0.0;
    }
  }
  for (int k = 0; k < 2; k++) {
    int m = k;
    for (int l = k + 1; l < 3; l++)
      if (d[l] < d[m]) m = l;
    if (m != k) {
      const double t = d[m];
      d[m] = d[k];
      d[k] = t;
      for (int i = 0; i < 3; i++) {
        const double v = V[i][m];
        V[i][m] = V[i][k];
        V[i][k] = v;
      }
    }
  }
  for (int i = 0; i < 3; i++) out[i] = V[i][2];
}

constexpr int kJT = 128;  // threads of a pair's CTA

// one CTA per pair of this rotation step; a [6][M][M], u [M][M]
__global__ void __launch_bounds__(kJT)
    k_jade_step(double2* __restrict__ a, double2* __restrict__ u, int M, const int2* __restrict__ pairs,
                double* __restrict__ delta) {
  __shared__ double red[kJT / 32][36];
  __shared__ double rot[3];  // c, Re s, Im s
  __shared__ double old_diag;
  const int2 pq = pairs[blockIdx.x];
  const int p = pq.x, q = pq.y;
  if (p >= M || q >= M) {
    if (threadIdx.x == 0) delta[blockIdx.x] = 0.0;
    return;
  }
  const size_t MM = (size_t)M * M;
  // the 18 pair elements: (sum conj(a_k[p][i]) u[q][i], sum conj(a_k[p][i]) u[p][i],
  // sum conj(a_k[q][i]) u[q][i]) for k < 6
  double s[36];
#pragma unroll
  for (int i = 0; i < 36; ++i) s[i] = 0.0;
  for (int i = threadIdx.x; i < M; i += blockDim.x) {
    const double2 up = u[(size_t)p * M + i], uq = u[(size_t)q * M + i];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double2 ap = cconj(a[k * MM + (size_t)p * M + i]), aq = cconj(a[k * MM + (size_t)q * M + i]);
      const double2 x0 = cmul(ap, uq), x1 = cmul(ap, up), x2 = cmul(aq, uq);
      s[6 * k + 0] += x0.x;
      s[6 * k + 1] += x0.y;
      s[6 * k + 2] += x1.x;
      s[6 * k + 3] += x1.y;
      s[6 * k + 4] += x2.x;
      s[6 * k + 5] += x2.y;
    }
  }
#pragma unroll
  for (int i = 0; i < 36; ++i)
    for (int o = 16; o > 0; o >>= 1) s[i] += __shfl_down_sync(0xffffffffu, s[i], o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < 36; ++i) red[w][i] = s[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double od = 0.0;
    for (int k = 0; k < 6; ++k) {
      double e[6];
      for (int i = 0; i < 6; ++i) {
        double v = 0.0;
        for (int ww = 0; ww < kJT / 32; ++ww) v += red[ww][6 * k + i];
        e[i] = v;
      }
      const double2 aij = make_double2(e[0], e[1]), aii = make_double2(e[2], e[3]), ajj = make_double2(e[4], e[5]);
      // h = (aii - ajj, aij + conj(aij), i (aij - conj(aij))) = (.., (2 Re aij, 0), (-2 Im aij, 0))
      const double2 h[3] = {make_double2(aii.x - ajj.x, aii.y - ajj.y), make_double2(2.0 * aij.x, 0.0),
                            make_double2(-2.0 * aij.y, 0.0)};
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) G[r][c] += h[r].x * h[c].x + h[r].y * h[c].y;
      od += a[k * MM + (size_t)p * M + p].x + a[k * MM + (size_t)q * M + q].x;
    }
    double v[3];
    jacobi3_top(G, v);
    double x = v[0], y = v[1], z = v[2];
    if (v[0] < 0.0) {
      x = -x;
      y = -y;
    }
    const double r = sqrt((x + 1.0) / 2.0);
    rot[0] = r;
    rot[1] = y / (2.0 * r);
    rot[2] = -z / (2.0 * r);
    old_diag = od;
  }
  __syncthreads();
  const double c = rot[0];
  const double2 sv = make_double2(rot[1], rot[2]), sc = cconj(sv);
  // rows p, q of a_k and u: row_p <- c row_p + conj(s) row_q, row_q <- -s row_p + c row_q
  for (int e = threadIdx.x; e < 7 * M; e += blockDim.x) {
    const int k = e / M, i = e % M;
    double2* base = (k < 6) ? a + k * MM : u;
    double2& rp = base[(size_t)p * M + i];
    double2& rq = base[(size_t)q * M + i];
    const double2 xv = rp, yv = rq;
    const double2 t1 = cmul(sc, yv), t2 = cmul(sv, xv);
    rp = make_double2(c * xv.x + t1.x, c * xv.y + t1.y);
    rq = make_double2(c * yv.x - t2.x, c * yv.y - t2.y);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double nd = 0.0;
    for (int k = 0; k < 6; ++k) nd += a[k * MM + (size_t)p * M + p].x + a[k * MM + (size_t)q * M + q].x;
    delta[blockIdx.x] = nd - old_diag;
  }
}

// out = sum_steps 2 |sum_pairs delta[step][pair]| (one block, fixed order)
__global__ void k_jade_change(const double* __restrict__ delta, int nsteps, int np, double* __restrict__ out) {
  __shared__ double part[256];
  double acc = 0.0;
  for (int s = threadIdx.x; s < nsteps; s += blockDim.x) {
    double t = 0.0;
    for (int i = 0; i < np; ++i) t += delta[(size_t)s * np + i];
    acc += 2.0 * fabs(t);
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)blockDim.x; ++i) t += part[i];
    out[0] = t;
  }
}

__global__ void k_identity(double2* __restrict__ u, int M) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < (long)M * M; e += (long)gridDim.x * blockDim.x)
    u[e] = make_double2((e / M == e % M) ? 1.0 : 0.0, 0.0);
}

// adiag[k][i] = sum_j conj(a_k[i][j]) u[i][j]; grid (M, 6)
__global__ void __launch_bounds__(128)
    k_jade_adiag(const double2* __restrict__ a, const double2* __restrict__ u, int M, double2* __restrict__ adiag) {
  __shared__ double red[4][2];
  const int i = blockIdx.x, k = blockIdx.y;
  const size_t MM = (size_t)M * M;
  double sr = 0.0, si = 0.0;
  for (int j = threadIdx.x; j < M; j += blockDim.x) {
    const double2 x = cmul(cconj(a[k * MM + (size_t)i * M + j]), u[(size_t)i * M + j]);
    sr += x.x;
    si += x.y;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sr += __shfl_down_sync(0xffffffffu, sr, o);
    si += __shfl_down_sync(0xffffffffu, si, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5][0] = sr;
    red[threadIdx.x >> 5][1] = si;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0, im = 0.0;
    for (int w = 0; w < 4; ++w) {
      r += red[w][0];
      im += red[w][1];
    }
    adiag[(size_t)k * M + i] = make_double2(r, im);
  }
}

// ------------------------------------------------------------------ rotate
// out[p][i] = sum_j psi[p][j] conj(u[i][j]); 64 x 64 output tiles, 256 threads with
// 4 x 4 outputs each, j in chunks of 8 through shared memory.
constexpr int kRT = 64, kRK = 8;

// FP64: 128 registers for two CTAs per SM (136 unbounded, one CTA: 2.98 -> 2.09 ms at
// 64^3 x 128 states); FP32 runs best unbounded
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 2 : 1)
    k_mlwf_rotate(const cplx<T>* __restrict__ psi, long ld, int M, long N, const double2* __restrict__ u,
                  cplx<T>* __restrict__ out, long ldo) {
  using R = T;
  __shared__ cplx<R> sP[kRK][kRT + 1];  // [j][point]
  __shared__ cplx<R> sU[kRK][kRT];      // [j][i] = conj(u[i][j])
  const long p0 = (long)blockIdx.x * kRT;
  const int i0 = blockIdx.y * kRT;
  const int tp = threadIdx.x % 16, ti = threadIdx.x / 16;
  cplx<R> acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = mk<R>(0, 0);
  for (int j0 = 0; j0 < M; j0 += kRK) {
    for (int e = threadIdx.x; e < kRK * kRT; e += blockDim.x) {
      const int jj = e % kRK, pp = e / kRK;
      const long p = p0 + pp;
      const int j = j0 + jj;
      sP[jj][pp] = (p < N && j < M) ? psi[p * ld + j] : mk<R>(0, 0);
      const int ii = e / kRK;  // same decomposition for u: [i][j] rows
      const int i = i0 + ii;
      if (i < M && j < M) {
        const double2 x = u[(size_t)i * M + j];
        sU[jj][ii] = mk<R>((R)x.x, (R)(-x.y));
      } else {
        sU[jj][ii] = mk<R>(0, 0);
      }
    }
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < kRK; ++jj) {
      cplx<R> pv[4], uv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) pv[a] = sP[jj][tp + 16 * a];
#pragma unroll
      for (int b = 0; b < 4; ++b) uv[b] = sU[jj][ti + 16 * b];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          acc[a][b].x = fma(pv[a].x, uv[b].x, fma(-pv[a].y, uv[b].y, acc[a][b].x));
          acc[a][b].y = fma(pv[a].x, uv[b].y, fma(pv[a].y, uv[b].x, acc[a][b].y));
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const long p = p0 + tp + 16 * a;
      const int i = i0 + ti + 16 * b;
      if (p < N && i < M) out[p * ldo + i] = acc[a][b];
    }
}

}  // namespace

namespace {
template <typename T>
long gram_slabs(long N, int Ma, int Mb) {
  constexpr int TM = 16 * GramCfg<T>::TMX, TN = 16 * GramCfg<T>::TNX, kGP = GramCfg<T>::GP;
  const long tiles = (long)((Ma + TM - 1) / TM) * ((Mb + TN - 1) / TN);
  const long chunks = (N + kGP - 1) / kGP;
  if (sizeof(T) == 4) return std::max<long>(1, (N + kSlabF32 - 1) / kSlabF32);
  return std::max<long>(1, std::min<long>(chunks, (148L * 4 + tiles - 1) / tiles));
}
size_t slab_bytes(long N, int Ma, int Mb) {
  const size_t MM = (size_t)Ma * Mb;
  return std::max((size_t)gram_slabs<double>(N, Ma, Mb) * 3 * MM * sizeof(double2),
                  (size_t)gram_slabs<float>(N, Ma, Mb) * 3 * MM * sizeof(float2));
}
}  // namespace

// the slabs of the larger layout, then Z [3][Ma][Mb] (FP64) at a 256-byte boundary
size_t mlwf_partial_bytes(long N, int Ma, int Mb) {
  return (slab_bytes(N, Ma, Mb) + 255) / 256 * 256 + 3 * (size_t)Ma * Mb * sizeof(double2);
}
size_t mlwf_partial_bytes(long N, int M) { return mlwf_partial_bytes(N, M, M); }

// Z [3][Ma][Mb] = sum_p conj(a_m) e^{i theta_d} b_n (FP64 sums of the slabs), in the
// partial buffer after the slabs; returns Z
template <typename T>
static int gram_impl(const void* pa, long lda, int Ma, const void* pb, long ldb, int Mb, long N, const GramGeom& g,
                     void* partial, double2** Zout, cudaStream_t st) {
  using P = typename GramCfg<T>::P;
  constexpr int TM = 16 * GramCfg<T>::TMX, TN = 16 * GramCfg<T>::TNX, kGP = GramCfg<T>::GP;
  const long slabs = gram_slabs<T>(N, Ma, Mb);
  const long per = ((N + slabs - 1) / slabs + kGP - 1) / kGP * kGP;
  const long nslab = (N + per - 1) / per;
  const dim3 grid((unsigned)(((Ma + TM - 1) / TM) * ((Mb + TN - 1) / TN)), (unsigned)nslab);
  k_mlwf_gram<T><<<grid, 256, 0, st>>>((const cplx<T>*)pa, lda, Ma, (const cplx<T>*)pb, ldb, Mb, N, g, per,
                                       (P*)partial);
  INQB_CUDA_TRY(cudaGetLastError());
  const long work = 3L * Ma * Mb;
  double2* Z = reinterpret_cast<double2*>(static_cast<char*>(partial) + (slab_bytes(N, Ma, Mb) + 255) / 256 * 256);
  k_mlwf_slab_sum<P><<<(unsigned)std::min<long>((work + 255) / 256, 148L * 32), 256, 0, st>>>((const P*)partial,
                                                                                             (int)nslab, work, Z);
  INQB_CUDA_TRY(cudaGetLastError());
  *Zout = Z;
  return INQB_OK;
}

static GramGeom gram_geom(const int nr[3], const double lat[3][3]) {
  GramGeom g;
  double len[3];
  for (int d = 0; d < 3; ++d) {
    g.nr[d] = nr[d];
    len[d] = sqrt(lat[d][0] * lat[d][0] + lat[d][1] * lat[d][1] + lat[d][2] * lat[d][2]);
  }
  // theta_d / pi = 2 r_d / |a_d|, r = sum_j f_j a_j
  for (int d = 0; d < 3; ++d)
    for (int j = 0; j < 3; ++j) g.frac_to_theta[d][j] = 2.0 * lat[j][d] / len[d];
  return g;
}

int launch_mlwf_gram(int precision, const void* psi, long ld, int M, long N, const int nr[3], const double lat[3][3],
                     const double* sums, void* partial, double2* a, void* stream) {
  const GramGeom g = gram_geom(nr, lat);
  cudaStream_t st = (cudaStream_t)stream;
  double2* Z = nullptr;
  INQB_TRY(precision == INQB_FP64 ? gram_impl<double>(psi, ld, M, psi, ld, M, N, g, partial, &Z, st)
                                  : gram_impl<float>(psi, ld, M, psi, ld, M, N, g, partial, &Z, st));
  return launch_mlwf_finish(Z, M, sums, 3, a, stream);
}

int launch_mlwf_gram_block(int precision, const void* pa, long lda, int Ma, const void* pb, long ldb, int Mb, long N,
                           const int nr[3], const double lat[3][3], void* partial, double2* Z, void* stream) {
  const GramGeom g = gram_geom(nr, lat);
  cudaStream_t st = (cudaStream_t)stream;
  double2* Zw = nullptr;
  INQB_TRY(precision == INQB_FP64 ? gram_impl<double>(pa, lda, Ma, pb, ldb, Mb, N, g, partial, &Zw, st)
                                  : gram_impl<float>(pa, lda, Ma, pb, ldb, Mb, N, g, partial, &Zw, st));
  INQB_CUDA_TRY(cudaMemcpyAsync(Z, Zw, sizeof(double2) * 3 * (size_t)Ma * Mb, cudaMemcpyDeviceToDevice, st));
  return INQB_OK;
}

int launch_mlwf_finish(const double2* Z, int M, const double* norms, int norm_stride, double2* a, void* stream) {
  const long work = 3L * M * M;
  k_mlwf_finish<<<(unsigned)std::min<long>((work + 255) / 256, 148L * 8), 256, 0, (cudaStream_t)stream>>>(
      Z, M, norms, norm_stride, a);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_identity(double2* u, int M, void* stream) {
  k_identity<<<(unsigned)std::min<long>(((long)M * M + 255) / 256, 1024), 256, 0, (cudaStream_t)stream>>>(u, M);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_jade_step(double2* a, double2* u, int M, const int2* pairs, int np, double* delta, void* stream) {
  k_jade_step<<<np, kJT, 0, (cudaStream_t)stream>>>(a, u, M, pairs, delta);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_jade_change(const double* delta, int nsteps, int np, double* out, void* stream) {
  k_jade_change<<<1, 256, 0, (cudaStream_t)stream>>>(delta, nsteps, np, out);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_jade_adiag(const double2* a, const double2* u, int M, double2* adiag, void* stream) {
  k_jade_adiag<<<dim3(M, 6), 128, 0, (cudaStream_t)stream>>>(a, u, M, adiag);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_mlwf_rotate(int precision, const void* psi, long ld, int M, long N, const double2* u, void* out, long ldo,
                       void* stream) {
  const dim3 grid((unsigned)((N + kRT - 1) / kRT), (unsigned)((M + kRT - 1) / kRT));
  if (precision == INQB_FP64)
    k_mlwf_rotate<double><<<grid, 256, 0, (cudaStream_t)stream>>>((const cplx<double>*)psi, ld, M, N, u,
                                                                   (cplx<double>*)out, ldo);
  else
    k_mlwf_rotate<float><<<grid, 256, 0, (cudaStream_t)stream>>>((const cplx<float>*)psi, ld, M, N, u,
                                                                  (cplx<float>*)out, ldo);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

}  // namespace inqb
