// Building blocks of the discrete adjoint of the ETRS propagator.
//
//   axpby        y <- a x + b y on orbital blocks
//   position     lambda <- s occ[m] r_d(p) psi      (d dipole / d psi*, dipole.hpp:23-40)
//   V gradient   gV[p] += Re(c sum_m conj(u) w)      (<u| dH/dV(p) |w>, H's local term)
//   A gradient   gA[d] += Re(c <u| dH/dA_d |w>)      kinetic (G + k + A)_d in Fourier space
//                plus the nonlocal position commutator i S [conj(p_u) r_w - conj(r_u) p_w]
//                from per-chunk moments (deterministic: no atomics on the moments)
//                (the structure of projector_all::position_commutator,
//                src/hamiltonian/projector_all.hpp:319-403).
// All sums are FP64 whatever the orbital precision.
#include <cuda_runtime.h>

#include "adjoint.h"
#include "dft.cuh"
#include "inqb_internal.h"
#include "plan.h"

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

// y = sum_{k < K} a_k x_k over orbital blocks (K <= kMaxTerms); y may be one of the x_k.
constexpr int kMaxTerms = 5;
template <typename T>
struct LinTerms {
  const cplx<T>* x[kMaxTerms];
  long ld[kMaxTerms];
  cplx<T> a[kMaxTerms];
  int K;
};

template <typename T>
__global__ void k_lincomb(long N, int M, LinTerms<T> t, cplx<T>* __restrict__ y, long ldy) {
  const long total = N * M;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long p = i / M;
    const int m = (int)(i - p * M);
    cplx<T> acc = mk<T>(0, 0);
#pragma unroll
    for (int k = 0; k < kMaxTerms; ++k)
      if (k < t.K) fma_acc(acc, t.a[k], t.x[k][p * t.ld[k] + m]);
    y[p * ldy + m] = acc;
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

// perturbations::kick::zero_step in the length gauge (src/perturbations/kick.hpp:20-61):
// psi *= exp(i E . r) with E = -kick field, r the cartesian point (symmetric range).
template <typename T>
__global__ void k_phase_kick(long N, int M, cplx<T>* __restrict__ psi, long ld, Lat g, double e0, double e1,
                             double e2) {
  const long total = N * M;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long p = i / M;
    const int m = (int)(i - p * M);
    const double ph = e0 * rcomp(g, p, 0) + e1 * rcomp(g, p, 1) + e2 * rcomp(g, p, 2);
    double sn, cs;
    sincos(ph, &sn, &cs);
    cplx<T>& v = psi[p * ld + m];
    const double x = v.x, y = v.y;
    v = mk<T>((T)(cs * x - sn * y), (T)(cs * y + sn * x));
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

// The same reduction on coefficients in the tile layout [g][ka][kz][kx][kb][G] that
// the H passes emit (ky = ka + Y2 kb); padded orbitals (m >= M) are skipped.
struct TileFourier {
  int G, Y1, Y2;
};

// Eight orbital blocks of a backward half step, Lambda_0..3 and Phi_0..3 (or their
// forward coefficients), and the weights of Xi_i = sum_j w[i][j] Lambda_j.
template <typename T>
struct EightBlocks {
  const cplx<T>* L[4];
  const cplx<T>* P[4];
  long ldL[4];
  long ldP;
};
struct PairWeights {
  double w[4][4][2];  // w[i][j] = conj(c_{i+j+1}) for i + j <= 3
};

template <typename T>
__global__ void k_velocity_dot_tiles(long nelem, int M, const cplx<T>* __restrict__ U, const cplx<T>* __restrict__ W,
                                     TileFourier tf, Recip r, double* __restrict__ acc) {
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += (long)gridDim.x * blockDim.x) {
    long t = e / tf.G;
    const int j = (int)(e - t * tf.G);
    const int kb = (int)(t % tf.Y1);
    t /= tf.Y1;
    const int kx = (int)(t % r.nr[0]);
    t /= r.nr[0];
    const int kz = (int)(t % r.nr[2]);
    t /= r.nr[2];
    const int ka = (int)(t % tf.Y2);
    const long g = t / tf.Y2;
    if (g * tf.G + j >= M) continue;
    const int k[3] = {kx, ka + tf.Y2 * kb, kz};
    double n[3];
    for (int c = 0; c < 3; c++) n[c] = (k[c] >= (r.nr[c] + 1) / 2) ? k[c] - r.nr[c] : k[c];
    double gf = 1.0;
    if (r.mask) {
      const long long a0 = (long long)r.nr[1] * r.nr[2], a1 = (long long)r.nr[0] * r.nr[2],
                      a2 = (long long)r.nr[0] * r.nr[1];
      const long long tot = (long long)r.nr[0] * r.nr[1] * r.nr[2];
      const long long i0 = (long long)n[0], i1 = (long long)n[1], i2 = (long long)n[2];
      if (4 * (i0 * i0 * a0 * a0 + i1 * i1 * a1 * a1 + i2 * i2 * a2 * a2) > tot * tot) gf = 0.0;
    }
    const cplx<T> a = U[e], b = W[e];
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

// Nonlocal part of <u| dH/dA_d |w>, step 1: moments of one chunk of an atom's
// sphere entries,
//   p_u[l] = sum_e beta_e[l] exp(i(k+A).r_e) u(r_e),  r_u[l][d] = the same with x_e[d],
// and likewise for w; 16 FP64 values (4 complex for u, 4 for w) per (l, orbital).
// Each entry is one atom-major record (phase, beta, position, grid point), so the
// only dependent load is the orbital gather.  Block: 32 orbitals x LMAX projectors
// x 2 entry lanes.  part[chunk][l][q][M].
template <typename T>
__global__ void __launch_bounds__(256)
    k_nl_moments(int L, int M, const cplx<T>* __restrict__ u, const cplx<T>* __restrict__ w, long ld,
                 const int* __restrict__ chunk_atom, const int* __restrict__ chunk_beg,
                 const int* __restrict__ atom_ptr, const AdjRec<T>* __restrict__ adj, double* __restrict__ part) {
  constexpr int LM = 4, Q = 16;
  __shared__ double red[LM][32][Q + 1];
  const int c = blockIdx.x;
  const int m = blockIdx.y * 32 + (threadIdx.x & 31);
  const int l = (threadIdx.x >> 5) & (LM - 1), es = threadIdx.x >> 7;
  const int a = chunk_atom[c];
  const int i0 = chunk_beg[c], i1 = min(i0 + kNlChunk, atom_ptr[a + 1]);
  double s[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) s[q] = 0.0;
  if (m < M && l < L) {
#pragma unroll 2
    for (int i = i0 + es; i < i1; i += 2) {
      const AdjRec<T> r = adj[i];
      const cplx<T> uu = u[(long)r.pt * ld + m], ww = w[(long)r.pt * ld + m];
      const double b = (double)r.beta[l];
      const double pr = (double)r.ph[0], pi = (double)r.ph[1];
      // b exp(i (k+A).r) u and the same for w, in FP64
      const double ur = b * (pr * uu.x - pi * uu.y), ui = b * (pr * uu.y + pi * uu.x);
      const double wr = b * (pr * ww.x - pi * ww.y), wi = b * (pr * ww.y + pi * ww.x);
      const double x0 = r.xyz[0], x1 = r.xyz[1], x2 = r.xyz[2];
      s[0] += ur; s[1] += ui;
      s[2] += x0 * ur; s[3] += x0 * ui; s[4] += x1 * ur; s[5] += x1 * ui; s[6] += x2 * ur; s[7] += x2 * ui;
      s[8] += wr; s[9] += wi;
      s[10] += x0 * wr; s[11] += x0 * wi; s[12] += x1 * wr; s[13] += x1 * wi; s[14] += x2 * wr; s[15] += x2 * wi;
    }
  }
  if (es == 1) {
#pragma unroll
    for (int q = 0; q < Q; ++q) red[l][threadIdx.x & 31][q] = s[q];
  }
  __syncthreads();
  if (es == 0 && m < M && l < L) {
#pragma unroll
    for (int q = 0; q < Q; ++q) part[(((long)c * L + l) * Q + q) * M + m] = s[q] + red[l][threadIdx.x & 31][q];
  }
}

// The moments of the four pairs (Lambda_j, Phi_j), pair j = blockIdx.z, into
// part[chunk][pair][l][q][M] (the same sums as k_nl_moments).  Warps are (projector l,
// half h); a lane holds orbital m = blockIdx.y * MW + lane % MW and walks the entry
// stream (lane / MW) + (32 / MW) h, so that fewer than 32 orbitals still fill the warp
// (MW = 16 for M <= 16).  The chunk's records are staged in shared memory first, and
// a lane gathers the orbital values of B entries before it adds them up (in its entry
// order), so B gathers are in flight instead of one record-then-gather chain.
template <typename T, int MW>
__global__ void __launch_bounds__(256)
    k_nl_moments_pairs(int L, int M, const __grid_constant__ EightBlocks<T> b, const int* __restrict__ chunk_atom,
                       const int* __restrict__ chunk_beg, const int* __restrict__ atom_ptr,
                       const AdjRec<T>* __restrict__ adj, double* __restrict__ part) {
  constexpr int LM = 4, Q = 16, SUB = 32 / MW, STREAMS = 2 * SUB;
  constexpr int B = sizeof(T) == 4 ? 8 : 4;
  constexpr int RV = (int)(sizeof(AdjRec<T>) / 16);
  static_assert(sizeof(AdjRec<T>) % 16 == 0, "records are copied in 16-byte pieces");
  __shared__ double red[LM][32][Q + 1];
  __shared__ __align__(16) AdjRec<T> R[kNlChunk];
  const int c = blockIdx.x, pr = blockIdx.z;
  const int lane = threadIdx.x & 31;
  const int m = blockIdx.y * MW + (lane % MW);
  const int l = (threadIdx.x >> 5) & (LM - 1), h = threadIdx.x >> 7;
  const int stream = lane / MW + SUB * h;
  const int a = chunk_atom[c];
  const int i0 = chunk_beg[c], n = min(kNlChunk, atom_ptr[a + 1] - i0);
  {
    const char* src = reinterpret_cast<const char*>(adj + i0);
    for (int q = threadIdx.x; q < n * RV; q += blockDim.x) {
      const unsigned d = (unsigned)__cvta_generic_to_shared(reinterpret_cast<char*>(R) + 16 * q);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 16 * q) : "memory");
    }
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
  }
  __syncthreads();
  const cplx<T>* u = b.L[pr];
  const cplx<T>* w = b.P[pr];
  const long ldu = b.ldL[pr], ldw = b.ldP;
  double s[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) s[q] = 0.0;
  if (m < M && l < L) {
    for (int k0 = stream; k0 < n; k0 += B * STREAMS) {
      cplx<T> uu[B], ww[B];
#pragma unroll
      for (int j = 0; j < B; ++j) {
        const int k = k0 + j * STREAMS;
        const long pt = R[min(k, n - 1)].pt;
        uu[j] = u[pt * ldu + m];
        ww[j] = w[pt * ldw + m];
      }
#pragma unroll
      for (int j = 0; j < B; ++j) {
        const int k = k0 + j * STREAMS;
        if (k >= n) continue;
        const AdjRec<T>& r = R[k];
        const double bb = (double)r.beta[l];
        const double phr = (double)r.ph[0], phi = (double)r.ph[1];
        const double ur = bb * (phr * uu[j].x - phi * uu[j].y), ui = bb * (phr * uu[j].y + phi * uu[j].x);
        const double wr = bb * (phr * ww[j].x - phi * ww[j].y), wi = bb * (phr * ww[j].y + phi * ww[j].x);
        const double x0 = r.xyz[0], x1 = r.xyz[1], x2 = r.xyz[2];
        s[0] += ur; s[1] += ui;
        s[2] += x0 * ur; s[3] += x0 * ui; s[4] += x1 * ur; s[5] += x1 * ui; s[6] += x2 * ur; s[7] += x2 * ui;
        s[8] += wr; s[9] += wi;
        s[10] += x0 * wr; s[11] += x0 * wi; s[12] += x1 * wr; s[13] += x1 * wi; s[14] += x2 * wr; s[15] += x2 * wi;
      }
    }
  }
  // the SUB streams of a warp meet by shuffles (lane % MW keeps the orbital), then the
  // two halves in shared memory
#pragma unroll
  for (int o = 16; o >= MW; o >>= 1)
#pragma unroll
    for (int q = 0; q < Q; ++q) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
  if (h == 1 && lane < MW) {
#pragma unroll
    for (int q = 0; q < Q; ++q) red[l][lane][q] = s[q];
  }
  __syncthreads();
  if (h == 0 && lane < MW && m < M && l < L) {
#pragma unroll
    for (int q = 0; q < Q; ++q)
      part[((((long)c * 4 + pr) * L + l) * Q + q) * M + m] = s[q] + red[l][lane][q];
  }
}

// Step 2: block (atom a, projector l, 32 orbitals); thread (q, m) sums moment q of
// orbital m over the atom's chunks, then the orbital's threads add
// S_l i [conj(p_u) r_w,d - conj(r_u,d) p_w] into acc[6 + 2d .. 6 + 2d + 1].
__global__ void __launch_bounds__(512)
    k_nl_combine(int L, int M, const int* __restrict__ atom_chunk_ptr, const double* __restrict__ part,
                 const double* __restrict__ scale, double* __restrict__ acc) {
  constexpr int Q = 16;
  __shared__ double mom[Q][33];
  const int a = blockIdx.x, l = blockIdx.y;
  const int mi = threadIdx.x & 31, q = threadIdx.x >> 5;
  const int m = blockIdx.z * 32 + mi;
  const int c0 = atom_chunk_ptr[a], c1 = atom_chunk_ptr[a + 1];
  // four independent partial sums keep four loads in flight (fixed order: deterministic)
  double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
  if (m < M) {
    const long stride = (long)L * Q * M;
    const double* pp = part + (((long)c0 * L + l) * Q + q) * M + m;
    int c = c0;
    for (; c + 3 < c1; c += 4, pp += 4 * stride) {
      v0 += pp[0];
      v1 += pp[stride];
      v2 += pp[2 * stride];
      v3 += pp[3 * stride];
    }
    for (; c < c1; ++c, pp += stride) v0 += pp[0];
  }
  mom[q][mi] = (v0 + v1) + (v2 + v3);
  __syncthreads();
  double out[6] = {0, 0, 0, 0, 0, 0};
  if (q == 0 && m < M) {
    const double S = scale[a * L + l];
    const double pur = mom[0][mi], pui = mom[1][mi], pwr = mom[8][mi], pwi = mom[9][mi];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double rur = mom[2 + 2 * d][mi], rui = mom[3 + 2 * d][mi];
      const double rwr = mom[10 + 2 * d][mi], rwi = mom[11 + 2 * d][mi];
      // z1 = conj(p_u) r_w, z2 = conj(r_u) p_w, result += S i (z1 - z2)
      const double z1r = pur * rwr + pui * rwi, z1i = pur * rwi - pui * rwr;
      const double z2r = rur * pwr + rui * pwi, z2i = rur * pwi - rui * pwr;
      out[2 * d] = -S * (z1i - z2i);
      out[2 * d + 1] = S * (z1r - z2r);
    }
  }
  if (q == 0) {
#pragma unroll
    for (int k = 0; k < 6; k++) {
      double x = out[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (mi == 0) atomicAdd(&acc[6 + k], x);
    }
  }
}

// ---------------------------------------------------------------- the gradient of one half step
// With Xi_i = sum_j w[i][j] Lambda_j (w[i][j] = conj(c_{i+j+1}), zero for i + j > 3),
// the half step's gradient terms are sums over i of bilinear forms in (Xi_i, Phi_i);
// these kernels read the eight blocks Lambda_0..3, Phi_0..3 once and weight them.


// gV[p] += 2 Re sum_m sum_i conj(Xi_i) Phi_i, one group of LPP lanes per grid point
// (LPP = 16 where M <= 16, so no lane idles).
template <typename T, int LPP>
__global__ void k_vgrad8(long N, int M, EightBlocks<T> b, PairWeights pw, double* __restrict__ gV) {
  const int lane = threadIdx.x & (LPP - 1);
  const long grp = ((long)blockIdx.x * blockDim.x + threadIdx.x) / LPP;
  const long ngrp = ((long)gridDim.x * blockDim.x) / LPP;
  // every lane of the warp runs the same number of iterations (the shuffles below)
  const long pend = (N + ngrp - 1) / ngrp * ngrp;
  for (long p = grp; p < pend; p += ngrp) {
    double re = 0.0;
    for (int m = lane; m < M && p < N; m += LPP) {
      double lr[4], li[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const cplx<T> v = b.L[j][p * b.ldL[j] + m];
        lr[j] = v.x;
        li[j] = v.y;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        double xr = 0.0, xi = 0.0;
#pragma unroll
        for (int j = 0; j < 4 - i; ++j) {
          xr += pw.w[i][j][0] * lr[j] - pw.w[i][j][1] * li[j];
          xi += pw.w[i][j][0] * li[j] + pw.w[i][j][1] * lr[j];
        }
        const cplx<T> f = b.P[i][p * b.ldP + m];
        re += xr * (double)f.x + xi * (double)f.y;  // Re conj(Xi) Phi
      }
    }
#pragma unroll
    for (int o = LPP / 2; o > 0; o >>= 1) re += __shfl_xor_sync(0xffffffffu, re, o);
    if (lane == 0 && p < N) gV[p] += 2.0 * re;
  }
}

// acc[2d..2d+1] += sum_{G,m} sum_i conj(Xi_i(G)) (G + kA)_d Phi_i(G) on the tile-layout
// coefficients (b.L / b.P point at coefficient blocks, ld unused).
// IDX: the index type of the element arithmetic (32-bit where nelem fits: the
// divisions below are much cheaper than in 64 bits).
template <typename T, typename IDX>
__global__ void k_velocity_dot8(IDX nelem, int M, EightBlocks<T> b, PairWeights pw, TileFourier tf, Recip r,
                                double* __restrict__ acc) {
  double s[6] = {0, 0, 0, 0, 0, 0};
  const IDX uG = (IDX)tf.G, uY1 = (IDX)tf.Y1, uY2 = (IDX)tf.Y2, unx = (IDX)r.nr[0], unz = (IDX)r.nr[2];
  for (IDX e = (IDX)blockIdx.x * blockDim.x + threadIdx.x; e < nelem; e += (IDX)gridDim.x * blockDim.x) {
    IDX t = e / uG;
    const int j0 = (int)(e - t * uG);
    IDX t2 = t / uY1;
    const int kb = (int)(t - t2 * uY1);
    t = t2 / unx;
    const int kx = (int)(t2 - t * unx);
    t2 = t / unz;
    const int kz = (int)(t - t2 * unz);
    const IDX g = t2 / uY2;
    const int ka = (int)(t2 - g * uY2);
    if ((long)g * tf.G + j0 >= M) continue;
    const int k[3] = {kx, ka + tf.Y2 * kb, kz};
    double n[3];
    for (int c = 0; c < 3; c++) n[c] = (k[c] >= (r.nr[c] + 1) / 2) ? k[c] - r.nr[c] : k[c];
    double gf = 1.0;
    if (r.mask) {
      const long long a0 = (long long)r.nr[1] * r.nr[2], a1 = (long long)r.nr[0] * r.nr[2],
                      a2 = (long long)r.nr[0] * r.nr[1];
      const long long tot = (long long)r.nr[0] * r.nr[1] * r.nr[2];
      const long long i0 = (long long)n[0], i1 = (long long)n[1], i2 = (long long)n[2];
      if (4 * (i0 * i0 * a0 * a0 + i1 * i1 * a1 * a1 + i2 * i2 * a2 * a2) > tot * tot) gf = 0.0;
    }
    double lr[4], li[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const cplx<T> v = b.L[j][e];
      lr[j] = v.x;
      li[j] = v.y;
    }
    double re = 0.0, im = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      double xr = 0.0, xi = 0.0;
#pragma unroll
      for (int j = 0; j < 4 - i; ++j) {
        xr += pw.w[i][j][0] * lr[j] - pw.w[i][j][1] * li[j];
        xi += pw.w[i][j][0] * li[j] + pw.w[i][j][1] * lr[j];
      }
      const cplx<T> f = b.P[i][e];
      re += xr * (double)f.x + xi * (double)f.y;
      im += xr * (double)f.y - xi * (double)f.x;
    }
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

// Nonlocal term over the pairs: block (atom, l, 32 orbitals), thread (q, m) sums
// moment q of each pair (Lambda_j, Phi_j) over the atom's chunks
// (part[chunk][pair][l][q][M], q < 8 of Lambda_j, q >= 8 of Phi_j); then per orbital
// sum_i S_l i [conj(p_Xi_i) r_Phi_i - conj(r_Xi_i) p_Phi_i] with p_Xi_i = sum_j w p_Lambda_j.
__global__ void __launch_bounds__(512)
    k_nl_combine8(int L, int M, const int* __restrict__ atom_chunk_ptr, const double* __restrict__ part,
                  const double* __restrict__ scale, PairWeights wb, double* __restrict__ acc) {
  constexpr int Q = 16;
  __shared__ double mom[4][Q][33];
  const int a = blockIdx.x, l = blockIdx.y;
  const int mi = threadIdx.x & 31, q = threadIdx.x >> 5;
  const int m = blockIdx.z * 32 + mi;
  const int c0 = atom_chunk_ptr[a], c1 = atom_chunk_ptr[a + 1];
  // the four pairs' chunk sums, chunk c into accumulator (c - c0) % 4: sixteen loads in
  // flight per thread, a fixed order (deterministic)
  double v[4][4];
#pragma unroll
  for (int pr = 0; pr < 4; ++pr) v[pr][0] = v[pr][1] = v[pr][2] = v[pr][3] = 0.0;
  if (m < M) {
    const long stride = 4L * L * Q * M;
    const double* pp = part + ((long)c0 * 4 * L + l) * Q * M + (long)q * M + m;
    const long pstride = (long)L * Q * M;  // next pair of the same chunk
    int c = c0;
    for (; c + 3 < c1; c += 4, pp += 4 * stride) {
#pragma unroll
      for (int pr = 0; pr < 4; ++pr)
#pragma unroll
        for (int k = 0; k < 4; ++k) v[pr][k] += pp[pr * pstride + k * stride];
    }
    for (int k = 0; c < c1; ++c, ++k, pp += stride)
#pragma unroll
      for (int pr = 0; pr < 4; ++pr) v[pr][k] += pp[pr * pstride];
  }
#pragma unroll
  for (int pr = 0; pr < 4; ++pr) mom[pr][q][mi] = (v[pr][0] + v[pr][1]) + (v[pr][2] + v[pr][3]);
  __syncthreads();
  if (q != 0) return;  // warp 0 goes on whole (lanes past M add zeros)
  const double S = scale[a * L + l];
  double out[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (m >= M) break;
    // moments of Xi_i (u side, q 0..7) from those of the Lambda_j
    double xu[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 4 - i; ++j) {
      const double wr = wb.w[i][j][0], wi = wb.w[i][j][1];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double vr = mom[j][2 * k][mi], vi = mom[j][2 * k + 1][mi];
        xu[2 * k] += wr * vr - wi * vi;
        xu[2 * k + 1] += wr * vi + wi * vr;
      }
    }
    const double pur = xu[0], pui = xu[1], pwr = mom[i][8][mi], pwi = mom[i][9][mi];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double rur = xu[2 + 2 * d], rui = xu[3 + 2 * d];
      const double rwr = mom[i][10 + 2 * d][mi], rwi = mom[i][11 + 2 * d][mi];
      const double z1r = pur * rwr + pui * rwi, z1i = pur * rwi - pui * rwr;
      const double z2r = rur * pwr + rui * pwi, z2i = rur * pwi - rui * pwr;
      out[2 * d] += -S * (z1i - z2i);
      out[2 * d + 1] += S * (z1r - z2r);
    }
  }
  // the q == 0 threads of this block are one full warp (threads 0..31)
#pragma unroll
  for (int k = 0; k < 6; k++) {
    double x = out[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (mi == 0) atomicAdd(&acc[6 + k], x);
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
template <typename T>
static int half_grad_impl(const inqb_ctx& ctx, const void* const Lam[4], const long ldL[4], const void* const Phi[4],
                          long ldP, const void* const FL[4], const void* const FP[4], const double w[4][4][2], int M,
                          double* gV, double* gA, cudaStream_t st) {
  PairWeights pw;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      for (int c = 0; c < 2; c++) pw.w[i][j][c] = (i + j <= 3) ? w[i][j][c] : 0.0;
  EightBlocks<T> b, fb;
  for (int j = 0; j < 4; j++) {
    b.L[j] = (const cplx<T>*)Lam[j];
    b.ldL[j] = ldL[j];
    b.P[j] = (const cplx<T>*)Phi[j];
    fb.L[j] = (const cplx<T>*)FL[j];
    fb.ldL[j] = 1;
    fb.P[j] = (const cplx<T>*)FP[j];
  }
  b.ldP = ldP;
  fb.ldP = 1;
  // V gradient
  const int vblocks = (int)std::min<long>((ctx.N * 32 + 255) / 256, 148L * 16);
  if (M <= 16)
    k_vgrad8<T, 16><<<vblocks, 256, 0, st>>>(ctx.N, M, b, pw, gV);
  else
    k_vgrad8<T, 32><<<vblocks, 256, 0, st>>>(ctx.N, M, b, pw, gV);
  INQB_CUDA_TRY(cudaGetLastError());
  // A gradient: kinetic velocity on the coefficients, nonlocal from the pair moments
  double* acc = ctx.d_red.as<double>();
  INQB_CUDA_TRY(cudaMemsetAsync(acc, 0, 12 * sizeof(double), st));
  Recip r;
  for (int i = 0; i < 3; i++) {
    r.nr[i] = ctx.nr[i];
    for (int j = 0; j < 3; j++) r.b[i][j] = ctx.cell.rlat[i][j];
  }
  ctx.cell.cov_to_cart(ctx.kA_cov, r.kA);
  r.mask = ctx.fourier_mask;
  const int G = ctx.plan->G_tile;
  const long nelem = (long)((M + G - 1) / G) * G * ctx.N;
  // six CTAs per SM keep enough coefficient loads in flight (the per-CTA sums end in
  // six atomics each)
  const int vdb = (int)std::min<long>((nelem + 255) / 256, 148L * 6);
  if (nelem < (1L << 31) - 256L * vdb)
    k_velocity_dot8<T, unsigned><<<vdb, 256, 0, st>>>((unsigned)nelem, M, fb, pw,
                                                      TileFourier{G, ctx.plan->y1, ctx.plan->y2}, r, acc);
  else
    k_velocity_dot8<T, long><<<vdb, 256, 0, st>>>(nelem, M, fb, pw, TileFourier{G, ctx.plan->y1, ctx.plan->y2}, r,
                                                  acc);
  INQB_CUDA_TRY(cudaGetLastError());
  const ProjTables& t = ctx.proj;
  const int nchunks = (int)t.chunk_atom.size();
  if (t.nproj > 0 && nchunks > 0) {
    if (ctx.d_nlpart.bytes < (size_t)nchunks * 4 * t.L * 16 * M * sizeof(double))
      return fail(INQB_ERR_INVALID, "nonlocal moment workspace not reserved");
    double* part = ctx.d_nlpart.as<double>();
    if (M <= 16)
      k_nl_moments_pairs<T, 16><<<dim3(nchunks, (M + 15) / 16, 4), 256, 0, st>>>(
          t.L, M, b, t.d_chunk_atom.as<int>(), t.d_chunk_beg.as<int>(), t.d_atom_ptr.as<int>(),
          t.d_adj_rec.as<AdjRec<T>>(), part);
    else
      k_nl_moments_pairs<T, 32><<<dim3(nchunks, (M + 31) / 32, 4), 256, 0, st>>>(
          t.L, M, b, t.d_chunk_atom.as<int>(), t.d_chunk_beg.as<int>(), t.d_atom_ptr.as<int>(),
          t.d_adj_rec.as<AdjRec<T>>(), part);
    INQB_CUDA_TRY(cudaGetLastError());
    k_nl_combine8<<<dim3(t.nproj, t.L, (M + 31) / 32), 512, 0, st>>>(t.L, M, t.d_atom_chunk_ptr.as<int>(), part,
                                                                   t.d_scale.as<double>(), pw, acc);
    INQB_CUDA_TRY(cudaGetLastError());
  }
  k_finish_dA<<<1, 32, 0, st>>>(acc, 1.0 / (double)ctx.N, 2.0, 0.0, gA);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_half_grad(const inqb_ctx& ctx, const void* const Lam[4], const long ldL[4], const void* const Phi[4],
                     long ldP, const void* const FL[4], const void* const FP[4], const double w[4][4][2], int M,
                     double* gV, double* gA, void* stream) {
  return ctx.precision == INQB_FP64
             ? half_grad_impl<double>(ctx, Lam, ldL, Phi, ldP, FL, FP, w, M, gV, gA, (cudaStream_t)stream)
             : half_grad_impl<float>(ctx, Lam, ldL, Phi, ldP, FL, FP, w, M, gV, gA, (cudaStream_t)stream);
}

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

template <typename T>
static int lincomb_impl(long N, int M, int K, const double (*a)[2], const void* const* x, const long* ldx, void* y,
                        long ldy, cudaStream_t st) {
  LinTerms<T> t{};
  t.K = K;
  for (int k = 0; k < K; k++) {
    t.x[k] = (const cplx<T>*)x[k];
    t.ld[k] = ldx[k];
    t.a[k] = mk<T>((T)a[k][0], (T)a[k][1]);
  }
  k_lincomb<T><<<grid_for(N * M, 256), 256, 0, st>>>(N, M, t, (cplx<T>*)y, ldy);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_lincomb(int precision, long N, int M, int K, const double (*a)[2], const void* const* x, const long* ldx,
                   void* y, long ldy, void* stream) {
  if (K < 1 || K > kMaxTerms) return fail(INQB_ERR_INVALID, "linear combination of 1 to 5 blocks");
  return precision == INQB_FP64 ? lincomb_impl<double>(N, M, K, a, x, ldx, y, ldy, (cudaStream_t)stream)
                                : lincomb_impl<float>(N, M, K, a, x, ldx, y, ldy, (cudaStream_t)stream);
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

int launch_phase_kick(int precision, const inqb_ctx& ctx, void* psi, long ld, int M, const double kick[3],
                      void* stream) {
  Lat g;
  for (int i = 0; i < 3; i++) {
    g.nr[i] = ctx.nr[i];
    for (int j = 0; j < 3; j++) g.lat[i][j] = ctx.cell.lat[i][j];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const long n = ctx.N * M;
  if (precision == INQB_FP64)
    k_phase_kick<double><<<grid_for(n, 256), 256, 0, st>>>(ctx.N, M, (cplx<double>*)psi, ld, g, -kick[0], -kick[1],
                                                           -kick[2]);
  else
    k_phase_kick<float><<<grid_for(n, 256), 256, 0, st>>>(ctx.N, M, (cplx<float>*)psi, ld, g, -kick[0], -kick[1],
                                                          -kick[2]);
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
                      double* acc, double cre, double cim, double* gA, cudaStream_t st, bool tiles) {
  Recip r;
  for (int i = 0; i < 3; i++) {
    r.nr[i] = ctx.nr[i];
    for (int j = 0; j < 3; j++) r.b[i][j] = ctx.cell.rlat[i][j];
  }
  ctx.cell.cov_to_cart(ctx.kA_cov, r.kA);
  r.mask = ctx.fourier_mask;
  INQB_CUDA_TRY(cudaMemsetAsync(acc, 0, 12 * sizeof(double), st));
  // two CTAs per SM striding over the data: each CTA ends in 6 atomics on the same
  // 6 accumulators, so their count, not the data, would otherwise set the time
  if (tiles) {
    const int G = ctx.plan->G_tile;
    const long nelem = (long)((M + G - 1) / G) * G * ctx.N;
    k_velocity_dot_tiles<T><<<(int)std::min<long>((nelem + 255) / 256, 148L * 2), 256, 0, st>>>(
        nelem, M, (const cplx<T>*)U, (const cplx<T>*)W, TileFourier{G, ctx.plan->y1, ctx.plan->y2}, r, acc);
  } else {
    k_velocity_dot<T><<<(int)std::min<long>((ctx.N * M + 255) / 256, 148L * 2), 256, 0, st>>>(
        ctx.N, M, (const cplx<T>*)U, (const cplx<T>*)W, M, r, acc);
  }
  INQB_CUDA_TRY(cudaGetLastError());
  const ProjTables& t = ctx.proj;
  const int nchunks = (int)t.chunk_atom.size();
  if (t.nproj > 0 && nchunks > 0) {
    if (ctx.d_nlpart.bytes < (size_t)nchunks * t.L * 16 * M * sizeof(double))
      return fail(INQB_ERR_INVALID, "nonlocal moment workspace not reserved");
    double* part = ctx.d_nlpart.as<double>();
    k_nl_moments<T><<<dim3(nchunks, (M + 31) / 32), 256, 0, st>>>(
        t.L, M, (const cplx<T>*)u, (const cplx<T>*)w, ld, t.d_chunk_atom.as<int>(), t.d_chunk_beg.as<int>(),
        t.d_atom_ptr.as<int>(), t.d_adj_rec.as<AdjRec<T>>(), part);
    INQB_CUDA_TRY(cudaGetLastError());
    k_nl_combine<<<dim3(t.nproj, t.L, (M + 31) / 32), 512, 0, st>>>(t.L, M, t.d_atom_chunk_ptr.as<int>(), part,
                                                                   t.d_scale.as<double>(), acc);
    INQB_CUDA_TRY(cudaGetLastError());
  }
  k_finish_dA<<<1, 32, 0, st>>>(acc, 1.0 / (double)ctx.N, cre, cim, gA);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_agrad(const inqb_ctx& ctx, const void* U, const void* W, const void* u, const void* w, long ld, int M,
                 double* acc, double cre, double cim, double* gA, void* stream, bool tiles) {
  return ctx.precision == INQB_FP64
             ? agrad_impl<double>(ctx, U, W, u, w, ld, M, acc, cre, cim, gA, (cudaStream_t)stream, tiles)
             : agrad_impl<float>(ctx, U, W, u, w, ld, M, acc, cre, cim, gA, (cudaStream_t)stream, tiles);
}

}  // namespace inqb
