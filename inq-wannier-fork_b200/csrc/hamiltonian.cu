// Fused Kohn-Sham Hamiltonian application on sm_100a.
//
// H|psi> (src/hamiltonian/ks_hamiltonian.hpp:132-152) is computed in three
// passes over HBM, each a shared-memory tile kernel:
//
//   plane_fwd  (CTA = one x-plane, G orbitals): load psi[ix][:][:][g..g+G) ->
//              KB projection of the real-space plane (gather + contraction with
//              beta, FP64 atomics into the projection accumulators) ->
//              forward FFT along z then y -> tmp[g][yz][ix][j]
//   line_kin   (CTA = C yz-columns, G orbitals): forward FFT along x ->
//              * (1/2 |G + k + A|^2) / N -> inverse FFT along x, in place in tmp
//   plane_inv  (CTA = one x-plane, G orbitals): inverse FFT along y then z ->
//              epilogue hpsi = alpha * (K + V psi + sum_e conj(ph_e) beta_e.proj)
//              + beta * base, written straight to the [N][ld] orbital layout.
//
// The nonlocal scatter is owner-computes over a per-point list of sphere
// entries, so the result is deterministic; the projection uses FP64 atomics,
// as the reference's scatter does (src/hamiltonian/projector_all.hpp:220-232).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <map>
#include <tuple>

#include "fft_tile.cuh"
#include "inqb_internal.h"
#include "plan.h"
#include "sizes.h"

namespace inqb {

constexpr int kThreads = 256;
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

// Line split per precision: FP32 lines up to 64 points and FP64 lines up to 32
// points are transformed by one thread in registers (N2 = 1); longer lines use
// the four-step team split of the size table.
template <typename T, int N>
struct LineSplit {
  static constexpr bool single = (sizeof(T) == 4 && N <= 64) || (sizeof(T) == 8 && N <= 32);
  static constexpr int N1 = single ? N : Split<N>::N1;
  static constexpr int N2 = single ? 1 : Split<N>::N2;
};
template <typename T, int N>
using PadAxis = Axis<LineSplit<T, N>::N1, LineSplit<T, N>::N2>;  // contiguous (z or x) axis
template <typename T, int N>
using RowAxis = Axis<LineSplit<T, N>::N1, LineSplit<T, N>::N2, 0>;  // strided (y) axis

// Geometry of a plane tile: G orbitals x NY rows x ZP z-slots.  Single-thread z
// lines get an odd row stride (conflict-free row walks); team lines keep the
// padded-slot layout whose row stride is 8 mod 16.
template <typename T, int NY, int NZ>
struct PlaneGeom {
  using AY = RowAxis<T, NY>;
  using AZ = PadAxis<T, NZ>;
  static constexpr int ZP = (AZ::N2 == 1) ? (NZ % 2 == 0 ? NZ + 1 : NZ) : AZ::SLOTS;
  static constexpr int PLANE = NY * ZP;
  static constexpr int BYTES1 = PLANE * (int)sizeof(cplx<T>);
  static constexpr int G = (BYTES1 * 8 <= 77824) ? 8 : (BYTES1 * 4 <= 77824) ? 4 : (BYTES1 * 2 <= 77824) ? 2 : 1;
  static constexpr int LINES = G * (NY > NZ ? NY : NZ);
  static constexpr int THREADS =
      (AZ::N2 == 1 && AY::N2 == 1) ? (LINES < 64 ? 64 : LINES > 512 ? 512 : ((LINES + 31) / 32) * 32) : 256;
  static constexpr size_t SMEM = sizeof(cplx<T>) * ((size_t)G * PLANE + NY + NZ);
};

// x-line tile: C columns x NX x G orbitals; column stride CS = G (mod 16) words.
template <typename T, int NX>
struct LineGeom {
  using AX = Axis<Split<NX>::N1, Split<NX>::N2>;  // team split: 256 short-register threads
  static constexpr int XP = AX::SLOTS;
  template <int G>
  static constexpr int cs() { return XP * G + ((XP % 2 == 0) ? G : 0); }
};

// ---------------------------------------------------------------- kernel params
template <typename T>
struct KinParams {
  T b[3][3];  // reciprocal vectors: G_cart = sum_d n_d b[d]
  T kA[3];    // cartesian k + A
  T scale;    // 1/N folded into the kinetic factor
  int mask;   // zero the Laplacian term outside the Fourier sphere (|n/N|^2 > 1/4)
  int nr[3];
  T shift;    // 1/2 |k+A|^2 / N, moved to the epilogue when the mask is on
};

// INQ's fourier_space::outside_sphere (src/basis/fourier_space.hpp:87-93) in exact
// integer arithmetic: sum_d (n_d / N_d)^2 > 1/4.
__device__ __forceinline__ bool outside_sphere(const int nr[3], int n0, int n1, int n2) {
  const long long a = (long long)nr[1] * nr[2], b = (long long)nr[0] * nr[2], c = (long long)nr[0] * nr[1];
  const long long lhs = 4 * ((long long)n0 * n0 * a * a + (long long)n1 * n1 * b * b + (long long)n2 * n2 * c * c);
  const long long tot = (long long)nr[0] * nr[1] * nr[2];
  return lhs > tot * tot;
}

template <typename T>
__device__ __forceinline__ T kinetic(const KinParams<T>& kp, int n0, int n1, int n2) {
  T g0 = (T)n0 * kp.b[0][0] + (T)n1 * kp.b[1][0] + (T)n2 * kp.b[2][0] + kp.kA[0];
  T g1 = (T)n0 * kp.b[0][1] + (T)n1 * kp.b[1][1] + (T)n2 * kp.b[2][1] + kp.kA[1];
  T g2 = (T)n0 * kp.b[0][2] + (T)n1 * kp.b[1][2] + (T)n2 * kp.b[2][2] + kp.kA[2];
  return (T)0.5 * kp.scale * (g0 * g0 + g1 * g1 + g2 * g2);
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

// G consecutive complex values of one grid point: 16-byte vector accesses when
// the caller proved alignment (vec), element accesses otherwise.
template <typename T, int G>
__device__ __forceinline__ void load_group(const cplx<T>* __restrict__ src, cplx<T> (&v)[G], int gcount, bool vec) {
  constexpr int PER16 = 16 / (int)sizeof(cplx<T>);  // complex values per 16 bytes
  if (vec && G % PER16 == 0) {
#pragma unroll
    for (int k = 0; k < G / PER16; ++k) {
      const float4 w = reinterpret_cast<const float4*>(src)[k];
      memcpy(&v[k * PER16], &w, 16);
    }
  } else {
#pragma unroll
    for (int j = 0; j < G; ++j) v[j] = (j < gcount) ? src[j] : mk<T>(0, 0);
  }
}

template <typename T, int G>
__device__ __forceinline__ void store_group(cplx<T>* __restrict__ dst, const cplx<T> (&v)[G], int gcount, bool vec) {
  constexpr int PER16 = 16 / (int)sizeof(cplx<T>);
  if (vec && G % PER16 == 0) {
#pragma unroll
    for (int k = 0; k < G / PER16; ++k) {
      float4 w;
      memcpy(&w, &v[k * PER16], 16);
      reinterpret_cast<float4*>(dst)[k] = w;
    }
  } else {
#pragma unroll
    for (int j = 0; j < G; ++j)
      if (j < gcount) dst[j] = v[j];
  }
}

}  // namespace inqb

#include "tiles.cuh"

namespace inqb {

// ---------------------------------------------------------------- pass 1: plane forward
// do_proj = 1: H apply (projection on); 0: plain forward FFT.
template <typename T, int NY, int NZ>
__global__ void __launch_bounds__(PlaneGeom<T, NY, NZ>::THREADS)
    k_plane_fwd(const cplx<T>* __restrict__ in, long ld, int M, cplx<T>* __restrict__ tmp, int nx,
                const cplx<T>* __restrict__ tw_y, const cplx<T>* __restrict__ tw_z, ProjView<T> pj, int do_proj,
                int vec) {
  using PG = PlaneGeom<T, NY, NZ>;
  using AY = typename PG::AY;
  using AZ = typename PG::AZ;
  constexpr int G = PG::G, ZP = PG::ZP, PLANE = PG::PLANE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twy = S + G * PLANE;
  cplx<T>* twz = twy + NY;

  // orbital group fastest: the CTAs of one plane run together and share the
  // plane's projector tables and the 32-byte sectors of psi in L2
  const int grp = blockIdx.x, ix = blockIdx.y;
  const int m0 = grp * G;
  const int gcount = min(G, M - m0);
  const bool v = vec && gcount == G;
  for (int i = threadIdx.x; i < NY; i += blockDim.x) twy[i] = tw_y[i];
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) twz[i] = tw_z[i];

  const long pbase = (long)ix * NY * NZ;
  constexpr int B = 8;  // points per batch of independent loads
  for (int q0 = threadIdx.x; q0 < NY * NZ; q0 += B * blockDim.x) {
    cplx<T> vals[B][G];
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int q = q0 + b * blockDim.x;
      if (q < NY * NZ) load_group<T, G>(in + (pbase + q) * ld + m0, vals[b], gcount, v);
    }
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int q = q0 + b * blockDim.x;
      if (q < NY * NZ) {
        const int iy = q / NZ, iz = q - iy * NZ;
        const int sl = iy * ZP + AZ::slot(iz);
#pragma unroll
        for (int j = 0; j < G; ++j) S[j * PLANE + sl] = vals[b][j];
      }
    }
  }
  __syncthreads();
  // z lines: (j, iy), contiguous
  step1<AZ, false>(S, G * NY * AZ::N2, twz, [](int it, int& base, int& es, int& j2) {
    j2 = it % AZ::N2;
    base = (it / AZ::N2) * ZP;
    es = 1;
  });
  __syncthreads();
  if (AZ::N2 > 1) {
    step2<AZ, false>(S, G * NY * AZ::N1, [](int it, int& base, int& es, int& k1) {
      k1 = it % AZ::N1;
      base = (it / AZ::N1) * ZP;
      es = 1;
    });
    __syncthreads();
  }
  // y lines: (j, iz), stride ZP; threads run along z
  step1<AY, false>(S, G * NZ * AY::N2, twy, [](int it, int& base, int& es, int& j2) {
    const int iz = it % NZ, r = it / NZ;
    j2 = r % AY::N2;
    base = (r / AY::N2) * PLANE + AZ::slot(iz);
    es = ZP;
  });
  __syncthreads();
  if (AY::N2 > 1) {
    step2<AY, false>(S, G * NZ * AY::N1, [](int it, int& base, int& es, int& k1) {
      const int iz = it % NZ, r = it / NZ;
      k1 = r % AY::N1;
      base = (r / AY::N1) * PLANE + AZ::slot(iz);
      es = ZP;
    });
    __syncthreads();
  }
  // store natural (ky, kz) to tmp[grp][yz][ix][j]
  const long NYZ = (long)NY * NZ;
  for (int q = threadIdx.x; q < NY * NZ; q += blockDim.x) {
    const int ky = q / NZ, kz = q - ky * NZ;
    const int sl = AY::slot_of_freq(ky) * ZP + AZ::slot_of_freq(kz);
    cplx<T> vals[G];
#pragma unroll
    for (int j = 0; j < G; ++j) vals[j] = S[j * PLANE + sl];
    store_group<T, G>(tmp + (((long)grp * NYZ + q) * nx + ix) * G, vals, G, vec);
  }
}

// ---------------------------------------------------------------- pass 2: x lines
// MODE 0: tmp -> tmp, forward x, kinetic, inverse x (H apply)
// MODE 1: tmp -> orbital layout out, forward x only (to_fourier)
// MODE 2: orbital layout in -> tmp, inverse x, scaled by 1/N (to_real)
template <typename T, int NX, int G, int C, int MODE>
__global__ void __launch_bounds__(kThreads) k_line_x(cplx<T>* __restrict__ tmp, const cplx<T>* __restrict__ ext_in,
                                                     cplx<T>* __restrict__ ext_out, long ld, int M, int ny, int nz,
                                                     const cplx<T>* __restrict__ tw_x, KinParams<T> kp, int vec) {
  using LG = LineGeom<T, NX>;
  using AX = typename LG::AX;
  constexpr int CS = LG::template cs<G>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twx = S + C * CS;
  for (int i = threadIdx.x; i < NX; i += blockDim.x) twx[i] = tw_x[i];

  const int grp = blockIdx.y;
  const int NYZ = ny * nz;
  const int yz0 = blockIdx.x * C;
  const int ncol = min(C, NYZ - yz0);
  const int m0 = grp * G;
  const int gcount = min(G, M - m0);

  // load
  if (MODE == 2) {
    const bool v = vec && gcount == G;
    for (int q = threadIdx.x; q < C * NX; q += blockDim.x) {
      const int c = q % C, x = q / C;  // consecutive threads: consecutive yz
      cplx<T> vals[G];
      if (c < ncol) {
        load_group<T, G>(ext_in + ((long)x * NYZ + yz0 + c) * ld + m0, vals, gcount, v);
      } else {
#pragma unroll
        for (int j = 0; j < G; ++j) vals[j] = mk<T>(0, 0);
      }
#pragma unroll
      for (int j = 0; j < G; ++j) S[c * CS + AX::slot(x) * G + j] = vals[j];
    }
  } else {
    // contiguous [C][NX][G] block of tmp: 16-byte loads, batched
    const cplx<T>* src = tmp + ((long)grp * NYZ + yz0) * NX * G;
    constexpr int P = 16 / (int)sizeof(cplx<T>);  // complex values per 16 bytes
    constexpr int NV = C * NX * G / P;
    static_assert((C * NX * G) % P == 0, "tile not a whole number of 16-byte vectors");
    const int nv = ncol * NX * G / P;
    constexpr int B = 4;
    for (int q0 = threadIdx.x; q0 < NV; q0 += B * blockDim.x) {
      float4 w[B];
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int q = q0 + b * blockDim.x;
        w[b] = (q < nv) ? reinterpret_cast<const float4*>(src)[q] : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const int q = q0 + b * blockDim.x;
        if (q < NV) {
          cplx<T> vals[P];
          memcpy(vals, &w[b], 16);
#pragma unroll
          for (int k = 0; k < P; ++k) {
            const int e = q * P + k;
            const int j = e % G, r = e / G, x = r % NX, c = r / NX;
            S[c * CS + AX::slot(x) * G + j] = vals[k];
          }
        }
      }
    }
  }
  __syncthreads();

  auto map1 = [](int it, int& base, int& es, int& j2) {
    const int j = it % G, r = it / G;
    j2 = r % AX::N2;
    base = (r / AX::N2) * CS + j;
    es = G;
  };
  auto map2 = [](int it, int& base, int& es, int& k1) {
    const int j = it % G, r = it / G;
    k1 = r % AX::N1;
    base = (r / AX::N1) * CS + j;
    es = G;
  };

  if (MODE == 0) {
    if (AX::N2 == 1) {
      // whole line in registers: forward, kinetic, inverse
      for (int it = threadIdx.x; it < C * G; it += blockDim.x) {
        const int j = it % G, c = it / G;
        const int yz = yz0 + c;
        const int ky = sym_freq(yz / nz, ny), kz = sym_freq(yz % nz, nz);
        T gp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) gp[d] = (T)ky * kp.b[1][d] + (T)kz * kp.b[2][d] + kp.kA[d];
        cplx<T> v[NX];
        const int base = c * CS + j;
#pragma unroll
        for (int x = 0; x < NX; ++x) v[x] = S[base + x * G];
        DFT<NX, false, T>::run(v);
#pragma unroll
        for (int x = 0; x < NX; ++x) {
          const T kx = (T)sym_freq(x, NX);
          const T g0 = kx * kp.b[0][0] + gp[0], g1 = kx * kp.b[0][1] + gp[1], g2 = kx * kp.b[0][2] + gp[2];
          T k = (T)0.5 * kp.scale * (g0 * g0 + g1 * g1 + g2 * g2);
          if (kp.mask) k = outside_sphere(kp.nr, sym_freq(x, NX), ky, kz) ? (T)0 : k - kp.shift;
          v[x] = k * v[x];
        }
        DFT<NX, true, T>::run(v);
#pragma unroll
        for (int x = 0; x < NX; ++x) S[base + x * G] = v[x];
      }
    } else {
      step1<AX, false>(S, C * G * AX::N2, twx, map1);
      __syncthreads();
      step2_fwd_op_inv<AX>(S, C * G * AX::N1, twx, map2, [&](int it, int kx, cplx<T> v) {
        const int c = (it / G) / AX::N1;
        const int yz = yz0 + c;
        const int ky = yz / nz, kz = yz - ky * nz;
        const int n0 = sym_freq(kx, NX), n1 = sym_freq(ky, ny), n2 = sym_freq(kz, nz);
        T k = kinetic(kp, n0, n1, n2);
        if (kp.mask) k = outside_sphere(kp.nr, n0, n1, n2) ? (T)0 : k - kp.shift;
        return k * v;
      });
      __syncthreads();
      step1_inv_transposed<AX>(S, C * G * AX::N2, map1);
    }
    __syncthreads();
    cplx<T>* dst = tmp + ((long)grp * NYZ + yz0) * NX * G;
    constexpr int P = 16 / (int)sizeof(cplx<T>);
    const int nv = ncol * NX * G / P;
    for (int q = threadIdx.x; q < nv; q += blockDim.x) {
      cplx<T> vals[P];
#pragma unroll
      for (int k = 0; k < P; ++k) {
        const int e = q * P + k;
        const int j = e % G, r = e / G, x = r % NX, c = r / NX;
        vals[k] = S[c * CS + AX::slot(x) * G + j];
      }
      float4 w;
      memcpy(&w, vals, 16);
      reinterpret_cast<float4*>(dst)[q] = w;
    }
  } else if (MODE == 1) {
    step1<AX, false>(S, C * G * AX::N2, twx, map1);
    __syncthreads();
    if (AX::N2 > 1) {
      step2<AX, false>(S, C * G * AX::N1, map2);
      __syncthreads();
    }
    for (int q = threadIdx.x; q < C * NX; q += blockDim.x) {
      const int c = q % C, kx = q / C;
      if (c >= ncol) continue;
      cplx<T> vals[G];
#pragma unroll
      for (int j = 0; j < G; ++j) vals[j] = S[c * CS + AX::slot_of_freq(kx) * G + j];
      store_group<T, G>(ext_out + ((long)kx * NYZ + yz0 + c) * ld + m0, vals, gcount, vec && gcount == G);
    }
  } else {
    step1<AX, true>(S, C * G * AX::N2, twx, map1);
    __syncthreads();
    if (AX::N2 > 1) {
      step2<AX, true>(S, C * G * AX::N1, map2);
      __syncthreads();
    }
    cplx<T>* dst = tmp + ((long)grp * NYZ + yz0) * NX * G;
    for (int q = threadIdx.x; q < ncol * NX * G; q += blockDim.x) {
      const int j = q % G, r = q / G, x = r % NX, c = r / NX;
      dst[q] = kp.scale * S[c * CS + AX::slot_of_freq(x) * G + j];
    }
  }
}

// ---------------------------------------------------------------- pass 3: plane inverse + epilogue
// MODE_H = 1: H epilogue; 0: plain copy (to_real).
template <typename T, int NY, int NZ, int MODE_H>
__global__ void __launch_bounds__(PlaneGeom<T, NY, NZ>::THREADS)
    k_plane_inv(const cplx<T>* __restrict__ tmp, const cplx<T>* __restrict__ in, long ld_in,
                cplx<T>* __restrict__ out, long ld_out, int M, int nx, const cplx<T>* __restrict__ tw_y,
                const cplx<T>* __restrict__ tw_z, ProjView<T> pj, EpiParams<T> ep, int vec) {
  using PG = PlaneGeom<T, NY, NZ>;
  using AY = typename PG::AY;
  using AZ = typename PG::AZ;
  constexpr int G = PG::G, ZP = PG::ZP, PLANE = PG::PLANE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twy = S + G * PLANE;
  cplx<T>* twz = twy + NY;

  const int grp = blockIdx.x, ix = blockIdx.y;
  const int m0 = grp * G;
  const int gcount = min(G, M - m0);
  const bool v = vec && gcount == G;
  for (int i = threadIdx.x; i < NY; i += blockDim.x) twy[i] = tw_y[i];
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) twz[i] = tw_z[i];

  const long NYZ = (long)NY * NZ;
  constexpr int B = 8;  // points per batch of independent loads
  for (int q0 = threadIdx.x; q0 < NY * NZ; q0 += B * blockDim.x) {
    cplx<T> vals[B][G];
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int q = q0 + b * blockDim.x;
      if (q < NY * NZ) load_group<T, G>(tmp + (((long)grp * NYZ + q) * nx + ix) * G, vals[b], G, vec);
    }
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const int q = q0 + b * blockDim.x;
      if (q < NY * NZ) {
        const int iy = q / NZ, iz = q - iy * NZ;
        const int sl = iy * ZP + AZ::slot(iz);
#pragma unroll
        for (int j = 0; j < G; ++j) S[j * PLANE + sl] = vals[b][j];
      }
    }
  }
  __syncthreads();
  step1<AY, true>(S, G * NZ * AY::N2, twy, [](int it, int& base, int& es, int& j2) {
    const int iz = it % NZ, r = it / NZ;
    j2 = r % AY::N2;
    base = (r / AY::N2) * PLANE + AZ::slot(iz);
    es = ZP;
  });
  __syncthreads();
  if (AY::N2 > 1) {
    step2<AY, true>(S, G * NZ * AY::N1, [](int it, int& base, int& es, int& k1) {
      const int iz = it % NZ, r = it / NZ;
      k1 = r % AY::N1;
      base = (r / AY::N1) * PLANE + AZ::slot(iz);
      es = ZP;
    });
    __syncthreads();
  }
  step1<AZ, true>(S, G * NY * AZ::N2, twz, [](int it, int& base, int& es, int& j2) {
    j2 = it % AZ::N2;
    base = (it / AZ::N2) * ZP;
    es = 1;
  });
  __syncthreads();
  if (AZ::N2 > 1) {
    step2<AZ, true>(S, G * NY * AZ::N1, [](int it, int& base, int& es, int& k1) {
      k1 = it % AZ::N1;
      base = (it / AZ::N1) * ZP;
      es = 1;
    });
    __syncthreads();
  }

  const long pbase = (long)ix * NYZ;
  constexpr int BE = 4;  // points per batch in the epilogue
  for (int q0 = threadIdx.x; q0 < NY * NZ; q0 += BE * blockDim.x) {
    cplx<T> x[BE][G], bb[BE][G];
    T vp[BE];
    if (MODE_H) {
#pragma unroll
      for (int b = 0; b < BE; ++b) {
        const int q = q0 + b * blockDim.x;
        if (q < NY * NZ) {
          const long p = pbase + q;
          vp[b] = ep.V[p] + ep.vshift;
          load_group<T, G>(in + p * ld_in + m0, x[b], gcount, v);
          if (ep.base) load_group<T, G>(ep.base + p * ep.ld_base + m0, bb[b], gcount, v);
        }
      }
    }
#pragma unroll
    for (int b = 0; b < BE; ++b) {
      const int q = q0 + b * blockDim.x;
      if (q >= NY * NZ) continue;
      const int iy = q / NZ, iz = q - iy * NZ;
      const int sl = AY::slot_of_freq(iy) * ZP + AZ::slot_of_freq(iz);
      const long p = pbase + q;
      cplx<T> h[G];
#pragma unroll
      for (int j = 0; j < G; ++j) h[j] = S[j * PLANE + sl];
      if (MODE_H) {
#pragma unroll
        for (int j = 0; j < G; ++j) {
          h[j].x = fma(vp[b], x[b][j].x, h[j].x);
          h[j].y = fma(vp[b], x[b][j].y, h[j].y);
          h[j] = ep.alpha * h[j];
          if (ep.base) h[j] = h[j] + ep.beta * bb[b][j];
        }
      }
      store_group<T, G>(out + p * ld_out + m0, h, gcount, v);
    }
  }
}

// ---------------------------------------------------------------- phases
template <typename T>
__global__ void k_phases(int nent, const float* __restrict__ relpos, double k0, double k1, double k2,
                         cplx<T>* __restrict__ phase, EntRec<T>* __restrict__ rec, EntRec<T>* __restrict__ rec_pt,
                         const int* __restrict__ pt_pos, AdjRec<T>* __restrict__ adj,
                         const int* __restrict__ atom_pos) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  const double th = k0 * (double)relpos[3 * e] + k1 * (double)relpos[3 * e + 1] + k2 * (double)relpos[3 * e + 2];
  double s, c;
  sincos(th, &s, &c);
  phase[e] = mk<T>((T)c, (T)s);
  rec[e].ph[0] = (T)c;
  rec[e].ph[1] = (T)s;
  rec_pt[pt_pos[e]].ph[0] = (T)c;
  rec_pt[pt_pos[e]].ph[1] = (T)s;
  adj[atom_pos[e]].ph[0] = (T)c;
  adj[atom_pos[e]].ph[1] = (T)s;
}

// ---------------------------------------------------------------- plan instantiation
template <typename T, int NX, int NY, int NZ>
struct Kernels {
  using PG = PlaneGeom<T, NY, NZ>;
  using LG = LineGeom<T, NX>;
  static constexpr int G = PG::G;
  static constexpr int CS = LG::template cs<G>();
  // x-line tile: 128 register lines (single-thread split) or 256 team items per CTA
  static constexpr int LINE_THREADS = (LG::AX::N2 == 1) ? 128 : kThreads;
  static constexpr int CX = (LINE_THREADS / (G * LG::AX::N2) > 0) ? (LINE_THREADS / (G * LG::AX::N2)) : 1;
  static constexpr size_t line_smem = sizeof(cplx<T>) * ((size_t)CX * CS + NX);
};

static bool aligned16(const void* p, long ld, size_t esz) {
  return ((uintptr_t)p % 16 == 0) && ((ld * (long)esz) % 16 == 0);
}

template <typename T, int NX, int NY, int NZ>
static int launch_h_impl(const LaunchArgs& a) {
  using K = Kernels<T, NX, NY, NZ>;
  using PG = typename K::PG;
  constexpr int G = K::G;
  static bool attr_done[64] = {};
  int dev = 0;
  INQB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 64 && !attr_done[dev]) {
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_plane_fwd<T, NY, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)PG::SMEM));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_plane_inv<T, NY, NZ, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)PG::SMEM));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_line_x<T, NX, G, K::CX, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::line_smem));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_line_x<T, NX, G, K::CX, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::line_smem));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_line_x<T, NX, G, K::CX, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::line_smem));
    attr_done[dev] = true;
  }
  const int groups = (a.M + G - 1) / G;
  const cplx<T>* tw = reinterpret_cast<const cplx<T>*>(a.tw);
  const cplx<T>* twx = tw;
  const cplx<T>* twy = tw + NX;
  const cplx<T>* twz = tw + NX + NY;
  cplx<T>* tmp = reinterpret_cast<cplx<T>*>(a.tmp);
  cudaStream_t st = (cudaStream_t)a.stream;
  const size_t esz = sizeof(cplx<T>);
  const bool gvec = (G * esz) % 16 == 0;
  const int vin = gvec && aligned16(a.in, a.ld_in, esz) && aligned16(tmp, 0, esz);
  const int vout = gvec && aligned16(a.out, a.ld_out, esz) && (a.base == nullptr || aligned16(a.base, a.ld_base, esz)) &&
                   (a.mode != LaunchArgs::H || aligned16(a.in, a.ld_in, esz));

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

  const dim3 gplane(groups, NX);
  const dim3 gline((NY * NZ + K::CX - 1) / K::CX, groups);
  if (a.mode == LaunchArgs::H) {
    using TG = TileGeom<T, NX, NY, NZ>;
    constexpr int GT = TG::G;
    static bool tile_attr_done[64] = {};
    if (dev < 64 && !tile_attr_done[dev]) {
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_fwd<T, NX, NY, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)TG::smem_fwd(kAccAtomsMax, kRecCapMax)));
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_x<T, NX, NY, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)TG::SMEM_X));
      INQB_CUDA_TRY(cudaFuncSetAttribute(k_tile_inv<T, NX, NY, NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)TG::smem_inv(kRecCapMax, kAccAtomsMax)));
      tile_attr_done[dev] = true;
    }
    const int tgroups = (a.M + GT - 1) / GT;
    // 16-byte vectors of G orbitals: full groups, aligned pointers and leading dimensions
    const int tvin = aligned16(a.in, a.ld_in, esz);
    const int tvout = tvin && aligned16(a.out, a.ld_out, esz);
    const int acc_cap = pj.nproj > 0 ? std::min(pj.max_plane_atoms, kAccAtomsMax) : 0;
    const int rec_cap = pj.nproj > 0 ? std::min(pj.max_tile_ent, kRecCapMax) : 0;
    const int seg_cap = pj.nproj > 0 ? std::min(pj.max_tile_seg, kAccAtomsMax) : 0;
    if (pj.nproj > 0 && pj.pt_stride != TG::PSTRIDE)
      return fail(INQB_ERR_INVALID, "projector tables were built for another tiling of this grid");
    if (pj.nproj > 0)
      INQB_CUDA_TRY(cudaMemsetAsync(pj.proj, 0, sizeof(double2) * (size_t)pj.nproj * pj.L * a.M, st));
    if (a.events[0]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[0], st));
    k_tile_fwd<T, NX, NY, NZ><<<dim3(tgroups, NX * TG::YSPLIT), TG::THREADS, TG::smem_fwd(acc_cap, rec_cap), st>>>(
        (const cplx<T>*)a.in, a.ld_in, a.M, tmp, twy, twz, pj, acc_cap, rec_cap, tvin);
    if (a.events[1]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[1], st));
    k_tile_x<T, NX, NY, NZ><<<dim3(TG::Y2 * NZ, tgroups), TG::THREADS, TG::SMEM_X, st>>>(tmp, twx, kp);
    if (a.events[2]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[2], st));
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
    const int rec_cap_inv = TG::PREFETCH ? rec_cap : 0;
    k_tile_inv<T, NX, NY, NZ><<<dim3(tgroups, NX * TG::Y1), TG::THREADS, TG::smem_inv(rec_cap_inv, seg_cap), st>>>(
        tmp, (const cplx<T>*)a.in, a.ld_in, (cplx<T>*)a.out, a.ld_out, a.M, twy, twz, pj, ep, rec_cap_inv, seg_cap,
        tvout);
    if (a.events[3]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[3], st));
  } else if (a.mode == LaunchArgs::FFT_FWD) {
    k_plane_fwd<T, NY, NZ><<<gplane, PG::THREADS, PG::SMEM, st>>>((const cplx<T>*)a.in, a.ld_in, a.M, tmp, NX, twy,
                                                                 twz, pj, 0, vin);
    k_line_x<T, NX, G, K::CX, 1><<<gline, K::LINE_THREADS, K::line_smem, st>>>(tmp, nullptr, (cplx<T>*)a.out, a.ld_out,
                                                                        a.M, NY, NZ, twx, kp, vout);
  } else {
    k_line_x<T, NX, G, K::CX, 2><<<gline, K::LINE_THREADS, K::line_smem, st>>>(tmp, (const cplx<T>*)a.in, nullptr,
                                                                        a.ld_in, a.M, NY, NZ, twx, kp, vin);
    EpiParams<T> ep{};
    k_plane_inv<T, NY, NZ, 0><<<gplane, PG::THREADS, PG::SMEM, st>>>(tmp, nullptr, 0, (cplx<T>*)a.out, a.ld_out,
                                                                     a.M, NX, twy, twz, pj, ep, vout);
  }
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

template <typename T>
static int launch_phases_impl(int nent, const float* relpos, const double kA[3], void* phase, void* rec,
                              void* rec_pt, const int* pt_pos, void* adj, const int* atom_pos, void* stream) {
  if (nent == 0) return INQB_OK;
  k_phases<T><<<(nent + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      nent, relpos, kA[0], kA[1], kA[2], (cplx<T>*)phase, (EntRec<T>*)rec, (EntRec<T>*)rec_pt, pt_pos,
      (AdjRec<T>*)adj, atom_pos);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_phases(int precision, int nent, const float* relpos, const double kA[3], void* phase, void* rec,
                  void* rec_pt, const int* pt_pos, void* adj, const int* atom_pos, void* stream) {
  return precision == INQB_FP64
             ? launch_phases_impl<double>(nent, relpos, kA, phase, rec, rec_pt, pt_pos, adj, atom_pos, stream)
             : launch_phases_impl<float>(nent, relpos, kA, phase, rec, rec_pt, pt_pos, adj, atom_pos, stream);
}

// ---------------------------------------------------------------- registry
template <typename T, int NX, int NY, int NZ>
static Plan make_plan() {
  using K = Kernels<T, NX, NY, NZ>;
  Plan p;
  p.G = K::G;
  p.G_tile = TileGeom<T, NX, NY, NZ>::G;
  p.launch = &launch_h_impl<T, NX, NY, NZ>;
  return p;
}

#define INQB_CUBIC(N) {std::make_tuple(N, N, N, 0), make_plan<double, N, N, N>()}, \
                      {std::make_tuple(N, N, N, 1), make_plan<float, N, N, N>()},
#define INQB_GRID(X, Y, Z) {std::make_tuple(X, Y, Z, 0), make_plan<double, X, Y, Z>()}, \
                           {std::make_tuple(X, Y, Z, 1), make_plan<float, X, Y, Z>()},

static const std::map<std::tuple<int, int, int, int>, Plan>& registry() {
  static const std::map<std::tuple<int, int, int, int>, Plan> reg = {
      INQB_CUBIC(16) INQB_CUBIC(20) INQB_CUBIC(24) INQB_CUBIC(32) INQB_CUBIC(40) INQB_CUBIC(48)
      INQB_CUBIC(64)
      INQB_GRID(18, 24, 20)
  };
  return reg;
}

const Plan* find_plan(int nx, int ny, int nz, int precision) {
  const auto& reg = registry();
  auto it = reg.find(std::make_tuple(nx, ny, nz, precision == INQB_FP64 ? 0 : 1));
  return it == reg.end() ? nullptr : &it->second;
}

}  // namespace inqb
