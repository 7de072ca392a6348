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

template <int N>
using PadAxis = Axis<Split<N>::N1, Split<N>::N2>;  // contiguous (z or x) axis
template <int N>
using RowAxis = Axis<Split<N>::N1, Split<N>::N2, 0>;  // strided (y) axis

// Orbitals per plane tile: largest power of two <= 8 whose tile fits ~76 KB.
template <typename T, int NY, int NZ>
constexpr int plane_group() {
  constexpr int bytes1 = NY * PadAxis<NZ>::SLOTS * (int)sizeof(cplx<T>);
  return (bytes1 * 8 <= 77824) ? 8 : (bytes1 * 4 <= 77824) ? 4 : (bytes1 * 2 <= 77824) ? 2 : 1;
}

// ---------------------------------------------------------------- kernel params
template <typename T>
struct KinParams {
  T b[3][3];  // reciprocal vectors: G_cart = sum_d n_d b[d]
  T kA[3];    // cartesian k + A
  T scale;    // 1/N folded into the kinetic factor
};

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
  const cplx<T>* base;      // optional [N][ld_base]
  long ld_base;
  cplx<T> alpha, beta;      // out = alpha * H in + beta * base
};

// ---------------------------------------------------------------- projection (pass 1)
// Sum over the sphere entries of plane ix:  proj[a][l][m] += scale[a][l] *
// sum_e beta_e[l] exp(+i (k+A).r_e) psi(r_e)[m]   (projector_all.hpp:104-165).
template <typename T, int G, int ZP, int PLANE, typename AZ>
__device__ __forceinline__ void project_plane(const cplx<T>* S, int NZ, int ix, int m0, int gcount, int M,
                                              const ProjView<T>& pj) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int s0 = pj.seg_ptr[ix], s1 = pj.seg_ptr[ix + 1];
  const cplx<T>* phase = (const cplx<T>*)pj.ent_phase;
  for (int s = s0 + warp; s < s1; s += nw) {
    const int a = pj.seg_atom[s];
    const int e0 = pj.seg_ent[s], e1 = pj.seg_ent[s + 1];
    cplx<T> acc[LMAX][G];
#pragma unroll
    for (int l = 0; l < LMAX; ++l)
#pragma unroll
      for (int j = 0; j < G; ++j) acc[l][j] = mk<T>(0, 0);
    for (int e = e0 + lane; e < e1; e += 32) {
      const int off = pj.ent_off[e];
      const int sl = (off / NZ) * ZP + AZ::slot(off % NZ);
      const cplx<T> ph = phase[e];
      T b[LMAX];
#pragma unroll
      for (int l = 0; l < LMAX; ++l) b[l] = (l < pj.L) ? pj.ent_beta[(long)e * pj.L + l] : (T)0;
#pragma unroll
      for (int j = 0; j < G; ++j) {
        cplx<T> x = ph * S[j * PLANE + sl];
#pragma unroll
        for (int l = 0; l < LMAX; ++l) {
          acc[l][j].x = fma(b[l], x.x, acc[l][j].x);
          acc[l][j].y = fma(b[l], x.y, acc[l][j].y);
        }
      }
    }
#pragma unroll
    for (int l = 0; l < LMAX; ++l)
#pragma unroll
      for (int j = 0; j < G; ++j)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          acc[l][j].x += __shfl_xor_sync(0xffffffffu, acc[l][j].x, o);
          acc[l][j].y += __shfl_xor_sync(0xffffffffu, acc[l][j].y, o);
        }
#pragma unroll
    for (int l = 0; l < LMAX; ++l)
#pragma unroll
      for (int j = 0; j < G; ++j) {
        if (lane == ((l * G + j) & 31) && l < pj.L && j < gcount) {
          const double sc = pj.scale[a * pj.L + l];
          double2* dst = &pj.proj[((long)a * pj.L + l) * M + m0 + j];
          atomicAdd(&dst->x, sc * (double)acc[l][j].x);
          atomicAdd(&dst->y, sc * (double)acc[l][j].y);
        }
      }
  }
}

// ---------------------------------------------------------------- pass 1: plane forward
// MODE_H: H apply (projection on); MODE_FFT: plain forward FFT.
template <typename T, int NY, int NZ, int G>
__global__ void __launch_bounds__(kThreads) k_plane_fwd(const cplx<T>* __restrict__ in, long ld, int M,
                                                        cplx<T>* __restrict__ tmp, int nx,
                                                        const cplx<T>* __restrict__ tw_y,
                                                        const cplx<T>* __restrict__ tw_z, ProjView<T> pj,
                                                        int do_proj) {
  using AY = RowAxis<NY>;
  using AZ = PadAxis<NZ>;
  constexpr int ZP = AZ::SLOTS;
  constexpr int PLANE = NY * ZP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twy = S + G * PLANE;
  cplx<T>* twz = twy + NY;

  const int ix = blockIdx.x, grp = blockIdx.y;
  const int m0 = grp * G;
  const int gcount = min(G, M - m0);
  for (int i = threadIdx.x; i < NY; i += blockDim.x) twy[i] = tw_y[i];
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) twz[i] = tw_z[i];

  const long pbase = (long)ix * NY * NZ;
  for (int q = threadIdx.x; q < NY * NZ; q += blockDim.x) {
    const int iy = q / NZ, iz = q - iy * NZ;
    const cplx<T>* src = in + (pbase + q) * ld + m0;
    const int sl = iy * ZP + AZ::slot(iz);
#pragma unroll
    for (int j = 0; j < G; ++j) S[j * PLANE + sl] = (j < gcount) ? src[j] : mk<T>(0, 0);
  }
  __syncthreads();
  if (do_proj && pj.nproj > 0) {
    project_plane<T, G, ZP, PLANE, AZ>(S, NZ, ix, m0, gcount, M, pj);
    __syncthreads();
  }
  // z lines: (j, iy), contiguous
  step1<AZ, false>(S, G * NY * AZ::N2, twz, [](int it, int& base, int& es, int& j2) {
    j2 = it % AZ::N2;
    base = (it / AZ::N2) * ZP;
    es = 1;
  });
  __syncthreads();
  step2<AZ, false>(S, G * NY * AZ::N1, [](int it, int& base, int& es, int& k1) {
    k1 = it % AZ::N1;
    base = (it / AZ::N1) * ZP;
    es = 1;
  });
  __syncthreads();
  // y lines: (j, iz), stride ZP; threads run along z
  step1<AY, false>(S, G * NZ * AY::N2, twy, [](int it, int& base, int& es, int& j2) {
    const int iz = it % NZ, r = it / NZ;
    j2 = r % AY::N2;
    base = (r / AY::N2) * PLANE + AZ::slot(iz);
    es = ZP;
  });
  __syncthreads();
  step2<AY, false>(S, G * NZ * AY::N1, [](int it, int& base, int& es, int& k1) {
    const int iz = it % NZ, r = it / NZ;
    k1 = r % AY::N1;
    base = (r / AY::N1) * PLANE + AZ::slot(iz);
    es = ZP;
  });
  __syncthreads();
  // store natural (ky, kz) to tmp[grp][yz][ix][j]
  const long NYZ = (long)NY * NZ;
  for (int q = threadIdx.x; q < NY * NZ; q += blockDim.x) {
    const int ky = q / NZ, kz = q - ky * NZ;
    const int sl = AY::slot_of_freq(ky) * ZP + AZ::slot_of_freq(kz);
    cplx<T>* dst = tmp + (((long)grp * NYZ + q) * nx + ix) * G;
#pragma unroll
    for (int j = 0; j < G; ++j) dst[j] = S[j * PLANE + sl];
  }
}

// ---------------------------------------------------------------- pass 2: x lines
// MODE 0: tmp -> tmp, forward x, kinetic, inverse x (H apply)
// MODE 1: tmp -> orbital layout out, forward x only (to_fourier)
// MODE 2: orbital layout in -> tmp, inverse x, scaled by 1/N (to_real)
template <typename T, int NX, int G, int C, int MODE>
__global__ void __launch_bounds__(kThreads) k_line_x(cplx<T>* __restrict__ tmp, const cplx<T>* __restrict__ ext_in,
                                                     cplx<T>* __restrict__ ext_out, long ld, int M, int ny, int nz,
                                                     const cplx<T>* __restrict__ tw_x, KinParams<T> kp) {
  using AX = PadAxis<NX>;
  constexpr int XP = AX::SLOTS;
  constexpr int CS = XP * G;
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
    for (int q = threadIdx.x; q < C * NX; q += blockDim.x) {
      const int c = q % C, x = q / C;  // consecutive threads: consecutive yz
      const cplx<T>* src = ext_in + ((long)x * NYZ + yz0 + c) * ld + m0;
#pragma unroll
      for (int j = 0; j < G; ++j)
        S[c * CS + AX::slot(x) * G + j] = (c < ncol && j < gcount) ? src[j] : mk<T>(0, 0);
    }
  } else {
    const cplx<T>* src = tmp + ((long)grp * NYZ + yz0) * NX * G;
    for (int q = threadIdx.x; q < C * NX * G; q += blockDim.x) {
      const int j = q % G, r = q / G, x = r % NX, c = r / NX;
      S[c * CS + AX::slot(x) * G + j] = (c < ncol) ? src[q] : mk<T>(0, 0);
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
    step1<AX, false>(S, C * G * AX::N2, twx, map1);
    __syncthreads();
    step2_fwd_op_inv<AX>(S, C * G * AX::N1, twx, map2, [&](int it, int kx, cplx<T> v) {
      const int c = (it / G) / AX::N1;
      const int yz = yz0 + c;
      const int ky = yz / nz, kz = yz - ky * nz;
      const T k = kinetic(kp, sym_freq(kx, NX), sym_freq(ky, ny), sym_freq(kz, nz));
      return k * v;
    });
    __syncthreads();
    step1_inv_transposed<AX>(S, C * G * AX::N2, map1);
    __syncthreads();
    cplx<T>* dst = tmp + ((long)grp * NYZ + yz0) * NX * G;
    for (int q = threadIdx.x; q < ncol * NX * G; q += blockDim.x) {
      const int j = q % G, r = q / G, x = r % NX, c = r / NX;
      dst[q] = S[c * CS + AX::slot(x) * G + j];
    }
  } else if (MODE == 1) {
    step1<AX, false>(S, C * G * AX::N2, twx, map1);
    __syncthreads();
    step2<AX, false>(S, C * G * AX::N1, map2);
    __syncthreads();
    for (int q = threadIdx.x; q < C * NX; q += blockDim.x) {
      const int c = q % C, kx = q / C;
      if (c >= ncol) continue;
      cplx<T>* dst = ext_out + ((long)kx * NYZ + yz0 + c) * ld + m0;
      for (int j = 0; j < gcount; ++j) dst[j] = S[c * CS + AX::slot_of_freq(kx) * G + j];
    }
  } else {
    step1<AX, true>(S, C * G * AX::N2, twx, map1);
    __syncthreads();
    step2<AX, true>(S, C * G * AX::N1, map2);
    __syncthreads();
    cplx<T>* dst = tmp + ((long)grp * NYZ + yz0) * NX * G;
    for (int q = threadIdx.x; q < ncol * NX * G; q += blockDim.x) {
      const int j = q % G, r = q / G, x = r % NX, c = r / NX;
      dst[q] = kp.scale * S[c * CS + AX::slot_of_freq(x) * G + j];
    }
  }
}

// ---------------------------------------------------------------- pass 3: plane inverse + epilogue
// MODE_H = 1: H epilogue; 0: plain copy (to_real).
template <typename T, int NY, int NZ, int G, int MODE_H>
__global__ void __launch_bounds__(kThreads) k_plane_inv(const cplx<T>* __restrict__ tmp,
                                                        const cplx<T>* __restrict__ in, long ld_in,
                                                        cplx<T>* __restrict__ out, long ld_out, int M, int nx,
                                                        const cplx<T>* __restrict__ tw_y,
                                                        const cplx<T>* __restrict__ tw_z, ProjView<T> pj,
                                                        EpiParams<T> ep) {
  using AY = RowAxis<NY>;
  using AZ = PadAxis<NZ>;
  constexpr int ZP = AZ::SLOTS;
  constexpr int PLANE = NY * ZP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twy = S + G * PLANE;
  cplx<T>* twz = twy + NY;

  const int ix = blockIdx.x, grp = blockIdx.y;
  const int m0 = grp * G;
  const int gcount = min(G, M - m0);
  for (int i = threadIdx.x; i < NY; i += blockDim.x) twy[i] = tw_y[i];
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) twz[i] = tw_z[i];

  const long NYZ = (long)NY * NZ;
  for (int q = threadIdx.x; q < NY * NZ; q += blockDim.x) {
    const int iy = q / NZ, iz = q - iy * NZ;
    const cplx<T>* src = tmp + (((long)grp * NYZ + q) * nx + ix) * G;
    const int sl = iy * ZP + AZ::slot(iz);
#pragma unroll
    for (int j = 0; j < G; ++j) S[j * PLANE + sl] = src[j];
  }
  __syncthreads();
  step1<AY, true>(S, G * NZ * AY::N2, twy, [](int it, int& base, int& es, int& j2) {
    const int iz = it % NZ, r = it / NZ;
    j2 = r % AY::N2;
    base = (r / AY::N2) * PLANE + AZ::slot(iz);
    es = ZP;
  });
  __syncthreads();
  step2<AY, true>(S, G * NZ * AY::N1, [](int it, int& base, int& es, int& k1) {
    const int iz = it % NZ, r = it / NZ;
    k1 = r % AY::N1;
    base = (r / AY::N1) * PLANE + AZ::slot(iz);
    es = ZP;
  });
  __syncthreads();
  step1<AZ, true>(S, G * NY * AZ::N2, twz, [](int it, int& base, int& es, int& j2) {
    j2 = it % AZ::N2;
    base = (it / AZ::N2) * ZP;
    es = 1;
  });
  __syncthreads();
  step2<AZ, true>(S, G * NY * AZ::N1, [](int it, int& base, int& es, int& k1) {
    k1 = it % AZ::N1;
    base = (it / AZ::N1) * ZP;
    es = 1;
  });
  __syncthreads();

  const long pbase = (long)ix * NYZ;
  const cplx<T>* phase = (const cplx<T>*)pj.ent_phase;
  for (int q = threadIdx.x; q < NY * NZ; q += blockDim.x) {
    const int iy = q / NZ, iz = q - iy * NZ;
    const int sl = AY::slot_of_freq(iy) * ZP + AZ::slot_of_freq(iz);
    const long p = pbase + q;
    cplx<T> h[G];
#pragma unroll
    for (int j = 0; j < G; ++j) h[j] = S[j * PLANE + sl];
    if (MODE_H) {
      const T v = ep.V[p];
      const cplx<T>* src = in + p * ld_in + m0;
#pragma unroll
      for (int j = 0; j < G; ++j)
        if (j < gcount) {
          const cplx<T> x = src[j];
          h[j].x = fma(v, x.x, h[j].x);
          h[j].y = fma(v, x.y, h[j].y);
        }
      if (pj.nproj > 0) {
        const int e0 = pj.pt_ptr[p], e1 = pj.pt_ptr[p + 1];
        for (int ei = e0; ei < e1; ++ei) {
          const int e = pj.pt_ent[ei];
          const int a = pj.ent_atom[e];
          const cplx<T> ph = phase[e];
          T b[LMAX];
#pragma unroll
          for (int l = 0; l < LMAX; ++l) b[l] = (l < pj.L) ? pj.ent_beta[(long)e * pj.L + l] : (T)0;
#pragma unroll
          for (int j = 0; j < G; ++j) {
            if (j >= gcount) continue;
            cplx<T> s = mk<T>(0, 0);
#pragma unroll
            for (int l = 0; l < LMAX; ++l) {
              if (l >= pj.L) continue;
              const double2 pr = pj.proj[((long)a * pj.L + l) * M + m0 + j];
              s.x = fma(b[l], (T)pr.x, s.x);
              s.y = fma(b[l], (T)pr.y, s.y);
            }
            h[j] = h[j] + mul_conj(s, ph);
          }
        }
      }
      cplx<T>* dst = out + p * ld_out + m0;
      const cplx<T>* bsrc = ep.base ? ep.base + p * ep.ld_base + m0 : nullptr;
#pragma unroll
      for (int j = 0; j < G; ++j)
        if (j < gcount) {
          cplx<T> r = ep.alpha * h[j];
          if (bsrc) r = r + ep.beta * bsrc[j];
          dst[j] = r;
        }
    } else {
      cplx<T>* dst = out + p * ld_out + m0;
#pragma unroll
      for (int j = 0; j < G; ++j)
        if (j < gcount) dst[j] = h[j];
    }
  }
}

// ---------------------------------------------------------------- phases
template <typename T>
__global__ void k_phases(int nent, const float* __restrict__ relpos, double k0, double k1, double k2,
                         cplx<T>* __restrict__ phase) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  const double th = k0 * (double)relpos[3 * e] + k1 * (double)relpos[3 * e + 1] + k2 * (double)relpos[3 * e + 2];
  double s, c;
  sincos(th, &s, &c);
  phase[e] = mk<T>((T)c, (T)s);
}

// ---------------------------------------------------------------- plan instantiation
template <typename T, int NX, int NY, int NZ>
struct Kernels {
  static constexpr int G = plane_group<T, NY, NZ>();
  static constexpr int CX = (kThreads / (G * Split<NX>::N2) > 0) ? (kThreads / (G * Split<NX>::N2)) : 1;
  static constexpr size_t plane_smem =
      sizeof(cplx<T>) * ((size_t)G * NY * PadAxis<NZ>::SLOTS + NY + NZ);
  static constexpr size_t line_smem = sizeof(cplx<T>) * ((size_t)CX * PadAxis<NX>::SLOTS * G + NX);
};

template <typename T, int NX, int NY, int NZ>
static int launch_h_impl(const LaunchArgs& a) {
  using K = Kernels<T, NX, NY, NZ>;
  constexpr int G = K::G;
  static bool attr_done = false;
  if (!attr_done) {
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_plane_fwd<T, NY, NZ, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::plane_smem));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_plane_inv<T, NY, NZ, G, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::plane_smem));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_plane_inv<T, NY, NZ, G, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::plane_smem));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_line_x<T, NX, G, K::CX, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::line_smem));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_line_x<T, NX, G, K::CX, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::line_smem));
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_line_x<T, NX, G, K::CX, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)K::line_smem));
    attr_done = true;
  }
  const int groups = (a.M + G - 1) / G;
  const cplx<T>* tw = reinterpret_cast<const cplx<T>*>(a.tw);
  const cplx<T>* twx = tw;
  const cplx<T>* twy = tw + NX;
  const cplx<T>* twz = tw + NX + NY;
  cplx<T>* tmp = reinterpret_cast<cplx<T>*>(a.tmp);
  cudaStream_t st = (cudaStream_t)a.stream;

  ProjView<T> pj = *reinterpret_cast<const ProjView<T>*>(a.proj_view);
  KinParams<T> kp;
  for (int d = 0; d < 3; d++) {
    for (int c = 0; c < 3; c++) kp.b[d][c] = (T)a.rlat[d][c];
    kp.kA[d] = (T)a.kA_cart[d];
  }
  kp.scale = (T)(1.0 / ((double)NX * NY * NZ));

  const dim3 gplane(NX, groups);
  const dim3 gline((NY * NZ + K::CX - 1) / K::CX, groups);
  if (a.mode == LaunchArgs::H) {
    if (pj.nproj > 0)
      INQB_CUDA_TRY(cudaMemsetAsync(pj.proj, 0, sizeof(double2) * (size_t)pj.nproj * pj.L * a.M, st));
    if (a.events[0]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[0], st));
    k_plane_fwd<T, NY, NZ, G><<<gplane, kThreads, K::plane_smem, st>>>(
        (const cplx<T>*)a.in, a.ld_in, a.M, tmp, NX, twy, twz, pj, 1);
    if (a.events[1]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[1], st));
    k_line_x<T, NX, G, K::CX, 0><<<gline, kThreads, K::line_smem, st>>>(tmp, nullptr, nullptr, 0, a.M, NY, NZ,
                                                                        twx, kp);
    if (a.events[2]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[2], st));
    EpiParams<T> ep;
    ep.V = (const T*)a.V;
    ep.base = (const cplx<T>*)a.base;
    ep.ld_base = a.ld_base;
    ep.alpha = mk<T>((T)a.alpha[0], (T)a.alpha[1]);
    ep.beta = mk<T>((T)a.beta[0], (T)a.beta[1]);
    k_plane_inv<T, NY, NZ, G, 1><<<gplane, kThreads, K::plane_smem, st>>>(
        tmp, (const cplx<T>*)a.in, a.ld_in, (cplx<T>*)a.out, a.ld_out, a.M, NX, twy, twz, pj, ep);
    if (a.events[3]) INQB_CUDA_TRY(cudaEventRecord((cudaEvent_t)a.events[3], st));
  } else if (a.mode == LaunchArgs::FFT_FWD) {
    k_plane_fwd<T, NY, NZ, G><<<gplane, kThreads, K::plane_smem, st>>>(
        (const cplx<T>*)a.in, a.ld_in, a.M, tmp, NX, twy, twz, pj, 0);
    k_line_x<T, NX, G, K::CX, 1><<<gline, kThreads, K::line_smem, st>>>(tmp, nullptr, (cplx<T>*)a.out, a.ld_out,
                                                                        a.M, NY, NZ, twx, kp);
  } else {
    k_line_x<T, NX, G, K::CX, 2><<<gline, kThreads, K::line_smem, st>>>(tmp, (const cplx<T>*)a.in, nullptr,
                                                                        a.ld_in, a.M, NY, NZ, twx, kp);
    EpiParams<T> ep{};
    k_plane_inv<T, NY, NZ, G, 0><<<gplane, kThreads, K::plane_smem, st>>>(
        tmp, nullptr, 0, (cplx<T>*)a.out, a.ld_out, a.M, NX, twy, twz, pj, ep);
  }
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

template <typename T>
static int launch_phases_impl(int nent, const float* relpos, const double kA[3], void* phase, void* stream) {
  if (nent == 0) return INQB_OK;
  k_phases<T><<<(nent + 255) / 256, 256, 0, (cudaStream_t)stream>>>(nent, relpos, kA[0], kA[1], kA[2],
                                                                   (cplx<T>*)phase);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

int launch_phases(int precision, int nent, const float* relpos, const double kA[3], void* phase, void* stream) {
  return precision == INQB_FP64 ? launch_phases_impl<double>(nent, relpos, kA, phase, stream)
                                : launch_phases_impl<float>(nent, relpos, kA, phase, stream);
}

// ---------------------------------------------------------------- registry
template <typename T, int NX, int NY, int NZ>
static Plan make_plan() {
  using K = Kernels<T, NX, NY, NZ>;
  Plan p;
  p.G = K::G;
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
