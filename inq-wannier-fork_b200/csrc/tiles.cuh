// Six-step tiles of H|psi> (src/hamiltonian/ks_hamiltonian.hpp:132-152).
//
// The y axis is split NY = Y2 * Y1 (the four-step split of the size table):
// y = y1 + Y1 * y2 and ky = ka + Y2 * kb.  Then
//   X[ka + Y2 kb] = sum_y1 w_Y1^{y1 kb} [ w_NY^{y1 ka} sum_y2 w_Y2^{y2 ka} x[y1 + Y1 y2] ]
// so a tile (x-plane ix, row class y1) of Y2 rows x NZ points finishes the z
// transform and the inner y stage on its own, and the outer y stage lands in
// the x-line pass.  Every tile moves whole 64-byte runs of G orbitals per grid
// point (G = 8 complex64 or 4 complex128; 32-byte runs for the long rows of
// 144^3), so the orbital-fastest layout [point][orbital] is read and written in
// full sectors.
//
//   pass A  k_tile_fwd  CTA (group, ix, half of the y1 classes), loops over y1: psi
//           rows -> KB projection (plane accumulators in shared memory, flushed
//           once per CTA) ->
//           z FFT -> inner y stage -> tmp[g][ka][kz][ix][y1][G]
//   pass B  k_tile_x    CTA (ka, kz, group): contiguous [ix][y1][G] block ->
//           outer y stage -> x FFT -> 1/2 |G + k + A|^2 / N -> inverse x ->
//           inverse outer y stage, in place
//   pass C  k_tile_inv  CTA (group, ix, y1): inverse inner y stage -> inverse z
//           -> nonlocal scatter -> alpha (K + V + V_nl) psi + beta base
#pragma once

#include "fft_tile.cuh"

namespace inqb {

// ---------------------------------------------------------------- cp.async
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

// Loads of data another CTA of the same launch wrote (the Fourier intermediate, the
// projection partial sums and results): through L2 (ld.global.cg), never a line an
// earlier load left in this SM's L1, so one persistent launch can run the passes.
__device__ __forceinline__ cplx<float> ld_l2(const cplx<float>* p) {
  const float2 v = __ldcg(reinterpret_cast<const float2*>(p));
  return mk<float>(v.x, v.y);
}
__device__ __forceinline__ cplx<double> ld_l2(const cplx<double>* p) {
  const double2 v = __ldcg(reinterpret_cast<const double2*>(p));
  return mk<double>(v.x, v.y);
}
__device__ __forceinline__ double2 ld_l2(const double2* p) { return __ldcg(p); }

// ---------------------------------------------------------------- geometry
template <typename T, int NX, int NY, int NZ>
struct TileGeom {
  using AX = Axis<Split<NX>::N1, Split<NX>::N2>;
  using AY = Axis<Split<NY>::N1, Split<NY>::N2>;
  using AZ = Axis<Split<NZ>::N1, Split<NZ>::N2>;
  static constexpr int Y2 = AY::N1;  // rows per tile
  static constexpr int Y1 = AY::N2;  // tiles per x-plane
  static constexpr int ZS = AZ::SLOTS;  // padded z slots per row
  // orbitals per tile: one 64-byte run per grid point, or in FP32 one 32-byte sector
  // where a 64-byte tile would pass 80 KB (long rows: 144^3), which buys a second CTA
  // per SM (measured: FP32 144^3 apply 75 -> 65 ms; FP64 is faster with 64 bytes)
  static constexpr int RUN = (sizeof(T) == 4 && Y2 * ZS * 64 > 80 * 1024) ? 32 : 64;
  static constexpr int G = RUN / (int)sizeof(cplx<T>);
  static constexpr int PV = 16 / (int)sizeof(cplx<T>);  // complex values per 16-byte vector
  static constexpr int VP = G / PV;                      // 16-byte vectors per point
  static constexpr int TILE = Y2 * ZS * G;  // complex values of a tile in shared memory
  static constexpr int PTS = Y2 * NZ;       // grid points of a tile
  static constexpr int XS = (Y1 + 1) * G;   // x-slot stride of the x-line block (one point of padding)
  static constexpr int XBLK = AX::SLOTS * XS;
  static constexpr int BLK = NX * Y1 * G;   // complex values of one tmp block [ix][y1][G]
  static constexpr int THREADS = 256;
  static constexpr size_t SMEM_MAX = 227 * 1024;  // dynamic shared memory a CTA may have
  static constexpr size_t smem_fwd(int acc_atoms, int rec_cap) {
    return sizeof(cplx<T>) * ((size_t)TILE + NY + NZ) + sizeof(double2) * (size_t)acc_atoms * LMAX * G +
           sizeof(EntRec<T>) * (size_t)rec_cap;
  }
  static constexpr size_t SMEM_X = sizeof(cplx<T>) * ((size_t)XBLK + NX) + sizeof(T) * 2 * Y1;
  static constexpr int PSTRIDE = (PTS + 1 + 3) / 4 * 4;  // ints of a tile's point index
  // pass C prefetches the input orbitals of its tile into shared memory in FP64
  // (two CTAs per SM either way, so the copy overlaps the transforms for free);
  // in FP32 the smaller footprint buys a third CTA per SM instead.
  static constexpr size_t TILE_BYTES = sizeof(cplx<T>) * (size_t)TILE;
  static constexpr bool PREFETCH = sizeof(T) == 8 && 2 * TILE_BYTES <= 150 * 1024;
  // pass C keeps four CTAs per SM in FP32 (64 registers a thread) and two with the
  // FP64 orbital prefetch (128 registers), where the shared memory allows them
  static constexpr int INV_MIN_CTAS = PREFETCH ? 2 : (TILE_BYTES <= 40 * 1024) ? 4 : 1;
  // complex values per atom segment of pass C's staged projections [l][orbital]: 64
  // bytes of padding, so that consecutive segments start in opposite halves of the
  // shared-memory banks
  static constexpr int PT_STRIDE = LMAX * G + 64 / (int)sizeof(cplx<T>);
  static constexpr size_t smem_inv(int rec_cap, int seg_cap) {
    return sizeof(cplx<T>) * ((size_t)TILE + (PREFETCH ? (size_t)PTS * G : 0) + NY + NZ) +
           sizeof(EntRec<T>) * (size_t)rec_cap + sizeof(int) * (size_t)PSTRIDE +
           sizeof(cplx<T>) * (size_t)seg_cap * PT_STRIDE;
  }
  // pass A default: two CTAs per x-plane where Y1 is even
  static constexpr int YSPLIT = (Y1 % 2 == 0) ? 2 : 1;
};

// Entry records staged in shared memory per tile; a tile with more entries
// reads its records from global memory.
constexpr int kRecCapMax = 1024;

// Start the cp.async copy of tile `tile`'s entry records (from `recs`) into R
// (cap records).  Returns the records to index with (e - roff): R when staged,
// else global memory.
template <typename T>
__device__ __forceinline__ const EntRec<T>* stage_entries(const ProjView<T>& pj, const EntRec<T>* recs, int tile,
                                                          int cap, EntRec<T>* R, int& roff) {
  const int e0 = pj.seg_ent[pj.seg_ptr[tile]], e1 = pj.seg_ent[pj.seg_ptr[tile + 1]];
  if (e1 - e0 > cap) {
    roff = 0;
    return recs;
  }
  constexpr int V = (int)(sizeof(EntRec<T>) / 16);
  const float4* src = reinterpret_cast<const float4*>(recs + e0);
  float4* dst = reinterpret_cast<float4*>(R);
  for (int q = threadIdx.x; q < (e1 - e0) * V; q += blockDim.x) cp_async16(dst + q, src + q);
  roff = e0;
  return R;
}

// Plane accumulators held in shared memory by pass A; atoms beyond this many per
// plane accumulate straight into global memory.
constexpr int kAccAtomsMax = 48;

template <typename T>
__device__ __forceinline__ int roff_base(const ProjView<T>& pj, int s0, bool on) {
  return on ? pj.seg_ent[s0] : 0;
}

// ---------------------------------------------------------------- pass A
// The body of one CTA (bx, by) of the pass; k_tile_fwd runs it at (blockIdx.x,
// blockIdx.y), the persistent batch kernel at the coordinates of a work item.
template <typename T, int NX, int NY, int NZ>
__device__ __forceinline__ void tile_fwd_body(int bx, int by, const cplx<T>* __restrict__ in, long ld, int M,
                                              cplx<T>* __restrict__ tmp, const cplx<T>* __restrict__ tw_y,
                                              const cplx<T>* __restrict__ tw_z, ProjView<T> pj, int acc_cap,
                                              int rec_cap, int ysplit, int vec) {
  using TG = TileGeom<T, NX, NY, NZ>;
  using AZ = typename TG::AZ;
  constexpr int G = TG::G, PV = TG::PV, VP = TG::VP, Y1 = TG::Y1, Y2 = TG::Y2, ZS = TG::ZS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twy = S + TG::TILE;
  cplx<T>* twz = twy + NY;
  double2* acc = reinterpret_cast<double2*>(twz + NZ);  // [acc_cap][LMAX][G]
  EntRec<T>* R = reinterpret_cast<EntRec<T>*>(acc + acc_cap * LMAX * G);  // [rec_cap]

  // ysplit CTAs share plane ix, each taking Y1 / ysplit row classes
  const int YS = ysplit, YPER = Y1 / ysplit;
  const int grp = bx, ix = by / YS, yh = by % YS;
  const int m0 = grp * G;
  const int gcount = min(G, M - m0);
  const bool v16 = vec && gcount == G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const bool proj_on = pj.nproj > 0;
  for (int i = threadIdx.x; i < NY; i += blockDim.x) twy[i] = tw_y[i];
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) twz[i] = tw_z[i];
  if (proj_on) {
    for (int i = threadIdx.x; i < acc_cap * LMAX * G; i += blockDim.x) acc[i] = make_double2(0.0, 0.0);
    // slots of the plane's atoms beyond the shared-memory accumulators start at zero
    if (pj.slots) {
      const int a0 = pj.plane_ptr[ix], na = pj.plane_ptr[ix + 1] - a0;
      for (int i = threadIdx.x; i < max(0, na - acc_cap) * LMAX * G; i += blockDim.x) {
        const int j = i % G, l = (i / G) % LMAX, sl = acc_cap + i / (G * LMAX);
        if (j < gcount) pj.slots[(((long)(a0 + sl) * YS + yh) * LMAX + l) * M + m0 + j] = make_double2(0.0, 0.0);
      }
    }
  }

  for (int y1 = yh * YPER; y1 < (yh + 1) * YPER; ++y1) {
    // -- rows y1 + Y1 r of plane ix, G orbitals per point
    if (v16) {
      for (int q = threadIdx.x; q < TG::PTS * VP; q += blockDim.x) {
        const int v = q % VP, pt = q / VP;
        const int z = pt % NZ, r = pt / NZ;
        const long p = ((long)ix * NY + y1 + Y1 * r) * NZ + z;
        cp_async16(S + (r * ZS + AZ::slot(z)) * G + v * PV, in + p * ld + m0 + v * PV);
      }
    } else {
      for (int q = threadIdx.x; q < TG::PTS * G; q += blockDim.x) {
        const int j = q % G, pt = q / G;
        const int z = pt % NZ, r = pt / NZ;
        const long p = ((long)ix * NY + y1 + Y1 * r) * NZ + z;
        S[(r * ZS + AZ::slot(z)) * G + j] = (j < gcount) ? in[p * ld + m0 + j] : mk<T>(0, 0);
      }
    }
    int roff = 0;
    const EntRec<T>* rec = proj_on ? stage_entries(pj, pj.ent_rec, ix * Y1 + y1, rec_cap, R, roff) : pj.ent_rec;
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    // -- KB projection of the tile (projector_all.hpp:104-165): lanes = (orbital j,
    // segment group); each group of G lanes walks one atom segment's entries, so a
    // warp has 32 / G segments in flight and no cross-lane reduction is needed
    if (proj_on) {
      constexpr int SGRP = 32 / G;
      const int j = lane % G, sg = lane / G;
      const int tile = ix * Y1 + y1;
      const int s0 = pj.seg_ptr[tile], s1 = pj.seg_ptr[tile + 1];
      for (int sb = s0 + warp * SGRP; sb < s1; sb += nw * SGRP) {
        const int s = sb + sg;
        if (s >= s1) continue;
        const int e0 = pj.seg_ent[s], e1 = pj.seg_ent[s + 1];
        cplx<T> a[LMAX];
#pragma unroll
        for (int l = 0; l < LMAX; ++l) a[l] = mk<T>(0, 0);
        for (int e = e0; e < e1; ++e) {
          const EntRec<T>& re = rec[e - roff];
          const int off = re.off;
          const int r = off / NZ, z = off - r * NZ;
          const cplx<T> x = mk<T>(re.ph[0], re.ph[1]) * S[(r * ZS + AZ::slot(z)) * G + j];
#pragma unroll
          for (int l = 0; l < LMAX; ++l) {
            const T b = re.beta[l];
            a[l].x = fma(b, x.x, a[l].x);
            a[l].y = fma(b, x.y, a[l].y);
          }
        }
        if (j < gcount) {
          const int sl = pj.seg_local[s];
          if (sl < acc_cap) {
            // one segment per atom in a tile, tiles separated by barriers: no race
#pragma unroll
            for (int l = 0; l < LMAX; ++l) {
              double2& d = acc[(sl * LMAX + l) * G + j];
              d.x += (double)a[l].x;
              d.y += (double)a[l].y;
            }
          } else if (pj.slots) {
            // beyond the shared-memory accumulators: this CTA's own slot in global
            // memory (zeroed at the start), the same ownership
            double2* d = pj.slots + (((long)(pj.plane_ptr[ix] + sl) * YS + yh) * LMAX) * M + m0 + j;
#pragma unroll
            for (int l = 0; l < LMAX; ++l) {
              double2 v = ld_l2(d + (long)l * M);
              v.x += (double)a[l].x;
              v.y += (double)a[l].y;
              d[(long)l * M] = v;
            }
          } else {
            const int at = pj.seg_atom[s];
#pragma unroll
            for (int l = 0; l < LMAX; ++l) {
              if (l >= pj.L) break;
              const double sc = pj.scale[at * pj.L + l];
              double2* dst = &pj.proj[((long)at * pj.L + l) * M + m0 + j];
              atomicAdd(&dst->x, sc * (double)a[l].x);
              atomicAdd(&dst->y, sc * (double)a[l].y);
            }
          }
        }
      }
      __syncthreads();
    }

    // -- z lines: (r, j), element stride G
    step1<AZ, false>(S, Y2 * G * AZ::N2, twz, [](int it, int& base, int& es, int& j2) {
      const int j = it % G, rest = it / G;
      j2 = rest % AZ::N2;
      base = (rest / AZ::N2) * ZS * G + j;
      es = G;
    });
    __syncthreads();
    step2<AZ, false>(S, Y2 * G * AZ::N1, [](int it, int& base, int& es, int& k1) {
      const int j = it % G, rest = it / G;
      k1 = rest % AZ::N1;
      base = (rest / AZ::N1) * ZS * G + j;
      es = G;
    });
    __syncthreads();

    // -- inner y stage: DFT_Y2 over the rows, twiddle w_NY^{y1 ka}, written straight
    // to tmp[g][ka][kz][ix][y1][G] (lanes along j write whole 64-byte runs)
    for (int it = threadIdx.x; it < NZ * G; it += blockDim.x) {
      const int j = it % G, kz = it / G;
      const int base = AZ::slot_of_freq(kz) * G + j;
      cplx<T> u[Y2];
#pragma unroll
      for (int r = 0; r < Y2; ++r) u[r] = S[base + r * ZS * G];
      DFT<Y2, false, T>::run(u);
#pragma unroll
      for (int ka = 1; ka < Y2; ++ka) u[ka] = u[ka] * twy[ka * Y1 + y1];
      cplx<T>* dst = tmp + (((long)grp * Y2 * NZ + kz) * NX + ix) * (Y1 * G) + y1 * G + j;
#pragma unroll
      for (int ka = 0; ka < Y2; ++ka) dst[(long)ka * NZ * TG::BLK] = u[ka];
    }
    __syncthreads();
  }

  // -- flush the plane accumulators: into this CTA's (plane, half) slots, which the
  // finish kernel adds per atom in a fixed order; without slots, proj[a][l][m] +=
  // dV ekb * sum with atomics
  if (proj_on) {
    const int a0 = pj.plane_ptr[ix];
    const int na = min(pj.plane_ptr[ix + 1] - a0, acc_cap);
    for (int i = threadIdx.x; i < na * LMAX * G; i += blockDim.x) {
      const int j = i % G, l = (i / G) % LMAX, sl = i / (G * LMAX);
      if (j >= gcount) continue;
      const double2 v = acc[i];
      if (pj.slots) {
        pj.slots[(((long)(a0 + sl) * YS + yh) * LMAX + l) * M + m0 + j] = v;
      } else if (l < pj.L) {
        const int at = pj.plane_atom[a0 + sl];
        const double sc = pj.scale[at * pj.L + l];
        double2* dst = &pj.proj[((long)at * pj.L + l) * M + m0 + j];
        atomicAdd(&dst->x, sc * v.x);
        atomicAdd(&dst->y, sc * v.y);
      }
    }
  }
}

template <typename T, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256)
    k_tile_fwd(const cplx<T>* __restrict__ in, long ld, int M, cplx<T>* __restrict__ tmp,
               const cplx<T>* __restrict__ tw_y, const cplx<T>* __restrict__ tw_z, ProjView<T> pj, int acc_cap,
               int rec_cap, int ysplit, int vec) {
  tile_fwd_body<T, NX, NY, NZ>(blockIdx.x, blockIdx.y, in, ld, M, tmp, tw_y, tw_z, pj, acc_cap, rec_cap, ysplit,
                               vec);
}

// ---------------------------------------------------------------- projection finish
// proj[a][l][m] = dV ekb[a][l] sum over the atom's (plane, half) slots, in the order of
// its planes and halves: pass A wrote one partial per slot, no atomics.  Item i =
// (a * L + l) * M + m; eight loads in flight, added in order.
template <typename T>
__device__ __forceinline__ void proj_finish_item(const ProjView<T>& pj, int M, int ysplit, long i) {
  const int m = (int)(i % M), l = (int)((i / M) % pj.L), a = (int)(i / ((long)M * pj.L));
  const int q0 = pj.aslot_ptr[a] * ysplit, q1 = pj.aslot_ptr[a + 1] * ysplit;
  double sx = 0.0, sy = 0.0;
  for (int qb = q0; qb < q1; qb += 8) {
    double2 v[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int q = qb + u;
      v[u] = make_double2(0.0, 0.0);
      if (q < q1) {
        const long slot = (long)pj.aslot[q / ysplit] * ysplit + q % ysplit;
        v[u] = ld_l2(pj.slots + (slot * LMAX + l) * M + m);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      sx += v[u].x;
      sy += v[u].y;
    }
  }
  const double sc = pj.scale[a * pj.L + l];
  pj.proj[i] = make_double2(sc * sx, sc * sy);
}

// ---------------------------------------------------------------- pass B
// One contiguous block tmp[g][ka][kz] = [ix][y1][G]; in shared memory the x
// index goes to padded slots of stride XS and (y1, j) stays contiguous.  With
// fin.slots set, the first CTAs also finish the fused projection (pass C reads it):
// thread t of CTA b handles item b * blockDim + t, so the few CTAs that carry the
// finish run beside thousands that do not.
template <typename T, int NX, int NY, int NZ>
__device__ __forceinline__ void tile_x_body(int bx, int by, cplx<T>* __restrict__ tmp,
                                            const cplx<T>* __restrict__ tw_x, KinParams<T> kp,
                                            cplx<T>* __restrict__ fout) {
  using TG = TileGeom<T, NX, NY, NZ>;
  using AX = typename TG::AX;
  constexpr int G = TG::G, PV = TG::PV, VP = TG::VP, Y1 = TG::Y1, Y2 = TG::Y2, XS = TG::XS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* X = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twx = X + TG::XBLK;
  T* kinB = reinterpret_cast<T*>(twx + NX);  // [Y1] linear and [Y1] constant term per kb
  T* kinC = kinB + Y1;

  const int kz = bx % NZ, ka = bx / NZ, grp = by;
  cplx<T>* blk = tmp + ((long)(grp * Y2 + ka) * NZ + kz) * TG::BLK;
  for (int i = threadIdx.x; i < NX; i += blockDim.x) twx[i] = tw_x[i];
  // Along an x line 1/2 |G + k + A|^2 / N = kA2 n0^2 + kinB n0 + kinC with
  // q = n1 b1 + n2 b2 + k + A:  kA2 = |b0|^2 / 2N, kinB = b0.q / N, kinC = |q|^2 / 2N
  if (threadIdx.x < Y1) {
    const int kb = threadIdx.x;
    const T n1 = (T)sym_freq(ka + Y2 * kb, NY), n2 = (T)sym_freq(kz, NZ);
    T q[3], bq = 0, qq = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      q[d] = n1 * kp.b[1][d] + n2 * kp.b[2][d] + kp.kA[d];
      bq += kp.b[0][d] * q[d];
      qq += q[d] * q[d];
    }
    kinB[kb] = kp.scale * bq;
    kinC[kb] = (T)0.5 * kp.scale * qq;
  }
  const T kinA = (T)0.5 * kp.scale *
                 (kp.b[0][0] * kp.b[0][0] + kp.b[0][1] * kp.b[0][1] + kp.b[0][2] * kp.b[0][2]);

  // outer y stage straight from HBM: a thread loads the Y1 values of its (ix, j)
  // column (lanes along j read whole 64-byte runs), DFT_Y1 over y1 -> kb, and
  // writes the column to shared memory once; two columns per thread in flight
  for (int it0 = threadIdx.x; it0 < NX * G; it0 += 2 * blockDim.x) {
    cplx<T> u[2][Y1];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int it = it0 + c * blockDim.x;
      if (it >= NX * G) continue;
      const int j = it % G, ix = it / G;
#pragma unroll
      for (int y = 0; y < Y1; ++y) u[c][y] = ld_l2(blk + (ix * Y1 + y) * G + j);
    }
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int it = it0 + c * blockDim.x;
      if (it >= NX * G) continue;
      const int j = it % G, ix = it / G;
      DFT<Y1, false, T>::run(u[c]);
      const int base = AX::slot(ix) * XS + j;
#pragma unroll
      for (int y = 0; y < Y1; ++y) X[base + y * G] = u[c][y];
    }
  }
  __syncthreads();

  auto map1 = [](int it, int& base, int& es, int& j2) {
    const int j = it % G, rest = it / G;
    j2 = rest % AX::N2;
    base = (rest / AX::N2) * G + j;
    es = XS;
  };
  auto map2 = [](int it, int& base, int& es, int& k1) {
    const int j = it % G, rest = it / G;
    k1 = rest % AX::N1;
    base = (rest / AX::N1) * G + j;
    es = XS;
  };
  const int n2 = sym_freq(kz, NZ);
  step1<AX, false>(X, Y1 * G * AX::N2, twx, map1);
  __syncthreads();
  // fout (optional): the forward coefficients of this block, before the kinetic
  // factor, as [kx][kb][G] (the adjoint's velocity terms read them)
  cplx<T>* fblk = fout ? fout + ((long)(grp * Y2 + ka) * NZ + kz) * TG::BLK : nullptr;
  step2_fwd_op_inv<AX>(X, Y1 * G * AX::N1, twx, map2, [&](int it, int kx, cplx<T> v) {
    const int kb = (it / G) / AX::N1;
    if (fblk) fblk[(kx * Y1 + kb) * G + it % G] = v;
    const int n0 = sym_freq(kx, NX);
    const T f0 = (T)n0;
    T k = fma(fma(kinA, f0, kinB[kb]), f0, kinC[kb]);
    if (kp.mask) k = outside_sphere(kp.nr, n0, sym_freq(ka + Y2 * kb, NY), n2) ? (T)0 : k - kp.shift;
    if (kp.pois != (T)0) k = ((T)2 * k < (T)1e-6) ? (T)0 : kp.pois / k;
    return k * v;
  });
  __syncthreads();
  step1_inv_transposed<AX>(X, Y1 * G * AX::N2, map1);
  __syncthreads();

  // inverse outer y stage kb -> y1, written straight back to HBM
  for (int it = threadIdx.x; it < NX * G; it += blockDim.x) {
    const int j = it % G, ix = it / G;
    const int base = AX::slot(ix) * XS + j;
    cplx<T> u[Y1];
#pragma unroll
    for (int y = 0; y < Y1; ++y) u[y] = X[base + y * G];
    DFT<Y1, true, T>::run(u);
#pragma unroll
    for (int y = 0; y < Y1; ++y) blk[(ix * Y1 + y) * G + j] = u[y];
  }
}

template <typename T, int NX, int NY, int NZ>
__global__ void __launch_bounds__(256)
    k_tile_x(cplx<T>* __restrict__ tmp, const cplx<T>* __restrict__ tw_x, KinParams<T> kp,
             cplx<T>* __restrict__ fout, ProjView<T> fin, int fin_M, int fin_ysplit) {
  if (fin.slots) {
    const long n = (long)fin.nproj * fin.L * fin_M;
    const long stride = (long)gridDim.x * gridDim.y * blockDim.x;
    for (long i = ((long)blockIdx.y * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
      proj_finish_item(fin, fin_M, fin_ysplit, i);
  }
  tile_x_body<T, NX, NY, NZ>(blockIdx.x, blockIdx.y, tmp, tw_x, kp, fout);
}

// ---------------------------------------------------------------- pass B of the plain FFTs
// DIR = 0 (to_fourier): block tmp[g][ka][kz] -> outer y stage -> forward x ->
//   out[kx][ky][kz][m] in natural frequency order (transform.hpp:115-188, sign -1).
// DIR = 1 (to_real, first half): in[kx][ky][kz][m] -> inverse x -> inverse outer
//   y stage -> block tmp[g][ka][kz]; pass C finishes with the inner y and z stages
//   and the 1/N (transform.hpp:250-332).
template <typename T, int NX, int NY, int NZ, int DIR>
__global__ void __launch_bounds__(256)
    k_tile_x_fft(cplx<T>* __restrict__ tmp, const cplx<T>* __restrict__ in, cplx<T>* __restrict__ out, long ld,
                 int M, const cplx<T>* __restrict__ tw_x, int vec) {
  using TG = TileGeom<T, NX, NY, NZ>;
  using AX = typename TG::AX;
  constexpr int G = TG::G, PV = TG::PV, VP = TG::VP, Y1 = TG::Y1, Y2 = TG::Y2, XS = TG::XS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* X = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* twx = X + TG::XBLK;

  const int kz = blockIdx.x % NZ, ka = blockIdx.x / NZ, grp = blockIdx.y;
  const int m0 = grp * G;
  const int gcount = min(G, M - m0);
  const bool v16 = vec && gcount == G;
  cplx<T>* blk = tmp + ((long)(grp * Y2 + ka) * NZ + kz) * TG::BLK;
  // point of frequency (kx, ka + Y2 kb, kz) in the orbital layout
  auto point = [&](int kx, int kb) { return ((long)kx * NY + ka + Y2 * kb) * NZ + kz; };
  auto map1 = [](int it, int& base, int& es, int& j2) {
    const int j = it % G, rest = it / G;
    j2 = rest % AX::N2;
    base = (rest / AX::N2) * G + j;
    es = XS;
  };
  auto map2 = [](int it, int& base, int& es, int& k1) {
    const int j = it % G, rest = it / G;
    k1 = rest % AX::N1;
    base = (rest / AX::N1) * G + j;
    es = XS;
  };
  for (int i = threadIdx.x; i < NX; i += blockDim.x) twx[i] = tw_x[i];

  if (DIR == 0) {
    for (int q = threadIdx.x; q < NX * Y1 * VP; q += blockDim.x) {
      const int v = q % VP, r = q / VP;
      const int y1 = r % Y1, ix = r / Y1;
      cp_async16(X + AX::slot(ix) * XS + y1 * G + v * PV, blk + (long)q * PV);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    // outer y stage: y1 -> kb
    for (int it = threadIdx.x; it < NX * G; it += blockDim.x) {
      const int j = it % G, ix = it / G;
      const int base = AX::slot(ix) * XS + j;
      cplx<T> u[Y1];
#pragma unroll
      for (int y = 0; y < Y1; ++y) u[y] = X[base + y * G];
      DFT<Y1, false, T>::run(u);
#pragma unroll
      for (int y = 0; y < Y1; ++y) X[base + y * G] = u[y];
    }
    __syncthreads();
    step1<AX, false>(X, Y1 * G * AX::N2, twx, map1);
    __syncthreads();
    step2<AX, false>(X, Y1 * G * AX::N1, map2);
    __syncthreads();
    // kx sits in slot_of_freq(kx)
    if (v16) {
      for (int q = threadIdx.x; q < NX * Y1 * VP; q += blockDim.x) {
        const int v = q % VP, r = q / VP;
        const int kb = r % Y1, kx = r / Y1;
        *reinterpret_cast<float4*>(out + point(kx, kb) * ld + m0 + v * PV) =
            *reinterpret_cast<const float4*>(X + AX::slot_of_freq(kx) * XS + kb * G + v * PV);
      }
    } else {
      for (int q = threadIdx.x; q < NX * Y1 * G; q += blockDim.x) {
        const int j = q % G, r = q / G;
        const int kb = r % Y1, kx = r / Y1;
        if (j < gcount) out[point(kx, kb) * ld + m0 + j] = X[AX::slot_of_freq(kx) * XS + kb * G + j];
      }
    }
  } else {
    // natural kx into slot(kx); the inverse from natural order leaves ix in slot_of_freq(ix)
    if (v16) {
      for (int q = threadIdx.x; q < NX * Y1 * VP; q += blockDim.x) {
        const int v = q % VP, r = q / VP;
        const int kb = r % Y1, kx = r / Y1;
        cp_async16(X + AX::slot(kx) * XS + kb * G + v * PV, in + point(kx, kb) * ld + m0 + v * PV);
      }
      cp_async_commit();
      cp_async_wait<0>();
    } else {
      for (int q = threadIdx.x; q < NX * Y1 * G; q += blockDim.x) {
        const int j = q % G, r = q / G;
        const int kb = r % Y1, kx = r / Y1;
        X[AX::slot(kx) * XS + kb * G + j] = (j < gcount) ? in[point(kx, kb) * ld + m0 + j] : mk<T>(0, 0);
      }
    }
    __syncthreads();
    step1<AX, true>(X, Y1 * G * AX::N2, twx, map1);
    __syncthreads();
    step2<AX, true>(X, Y1 * G * AX::N1, map2);
    __syncthreads();
    // inverse outer y stage: kb -> y1
    for (int it = threadIdx.x; it < NX * G; it += blockDim.x) {
      const int j = it % G, ix = it / G;
      const int base = AX::slot_of_freq(ix) * XS + j;
      cplx<T> u[Y1];
#pragma unroll
      for (int y = 0; y < Y1; ++y) u[y] = X[base + y * G];
      DFT<Y1, true, T>::run(u);
#pragma unroll
      for (int y = 0; y < Y1; ++y) X[base + y * G] = u[y];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NX * Y1 * VP; q += blockDim.x) {
      const int v = q % VP, r = q / VP;
      const int y1 = r % Y1, ix = r / Y1;
      *reinterpret_cast<float4*>(blk + (long)q * PV) =
          *reinterpret_cast<const float4*>(X + AX::slot_of_freq(ix) * XS + y1 * G + v * PV);
    }
  }
}

// ---------------------------------------------------------------- pass C
// The input orbitals of the tile (for V psi) are fetched into shared memory
// with cp.async at the start, so that read overlaps the inverse transforms.
// MODE_H = 1: the H epilogue; 0: out = alpha * (inverse transform), the second
// half of to_real (alpha = 1/N), reading neither orbitals, V nor projectors.
template <typename T, int NX, int NY, int NZ, int MODE_H>
__device__ __forceinline__ void tile_inv_body(int bx, int by, const cplx<T>* __restrict__ tmp,
                                              const cplx<T>* __restrict__ in, long ld_in, cplx<T>* __restrict__ out,
                                              long ld_out, int M, const cplx<T>* __restrict__ tw_y,
                                              const cplx<T>* __restrict__ tw_z, const ProjView<T>& pj,
                                              const EpiParams<T>& ep, int rec_cap, int seg_cap, int vec) {
  using TG = TileGeom<T, NX, NY, NZ>;
  using AZ = typename TG::AZ;
  constexpr int G = TG::G, PV = TG::PV, VP = TG::VP, Y1 = TG::Y1, Y2 = TG::Y2, ZS = TG::ZS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<T>* S = reinterpret_cast<cplx<T>*>(smem_raw);
  cplx<T>* P = S + TG::TILE;  // [PTS][G] input orbitals of the tile (PREFETCH)
  cplx<T>* twy = P + (TG::PREFETCH ? TG::PTS * G : 0);
  cplx<T>* twz = twy + NY;
  EntRec<T>* R = reinterpret_cast<EntRec<T>*>(twz + NZ);  // [rec_cap] records in point order
  int* TP = reinterpret_cast<int*>(R + rec_cap);           // [PSTRIDE] point index of the tile
  cplx<T>* PT = reinterpret_cast<cplx<T>*>(TP + TG::PSTRIDE);  // [seg_cap][PT_STRIDE] projections

  const int grp = bx, ix = by / Y1, y1 = by % Y1;
  const int m0 = grp * G;
  const int gcount = min(G, M - m0);
  const bool v16 = vec && gcount == G;

  // group 0: the (ka, kz) runs of this tile, needed first; group 1: what only the
  // epilogue reads (entry records, point index, and in FP64 the input orbitals).
  // (Reading the runs into registers for the y stage measured slower than staging.)
  for (int q = threadIdx.x; q < TG::PTS * VP; q += blockDim.x) {
    const int v = q % VP, pt = q / VP;
    const int kz = pt % NZ, ka = pt / NZ;
    cp_async16(S + (ka * ZS + AZ::slot(kz)) * G + v * PV,
               tmp + (((long)(grp * Y2 + ka) * NZ + kz) * NX + ix) * (Y1 * G) + y1 * G + v * PV);
  }
  cp_async_commit();
  const bool proj_on = MODE_H && pj.nproj > 0;
  const int tile = ix * Y1 + y1;
  int roff = 0, s0 = 0, nseg = 0;
  const EntRec<T>* rec = pj.ent_rec_pt;
  if (proj_on) {
    rec = stage_entries(pj, pj.ent_rec_pt, tile, rec_cap, R, roff);
    const int* tp = pj.pt_ptr + (long)tile * TG::PSTRIDE;
    for (int q = threadIdx.x; q < TG::PSTRIDE / 4; q += blockDim.x)
      cp_async16(reinterpret_cast<int4*>(TP) + q, reinterpret_cast<const int4*>(tp) + q);
    s0 = pj.seg_ptr[tile];
    nseg = pj.seg_ptr[tile + 1] - s0;
  }
  // the point index counts from the tile's first record
  const int rbase = (rec == R) ? 0 : roff_base(pj, s0, proj_on);
  if (MODE_H && TG::PREFETCH && v16) {
    for (int q = threadIdx.x; q < TG::PTS * VP; q += blockDim.x) {
      const int v = q % VP, pt = q / VP;
      const int z = pt % NZ, r = pt / NZ;
      const long p = ((long)ix * NY + y1 + Y1 * r) * NZ + z;
      cp_async16(P + pt * G + v * PV, in + p * ld_in + m0 + v * PV);
    }
  }
  cp_async_commit();
  for (int i = threadIdx.x; i < NY; i += blockDim.x) twy[i] = tw_y[i];
  for (int i = threadIdx.x; i < NZ; i += blockDim.x) twz[i] = tw_z[i];
  // the tile's atom projections, in the tile precision, as [segment][l][orbital] with
  // a segment stride of PT_STRIDE: the lanes of one grid point read one contiguous run
  // per l (a thread's PV orbitals as one 16-byte vector)
  const bool pt_staged = nseg <= seg_cap;
  if (proj_on && pt_staged) {
    for (int i = threadIdx.x; i < nseg * LMAX * G; i += blockDim.x) {
      const int j = i % G, l = (i / G) % LMAX, ts = i / (G * LMAX);
      cplx<T> v = mk<T>(0, 0);
      if (l < pj.L && j < gcount) {
        const double2 d = ld_l2(pj.proj + ((long)pj.seg_atom[s0 + ts] * pj.L + l) * M + m0 + j);
        v = mk<T>((T)d.x, (T)d.y);
      }
      PT[ts * TG::PT_STRIDE + l * G + j] = v;
    }
  }
  cp_async_wait<1>();
  __syncthreads();

  // inverse inner y stage: conj twiddle, inverse DFT_Y2 over ka -> rows
  for (int it = threadIdx.x; it < NZ * G; it += blockDim.x) {
    const int j = it % G, zi = it / G;
    const int base = AZ::slot(zi) * G + j;
    cplx<T> u[Y2];
#pragma unroll
    for (int ka = 0; ka < Y2; ++ka) u[ka] = S[base + ka * ZS * G];
#pragma unroll
    for (int ka = 1; ka < Y2; ++ka) u[ka] = mul_conj(u[ka], twy[ka * Y1 + y1]);
    DFT<Y2, true, T>::run(u);
#pragma unroll
    for (int r = 0; r < Y2; ++r) S[base + r * ZS * G] = u[r];
  }
  __syncthreads();
  // inverse z from natural order: element z ends in slot_of_freq(z)
  step1<AZ, true>(S, Y2 * G * AZ::N2, twz, [](int it, int& base, int& es, int& j2) {
    const int j = it % G, rest = it / G;
    j2 = rest % AZ::N2;
    base = (rest / AZ::N2) * ZS * G + j;
    es = G;
  });
  __syncthreads();
  step2<AZ, true>(S, Y2 * G * AZ::N1, [](int it, int& base, int& es, int& k1) {
    const int j = it % G, rest = it / G;
    k1 = rest % AZ::N1;
    base = (rest / AZ::N1) * ZS * G + j;
    es = G;
  });
  __syncthreads();

  // epilogue: out = alpha (K psi + (V + vshift) psi + V_nl psi) + beta base, with
  // V_nl psi(r) = sum over the entries at r of conj(exp(i (k+A).r_e)) sum_l
  // beta_e[l] proj[a_e][l] (projector_all.hpp:182-232), summed by the point's owner.
  // BE pieces of PV orbitals per thread, their loads issued together.
  // pieces per thread whose loads are issued together: FP32 keeps four CTAs per SM
  // within 64 registers a thread, FP64 (two CTAs per SM) takes more in flight
  constexpr int BE = (TG::INV_MIN_CTAS == 4) ? 2 : 4;
  cp_async_wait<0>();
  __syncthreads();
  if (!MODE_H) {
    for (int q = threadIdx.x; q < TG::PTS * VP; q += blockDim.x) {
      const int v = q % VP, pt = q / VP;
      const int z = pt % NZ, r = pt / NZ;
      const long p = ((long)ix * NY + y1 + Y1 * r) * NZ + z;
      const int jb = v * PV;
      const int sl = (r * ZS + AZ::slot_of_freq(z)) * G + jb;
      cplx<T> h[PV];
#pragma unroll
      for (int k = 0; k < PV; ++k) h[k] = ep.alpha * S[sl + k];
      if (v16) {
        float4 w;
        memcpy(&w, h, 16);
        *reinterpret_cast<float4*>(out + p * ld_out + m0 + jb) = w;
      } else {
#pragma unroll
        for (int k = 0; k < PV; ++k)
          if (jb + k < gcount) out[p * ld_out + m0 + jb + k] = h[k];
      }
    }
    return;
  }
  for (int q0 = threadIdx.x; q0 < TG::PTS * VP; q0 += BE * blockDim.x) {
    cplx<T> x[BE][PV];
    T vp[BE];
    // the first entry record of each point, fetched with the orbitals
    EntRec<T> r0[BE];
    int k0[BE], k1[BE];
#pragma unroll
    for (int b = 0; b < BE; ++b) {
      const int q = q0 + b * blockDim.x;
      k0[b] = k1[b] = 0;
      if (q >= TG::PTS * VP) continue;
      const int v = q % VP, pt = q / VP;
      const int z = pt % NZ, r = pt / NZ;
      const long p = ((long)ix * NY + y1 + Y1 * r) * NZ + z;
      const int jb = v * PV;
      if (proj_on) {
        k0[b] = TP[pt];
        k1[b] = TP[pt + 1];
        // FP32 reads records from global memory: start the first one now; FP64 has
        // them in shared memory already
        if (!TG::PREFETCH && k1[b] > k0[b]) r0[b] = rec[k0[b] + rbase];
      }
      vp[b] = ep.V[p] + ep.vshift;
      if (TG::PREFETCH && v16) {
#pragma unroll
        for (int k = 0; k < PV; ++k) x[b][k] = P[pt * G + jb + k];
      } else if (v16) {
        const float4 w = *reinterpret_cast<const float4*>(in + p * ld_in + m0 + jb);
        memcpy(x[b], &w, 16);
      } else {
#pragma unroll
        for (int k = 0; k < PV; ++k) x[b][k] = (jb + k < gcount) ? in[p * ld_in + m0 + jb + k] : mk<T>(0, 0);
      }
    }
#pragma unroll
    for (int b = 0; b < BE; ++b) {
      const int q = q0 + b * blockDim.x;
      if (q >= TG::PTS * VP) continue;
      const int v = q % VP, pt = q / VP;
      const int z = pt % NZ, r = pt / NZ;
      const long p = ((long)ix * NY + y1 + Y1 * r) * NZ + z;
      const int jb = v * PV;
      const int sl = (r * ZS + AZ::slot_of_freq(z)) * G + jb;
      cplx<T> h[PV];
#pragma unroll
      for (int k = 0; k < PV; ++k) h[k] = S[sl + k];
      if (proj_on && pt_staged) {
        for (int kk = k0[b]; kk < k1[b]; ++kk) {
          const EntRec<T> re = (!TG::PREFETCH && kk == k0[b]) ? r0[b] : rec[kk + rbase];
          const cplx<T> ph = mk<T>(re.ph[0], re.ph[1]);
          const cplx<T>* pt = PT + re.tseg * TG::PT_STRIDE + jb;
          // per orbital k, t_k = sum over l in increasing order; the PV orbitals of
          // one l are adjacent (one 16-byte load)
          cplx<T> t[PV];
#pragma unroll
          for (int k = 0; k < PV; ++k) t[k] = mk<T>(0, 0);
#pragma unroll
          for (int l = 0; l < LMAX; ++l) {
#pragma unroll
            for (int k = 0; k < PV; ++k) {
              const cplx<T> pv = pt[l * G + k];
              t[k].x = fma(re.beta[l], pv.x, t[k].x);
              t[k].y = fma(re.beta[l], pv.y, t[k].y);
            }
          }
#pragma unroll
          for (int k = 0; k < PV; ++k) h[k] = h[k] + mul_conj(t[k], ph);
        }
      } else if (proj_on) {
        // more atom segments in this tile than staged: projections from global memory
        for (int kk = k0[b]; kk < k1[b]; ++kk) {
          const EntRec<T> re = (!TG::PREFETCH && kk == k0[b]) ? r0[b] : rec[kk + rbase];
          const cplx<T> ph = mk<T>(re.ph[0], re.ph[1]);
#pragma unroll
          for (int k = 0; k < PV; ++k) {
            cplx<T> t = mk<T>(0, 0);
#pragma unroll
            for (int l = 0; l < LMAX; ++l) {
              cplx<T> pv = mk<T>(0, 0);
              if (l < pj.L && jb + k < gcount) {
                const double2 d = ld_l2(pj.proj + ((long)pj.seg_atom[s0 + re.tseg] * pj.L + l) * M + m0 + jb + k);
                pv = mk<T>((T)d.x, (T)d.y);
              }
              t.x = fma(re.beta[l], pv.x, t.x);
              t.y = fma(re.beta[l], pv.y, t.y);
            }
            h[k] = h[k] + mul_conj(t, ph);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < PV; ++k) {
        h[k].x = fma(vp[b], x[b][k].x, h[k].x);
        h[k].y = fma(vp[b], x[b][k].y, h[k].y);
        h[k] = ep.alpha * h[k];
        if (ep.base) {
          const cplx<T> bb = (jb + k < gcount) ? ep.base[p * ep.ld_base + m0 + jb + k] : mk<T>(0, 0);
          h[k] = h[k] + ep.beta * bb;
        }
      }
      if (v16) {
        float4 w;
        memcpy(&w, h, 16);
        *reinterpret_cast<float4*>(out + p * ld_out + m0 + jb) = w;
      } else {
#pragma unroll
        for (int k = 0; k < PV; ++k)
          if (jb + k < gcount) out[p * ld_out + m0 + jb + k] = h[k];
      }
    }
  }
}

template <typename T, int NX, int NY, int NZ, int MODE_H = 1>
__global__ void __launch_bounds__(256, TileGeom<T, NX, NY, NZ>::INV_MIN_CTAS)
    k_tile_inv(const cplx<T>* __restrict__ tmp, const cplx<T>* __restrict__ in, long ld_in,
               cplx<T>* __restrict__ out, long ld_out, int M, const cplx<T>* __restrict__ tw_y,
               const cplx<T>* __restrict__ tw_z, ProjView<T> pj, EpiParams<T> ep, int rec_cap, int seg_cap,
               int vec) {
  tile_inv_body<T, NX, NY, NZ, MODE_H>(blockIdx.x, blockIdx.y, tmp, in, ld_in, out, ld_out, M, tw_y, tw_z, pj, ep,
                                       rec_cap, seg_cap, vec);
}

}  // namespace inqb
