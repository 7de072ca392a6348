// The KB projection of H|psi> as its own kernel: projector_all::project
// (src/hamiltonian/projector_all.hpp:98-216) written as the reference shapes it, a
// gather of the orbitals at each atom's sphere points followed by a dense
// (projector x orbital) contraction and the KB scale:
//
//   proj[a][l][m] = dV ekb[a][l] sum_s beta_l(s) exp(+i (k+A).r_s) psi[pt(s)][m]
//
// Each CTA owns one (atom, orbital block) and sums all of that atom's sphere points
// in a fixed order, so the result does not depend on scheduling (no atomics).
//
//   mixed   k_project_tc: tcgen05 tensor-core MMAs, kind::tf32, FP32 accumulation in
//           tensor memory, with a split-precision correction.  A chunk of 32 sphere
//           points is gathered (cp.async, whole 512-byte orbital rows) into a
//           staging buffer, four chunks in flight; a pass over shared memory
//           transposes it into the K-major operand and splits each value x into
//           hi = tf32(x) and lo = tf32(x - hi).  The coefficient table holds the same
//           split, so hi*hi + hi*lo + lo*hi + lo*lo restores FP32 products.  Each chunk's
//           accumulator is added to FP64 registers (two accumulators in tensor
//           memory alternate, so the MMAs of one chunk overlap the read-out of the
//           previous one).
//   FP64    k_project_f64: the same decomposition on the CUDA cores in FP64.
//
// The coefficient tables B = beta exp(+i (k+A).r) depend on k + A and are rebuilt by
// k_project_table whenever the phases change.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "dft.cuh"
#include "inqb_internal.h"
#include "project.h"

namespace inqb {

namespace {

// ---------------------------------------------------------------- PTX helpers (sm_100a)
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16_zfill(void* smem, const void* gmem, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(smem)), "l"(gmem), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Wait, with every lane of the warp, for the phase with the given parity to complete;
// false if `deadline` (ns of the global timer) passes first.  The outcome is the same
// for all lanes, so the warp stays converged for the .sync.aligned loads after it.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, uint64_t deadline) {
  const uint32_t a = smem_addr(bar);
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (__all_sync(0xffffffffu, done != 0)) return true;
    if (__any_sync(0xffffffffu, globaltimer_ns() > deadline)) return false;
  }
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// tensor-memory columns held by one CTA (two accumulators of 16 columns)
constexpr uint32_t kTmemCols = 32;

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst_smem)),
               "r"(kTmemCols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTmemCols) : "memory");
}

// Shared-memory matrix descriptor of tcgen05.mma, no swizzle: start address, leading
// and stride byte offsets (16-byte units), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint64_t a = (smem_addr(p) >> 4) & 0x3FFFu;
  return a | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
         ((uint64_t)1 << 46);
}

// D[tmem] (+)= A[smem] B[smem], kind::tf32, one CTA.
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive on the mbarrier once the MMAs issued so far by this thread have completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}
// 16 consecutive FP32 columns of this warp's 32 tensor-memory lanes.  The load and its
// wait are one asm statement, so no use of the registers can be scheduled before the
// wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Round to the nearest TF32 value (10 stored mantissa bits), as an FP32 bit pattern.
__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// ---------------------------------------------------------------- tensor-core geometry
//   MMA shape M = 128 (64 orbitals x (re, im)), N = 16, K = 8 per instruction; both
//   operands K-major without swizzle (core matrices of 8 rows x 16 bytes).
//   The gather lands each sphere point's 512-byte orbital row whole in a staging
//   buffer ([point][128 floats]); the split pass transposes it into
//   A (M x K): element (row, k) at byte
//     (row % 8) * 16 + (row / 8) * 128 + (k % 4) * 4 + (k / 4) * 2048.
//   B (N x K): element (n, k) at byte
//     (n / 8) * 1024 + (k / 4) * 128 + (n % 8) * 16 + (k % 4) * 4,
//   columns n = [Re B hi (l 0-3) | Im B hi | Re B lo | Im B lo], built by
//   k_project_table in exactly this layout (one 2 KB piece per chunk).
constexpr int kRows = 2 * kProjOrbTC;            // 128
constexpr int kN = 16;
constexpr int kABytes = kProjChunk * kRows * 4;  // 16 KB per chunk
constexpr int kBBytes = kProjChunk * kN * 4;     // 2 KB per chunk
constexpr int kStages = 6;                       // gathered chunks in flight
constexpr int kStageBytes = kABytes + kBBytes;   // staging rows + B
constexpr int kTCThreads = 512;  // 16 warps: four per scheduler hide the split pass's latencies
// stages | A hi, A lo of two chunks (double-buffered against the MMAs) | barriers
constexpr size_t kSplitOff = (size_t)kStages * kStageBytes;
constexpr size_t kTCSmem = kSplitOff + 4 * (size_t)kABytes + 64;

// c_format F32 (bits 4-5), a/b format TF32 (bits 7-9, 10-12), A and B K-major (bits
// 15, 16 clear), N >> 3 (bits 17-22), M >> 4 (bits 24-28)
constexpr uint32_t kIdesc =
    (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kN >> 3) << 17) | ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ int b_index(int n, int k) {  // in floats
  return (n >> 3) * 256 + (k >> 2) * 32 + (n & 7) * 4 + (k & 3);
}

// A device-side wait that gives up: the kernel records it and returns.
constexpr uint64_t kWaitLimitNs = 1000000000ull;  // 1 s

__global__ void __launch_bounds__(kTCThreads, 1)
    k_project_tc(const cplx<float>* __restrict__ in, long ld, int M, const int* __restrict__ pc_ptr,
                 const int* __restrict__ pc_pt, const float* __restrict__ pc_b, const double* __restrict__ scale,
                 int L, double2* __restrict__ proj, int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kSplitOff + 4 * (size_t)kABytes);  // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 2);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

  const int ob = blockIdx.x, a = blockIdx.y;
  const int m0 = ob * kProjOrbTC;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int c0 = pc_ptr[a], nch = pc_ptr[a + 1] - c0;

  if (warp == 0) tmem_alloc(tmem_slot);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  auto stage_rows = [&](int s) { return smem + (size_t)s * kStageBytes; };
  auto stage_b = [&](int s) { return smem + (size_t)s * kStageBytes + kABytes; };
  auto split_hi = [&](int b) { return smem + kSplitOff + (size_t)(2 * b) * kABytes; };
  auto split_lo = [&](int b) { return smem + kSplitOff + (size_t)(2 * b + 1) * kABytes; };

  // A thread gathers the 16-byte pieces (point k = W i + warp, piece q = lane), i <
  // kPer, of a chunk, W = warps per CTA.  Their grid points are read one chunk ahead of
  // the gather, so the index load is off the critical path.
  constexpr int kWarps = kTCThreads / 32;
  constexpr int kPer = (kProjChunk * 32) / kTCThreads;  // pieces per thread
  auto fetch_points = [&](int c, int (&pt)[kPer]) {
#pragma unroll
    for (int i = 0; i < kPer; i++)
      pt[i] = (c < nch) ? pc_pt[(size_t)(c0 + c) * kProjChunk + kWarps * i + warp] : -1;
  };
  // gather of chunk c into stage s: 32 rows of 32 pieces of 16 bytes, then the B piece
  auto load_chunk = [&](int c, int s, const int (&pt)[kPer]) {
    if (c < nch) {
      unsigned char* R = stage_rows(s);
      const int q = lane;
      const int nval = M - m0 - 2 * q;  // orbitals of this piece inside the block
#pragma unroll
      for (int i = 0; i < kPer; i++) {
        const int k = kWarps * i + warp;
        const int bytes = (pt[i] < 0 || nval <= 0) ? 0 : (nval >= 2 ? 16 : 8);
        const cplx<float>* src = bytes ? in + (long)pt[i] * ld + m0 + 2 * q : in;
        cp_async16_zfill(R + k * 512 + q * 16, src, bytes);
      }
      if (tid < kBBytes / 16)
        cp_async16_zfill(stage_b(s) + tid * 16, pc_b + (size_t)(c0 + c) * (kBBytes / 4) + tid * 4, 16);
    }
    cp_async_commit();
  };

  int pts[kPer];
  for (int c = 0; c < kStages - 1; c++) {
    fetch_points(c, pts);
    load_chunk(c, c, pts);
  }
  fetch_points(kStages - 1, pts);

  double accR[4] = {0, 0, 0, 0}, accI[4] = {0, 0, 0, 0};
  // read the accumulator of chunk c into the FP64 sums (every warp: its 32 rows)
  auto drain = [&](int c) -> bool {
    if (warp >= 4) return true;  // warps 0-3 read the four lane quadrants
    const uint64_t deadline = globaltimer_ns() + kWaitLimitNs;
    if (!mbar_wait_warp(&bar[c & 1], (uint32_t)((c >> 1) & 1), deadline)) {
      *abort_flag = 1;
      return false;
    }
    tc_fence_after();
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((c & 1) * kN), v);
#pragma unroll
    for (int l = 0; l < 4; l++) {
      accR[l] += (double)v[l] + (double)v[8 + l];
      accI[l] += (double)v[4 + l] + (double)v[12 + l];
    }
    return true;
  };

  bool ok = true;
  for (int c = 0; c < nch; c++) {
    const int s = c % kStages, b = c & 1;
    cp_async_wait<kStages - 2>();
    __syncthreads();
    // transpose into the K-major operand and split: hi = tf32(x), lo = tf32(x - hi).
    // Buffer b was last read by the MMAs of chunk c - 2, which completed before its
    // accumulator was read in the previous iteration.
    {
      const float* R = reinterpret_cast<const float*>(stage_rows(s));
      unsigned char* H = split_hi(b);
      unsigned char* Lo = split_lo(b);
#pragma unroll
      for (int it = 0; it < (kRows * kProjChunk / 4) / kTCThreads; it++) {
        const int item = it * kTCThreads + tid;
        const int row = item % kRows, kc = item / kRows;  // four points kc of one operand row
        float x[4], h[4], t[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          x[j] = R[(4 * kc + j) * kRows + row];
          h[j] = tf32_round(x[j]);
          t[j] = tf32_round(x[j] - h[j]);
        }
        const int off = (row & 7) * 16 + (row >> 3) * 128 + kc * 2048;
        *reinterpret_cast<float4*>(H + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(Lo + off) = make_float4(t[0], t[1], t[2], t[3]);
      }
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t d = tmem + (uint32_t)(b * kN);
#pragma unroll
      for (int kk = 0; kk < kProjChunk / 8; kk++) {
        const uint64_t ah = smem_desc(split_hi(b) + kk * 4096, 2048, 128);
        const uint64_t al = smem_desc(split_lo(b) + kk * 4096, 2048, 128);
        const uint64_t bd = smem_desc(stage_b(s) + kk * 256, 128, 1024);
        mma_tf32(d, ah, bd, kIdesc, kk > 0 ? 1u : 0u);
        mma_tf32(d, al, bd, kIdesc, 1u);
      }
      mma_commit(&bar[b]);
    }
    // the previous chunk's accumulator, while this chunk's MMAs run
    if (c > 0 && ok) ok = drain(c - 1);
    tc_fence_before();
    __syncthreads();
    if (*abort_flag) {
      ok = false;
      break;
    }
    // stage (c - 1) % kStages is free: its rows were split in the previous iteration
    // and its B piece was read by MMAs that completed before the drain above
    load_chunk(c + kStages - 1, (c + kStages - 1) % kStages, pts);
    fetch_points(c + kStages, pts);
  }
  if (ok && nch > 0) ok = drain(nch - 1);
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  }
  cp_async_wait_all();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem);
  if (*abort_flag || !ok) return;

  // row = 32 warp + lane holds (re or im part of) orbital m0 + row / 2; even lanes
  // combine their row (Re psi) with the odd partner's (Im psi)
  double pR[4], pI[4];
#pragma unroll
  for (int l = 0; l < 4; l++) {
    pR[l] = __shfl_xor_sync(0xffffffffu, accR[l], 1);
    pI[l] = __shfl_xor_sync(0xffffffffu, accI[l], 1);
  }
  const int m = m0 + (warp * 32 + lane) / 2;
  if (warp < 4 && (lane & 1) == 0 && m < M) {
    for (int l = 0; l < L && l < 4; l++) {
      const double sc = scale[a * L + l];
      // Re = sum Re B x - Im B y; Im = sum Re B y + Im B x
      proj[((long)a * L + l) * M + m] = make_double2(sc * (accR[l] - pI[l]), sc * (pR[l] + accI[l]));
    }
  }
}

// FP64: 8 warps share one atom's points, lanes are 32 orbitals; the warps' partial
// sums meet in shared memory in a fixed order.
constexpr int kF64Threads = 256;
constexpr int kF64Orb = 32;

__global__ void __launch_bounds__(kF64Threads)
    k_project_f64(const cplx<double>* __restrict__ in, long ld, int M, const int* __restrict__ pc_ptr,
                  const int* __restrict__ pc_pt, const double* __restrict__ pc_b, const double* __restrict__ scale,
                  int L, double2* __restrict__ proj) {
  __shared__ double red[kF64Threads / 32][8][kF64Orb + 1];
  const int ob = blockIdx.x, a = blockIdx.y;
  const int m = ob * kF64Orb + (threadIdx.x & 31), warp = threadIdx.x >> 5;
  const bool valid = m < M;
  const int e0 = pc_ptr[a] * kProjChunk, e1 = pc_ptr[a + 1] * kProjChunk;
  double pr[4] = {0, 0, 0, 0}, pi[4] = {0, 0, 0, 0};
  // Software-pipelined over steps of U entries per warp: the orbital values of step
  // i + 1 are in flight while step i is summed, and the grid points of step i + 2
  // are read meanwhile.
  constexpr int U = 8;
  constexpr int STEP = (kF64Threads / 32) * U;
  auto points = [&](int eb, int (&pt)[U]) {
#pragma unroll
    for (int u = 0; u < U; u++) pt[u] = (eb + u < e1) ? pc_pt[eb + u] : -1;
  };
  auto values = [&](const int (&pt)[U], cplx<double> (&x)[U]) {
#pragma unroll
    for (int u = 0; u < U; u++) x[u] = (pt[u] >= 0 && valid) ? in[(long)pt[u] * ld + m] : mk<double>(0, 0);
  };
  int pt_cur[U], pt_nxt[U];
  cplx<double> x_cur[U];
  const int eb0 = e0 + warp * U;
  points(eb0, pt_cur);
  values(pt_cur, x_cur);
  points(eb0 + STEP, pt_nxt);
  for (int eb = eb0; eb < e1; eb += STEP) {
    cplx<double> x_nxt[U];
    values(pt_nxt, x_nxt);
    int pt_after[U];
    points(eb + 2 * STEP, pt_after);
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (pt_cur[u] < 0) continue;
      const double* b = pc_b + (size_t)(eb + u) * 8;
#pragma unroll
      for (int l = 0; l < 4; l++) {
        const double br = b[l], bi = b[4 + l];
        pr[l] = fma(br, x_cur[u].x, fma(-bi, x_cur[u].y, pr[l]));
        pi[l] = fma(br, x_cur[u].y, fma(bi, x_cur[u].x, pi[l]));
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      x_cur[u] = x_nxt[u];
      pt_cur[u] = pt_nxt[u];
      pt_nxt[u] = pt_after[u];
    }
  }
#pragma unroll
  for (int l = 0; l < 4; l++) {
    red[warp][l][threadIdx.x & 31] = pr[l];
    red[warp][4 + l][threadIdx.x & 31] = pi[l];
  }
  __syncthreads();
  if (warp == 0 && valid) {
    const int j = threadIdx.x & 31;
    for (int l = 0; l < L && l < 4; l++) {
      double sr = 0.0, si = 0.0;
      for (int w = 0; w < kF64Threads / 32; w++) {
        sr += red[w][l][j];
        si += red[w][4 + l][j];
      }
      const double sc = scale[a * L + l];
      proj[((long)a * L + l) * M + m] = make_double2(sc * sr, sc * si);
    }
  }
}

// Coefficient tables B = beta_l exp(+i (k+A).r) of every chunk entry: the mixed
// context's split TF32 pieces in the MMA's B layout, the FP64 context's plain
// [entry][Re l | Im l] rows.  One thread per entry.
template <bool TC>
__global__ void k_project_table(int nent, const float* __restrict__ relpos, const double* __restrict__ beta,
                                double k0, double k1, double k2, void* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  const double th = k0 * (double)relpos[3 * e] + k1 * (double)relpos[3 * e + 1] + k2 * (double)relpos[3 * e + 2];
  double s, c;
  sincos(th, &s, &c);
  if (TC) {
    float* o = static_cast<float*>(out) + (size_t)(e / kProjChunk) * (kBBytes / 4);
    const int k = e % kProjChunk;
#pragma unroll
    for (int l = 0; l < 4; l++) {
      const double br = beta[4 * (size_t)e + l] * c, bi = beta[4 * (size_t)e + l] * s;
      const float hr = tf32_round((float)br), hi = tf32_round((float)bi);
      o[b_index(l, k)] = hr;
      o[b_index(4 + l, k)] = hi;
      o[b_index(8 + l, k)] = tf32_round((float)(br - (double)hr));
      o[b_index(12 + l, k)] = tf32_round((float)(bi - (double)hi));
    }
  } else {
    double* o = static_cast<double*>(out) + (size_t)e * 8;
#pragma unroll
    for (int l = 0; l < 4; l++) {
      o[l] = beta[4 * (size_t)e + l] * c;
      o[4 + l] = beta[4 * (size_t)e + l] * s;
    }
  }
}

}  // namespace

size_t project_table_bytes(int precision, int nchunks) {
  return precision == INQB_FP64 ? (size_t)nchunks * kProjChunk * 8 * sizeof(double)
                                : (size_t)nchunks * (size_t)kBBytes;
}

int launch_project_table(int precision, int nchunks, const float* relpos, const double* beta, const double kA[3],
                         void* table, void* stream) {
  const int nent = nchunks * kProjChunk;
  if (nent == 0) return INQB_OK;
  const int blocks = (nent + 255) / 256;
  if (precision == INQB_FP64)
    k_project_table<false><<<blocks, 256, 0, (cudaStream_t)stream>>>(nent, relpos, beta, kA[0], kA[1], kA[2], table);
  else
    k_project_table<true><<<blocks, 256, 0, (cudaStream_t)stream>>>(nent, relpos, beta, kA[0], kA[1], kA[2], table);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

bool project_supported(int precision, const void* in, long ld) {
  if (precision == INQB_FP64) return ((uintptr_t)in % 16) == 0;
  return ((uintptr_t)in % 16) == 0 && (ld % 2) == 0;  // 16-byte pieces of complex64 rows
}

int launch_project(int precision, const void* in, long ld, int M, int nproj, int L, const int* pc_ptr,
                   const int* pc_pt, const void* table, const double* scale, double2* proj, int* err, void* stream) {
  if (nproj == 0 || M <= 0) return INQB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == INQB_FP64) {
    const dim3 grid((M + kF64Orb - 1) / kF64Orb, nproj);
    k_project_f64<<<grid, kF64Threads, 0, st>>>(static_cast<const cplx<double>*>(in), ld, M, pc_ptr, pc_pt,
                                                static_cast<const double*>(table), scale, L, proj);
  } else {
    // the shared-memory limit, set once per device (contexts on several host threads)
    static std::once_flag attr_once[64];
    int dev = 0;
    INQB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64) return fail(INQB_ERR_UNSUPPORTED, "device index above 63");
    cudaError_t attr_rc = cudaSuccess;
    std::call_once(attr_once[dev], [&attr_rc] {
      attr_rc = cudaFuncSetAttribute(k_project_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTCSmem);
    });
    INQB_CUDA_TRY(attr_rc);
    const dim3 grid((M + kProjOrbTC - 1) / kProjOrbTC, nproj);
    k_project_tc<<<grid, kTCThreads, kTCSmem, st>>>(static_cast<const cplx<float>*>(in), ld, M, pc_ptr, pc_pt,
                                                     static_cast<const float*>(table), scale, L, proj, err);
  }
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

}  // namespace inqb
