// The persistent batch launch (batch.h): k_batch_h runs the three tile passes of a
// batch of cells (the bodies of tiles.cuh) as work items taken from a device ticket
// counter, with bounded waits on per-(cell, group) completion counters.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "batch.h"
#include "launch_h.cuh"

namespace inqb {

namespace {

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// One thread waits until *c >= target.  False when the error word is set meanwhile
// (another CTA gave up) or when limit_ns passes (then this CTA sets it).
__device__ bool wait_counter(const unsigned* c, unsigned target, int* err, long long limit_ns) {
  const uint64_t t0 = global_ns();
  while (ld_acquire(c) < target) {
    if (ld_acquire(reinterpret_cast<const unsigned*>(err)) != 0u) return false;
    if ((long long)(global_ns() - t0) > limit_ns) {
      atomicExch(err, 1);
      return false;
    }
    __nanosleep(256);
  }
  return true;
}

template <typename T>
struct BatchParams {
  BatchCell<T> cells[kMaxBatchCells];
};

// One (grid, stage) body over the item's count CTAs of the pass (a barrier between
// them, as the shared memory is reused).  c lives in the kernel's parameter space, so
// the body reads its arguments from the constant bank, as in a kernel of its own.
template <typename T, int N, int STAGE>
__device__ __forceinline__ void run_stage(const BatchCell<T>& c, int bx, int by, int count) {
  const cplx<T>* twx = c.tw;
  const cplx<T>* twy = c.tw + N;
  const cplx<T>* twz = c.tw + 2 * N;
  if (STAGE == kStageA) {
    for (int t = 0; t < count; t++) {
      if (t) __syncthreads();
      tile_fwd_body<T, N, N, N>(bx, by + t, c.in, c.ld_in, c.M, c.tmp, twy, twz, c.pj, c.acc_cap, c.rec_cap_a,
                                c.ysplit, c.vin);
    }
  } else if (STAGE == kStageFinish) {
    // proj[a][l][m] of the G orbitals m of group bx, each in the fixed order of its slots
    constexpr int G = TileGeom<T, N, N, N>::G;
    const int m0 = bx * G;
    const int n = c.pj.nproj * c.pj.L * G;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const int m = m0 + i % G;
      if (m < c.M) proj_finish_item(c.pj, c.M, c.ysplit, (long)(i / G) * c.M + m);
    }
  } else if (STAGE == kStageB) {
    for (int t = 0; t < count; t++) {
      if (t) __syncthreads();
      tile_x_body<T, N, N, N>(bx + t, by, c.tmp, twx, c.kp, nullptr);
    }
  } else {
    for (int t = 0; t < count; t++) {
      if (t) __syncthreads();
      tile_inv_body<T, N, N, N, 1>(bx, by + t, c.tmp, c.in, c.ld_in, c.out, c.ld_out, c.M, twy, twz, c.pj, c.ep,
                                   c.rec_cap_inv, c.seg_cap, c.vio);
    }
  }
}

template <typename T, int N>
__device__ __forceinline__ void run_item(const BatchCell<T>& c, const BatchItem& it) {
  // it is the item in shared memory: its fields are read where they are used
  switch (it.stage) {
    case kStageA:
      run_stage<T, N, kStageA>(c, it.bx, it.by, it.count);
      break;
    case kStageFinish:
      run_stage<T, N, kStageFinish>(c, it.bx, it.by, it.count);
      break;
    case kStageB:
      run_stage<T, N, kStageB>(c, it.bx, it.by, it.count);
      break;
    default:
      run_stage<T, N, kStageC>(c, it.bx, it.by, it.count);
  }
}

__device__ __forceinline__ void red_release(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Thread 0 keeps the queue moving beside the work: while the CTA runs an item, the
// next item's descriptor is on its way into shared memory (cp.async) and the ticket of
// the one after it is being taken; at the top of the loop it waits for the next
// item's inputs.  Only that ticket stays in a register across the item's work.  The
// CTA publishes an item's completion as a grid barrier arrives: a CTA barrier, then
// one release add by thread 0.
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2)
    k_batch_h(const __grid_constant__ BatchParams<T> p, const BatchItem* __restrict__ items, int nitems,
              unsigned* __restrict__ ctr, int* __restrict__ err, long long wait_ns) {
  static_assert(sizeof(BatchItem) % 16 == 0, "items are copied in 16-byte pieces");
  __shared__ __align__(16) BatchItem s_it, s_nx;
  __shared__ int s_go, s_have;
  // copy item t (if any) into s_nx
  auto fetch = [&](unsigned t) {
    s_have = t < (unsigned)nitems;
    if (t < (unsigned)nitems) {
      const char* src = reinterpret_cast<const char*>(items + t);
#pragma unroll
      for (int q = 0; q < (int)(sizeof(BatchItem) / 16); q++)
        cp_async16(reinterpret_cast<char*>(&s_nx) + 16 * q, src + 16 * q);
    }
    cp_async_commit();
  };
  unsigned t_next = 0;
  if (threadIdx.x == 0) {
    fetch(atomicAdd(&ctr[0], 1u));
    t_next = atomicAdd(&ctr[0], 1u);
  }
  while (true) {
    if (threadIdx.x == 0) {
      cp_async_wait<0>();
      int go = s_have;
      if (go)
        go = (s_nx.wait >= 0) ? wait_counter(&ctr[s_nx.wait], (unsigned)s_nx.target, err, wait_ns)
                              : ld_acquire(reinterpret_cast<const unsigned*>(err)) == 0u;
      s_go = go;
      if (go) {
        s_it = s_nx;
        fetch(t_next);
        t_next = atomicAdd(&ctr[0], 1u);
      }
    }
    __syncthreads();
    if (!s_go) break;
    const int cell = s_it.cell;
    switch (s_it.kind) {
#define INQB_BATCH_CASE(K, N)                  \
  case K:                                      \
    run_item<T, N>(p.cells[cell], s_it);       \
    break;
      INQB_BATCH_GRIDS(INQB_BATCH_CASE)
#undef INQB_BATCH_CASE
      default:
        break;
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_it.signal >= 0) red_release(&ctr[s_it.signal], (unsigned)s_it.count);
  }
  if (threadIdx.x == 0) cp_async_wait<0>();
}

// Raise the kernel's dynamic shared-memory limit to smem (never lowers it, so plans
// of other batches stay launchable); the static words of the kernel count against the
// 227 KB a CTA may have.
template <typename T>
int ensure_batch_smem(size_t smem) {
  static std::mutex mu;
  static size_t cur[64] = {};
  int dev = 0;
  INQB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 64) return fail(INQB_ERR_UNSUPPORTED, "device index above 63");
  if (smem + 1024 > 227 * 1024) return fail(INQB_ERR_UNSUPPORTED, "batch cell tiles exceed shared memory");
  std::lock_guard<std::mutex> lock(mu);
  if (smem > cur[dev]) {
    INQB_CUDA_TRY(cudaFuncSetAttribute(k_batch_h<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cur[dev] = smem;
  }
  return INQB_OK;
}

}  // namespace

int build_batch_items(const std::vector<BatchCellDesc>& cells, int ctas, std::vector<BatchItem>& items,
                      int& ncounters, int tiles_per_item, int lag) {
  items.clear();
  ncounters = 0;
  if (ctas < 1) return fail(INQB_ERR_INVALID, "batch launch without CTAs");
  // units (cell, group) in cell order
  std::vector<std::pair<int, int>> units;
  long total = 0;
  for (size_t c = 0; c < cells.size(); c++) {
    const BatchCellDesc& d = cells[c];
    if (d.kind < 0 || d.groups <= 0 || d.a_per <= 0 || d.b_per <= 0 || d.c_per <= 0)
      return fail(INQB_ERR_INVALID, "batch cell without work");
    for (int g = 0; g < d.groups; g++) units.push_back({(int)c, g});
    total += (long)d.groups * (d.a_per + d.finish + d.b_per + d.c_per);
  }
  const long U = (long)units.size();
  if (2 * U + 1 > (1L << 30) || total > (1L << 30)) return fail(INQB_ERR_INVALID, "batch too large");
  // about eight items per CTA, at most kBatchTilesPerItem CTAs of a pass each
  const int K = tiles_per_item > 0 ? tiles_per_item
                             : (int)std::max(1L, std::min<long>(kBatchTilesPerItem, total / (8L * ctas)));
  // lag = units: all A items, then the finish and B items, then the C items (measured
  // faster than shorter lags, which mix more passes and grids on an SM at once)
  if (lag <= 0) lag = (int)std::max(1L, U);
  auto item = [&](int u, int stage, int bx, int by, int count, int wait, int target, int signal) {
    BatchItem it{};
    it.cell = units[u].first;
    it.stage = stage;
    it.bx = bx;
    it.by = by;
    it.count = count;
    it.wait = wait;
    it.target = target;
    it.signal = signal;
    it.kind = cells[it.cell].kind;
    items.push_back(it);
  };
  auto cA = [](long u) { return (int)(1 + 2 * u); };
  auto cB = [](long u) { return (int)(2 + 2 * u); };
  items.reserve((size_t)(total / K + 3 * U));
  for (long s = 0; s < U + 2L * lag; s++) {
    if (s < U) {  // pass A grid (groups, NX * ysplit): by advances
      const BatchCellDesc& d = cells[units[s].first];
      for (int y = 0; y < d.a_per; y += K) item((int)s, kStageA, units[s].second, y, std::min(K, d.a_per - y), -1, 0,
                                                cA(s));
    }
    const long b = s - lag;
    if (b >= 0 && b < U) {  // finish, then pass B grid (Y2 * NZ, groups): bx advances
      const BatchCellDesc& d = cells[units[b].first];
      const int g = units[b].second;
      if (d.finish) item((int)b, kStageFinish, g, 0, 1, cA(b), d.a_per, cB(b));
      for (int x = 0; x < d.b_per; x += K)
        item((int)b, kStageB, x, g, std::min(K, d.b_per - x), cA(b), d.a_per, cB(b));
    }
    const long c = s - 2L * lag;
    if (c >= 0 && c < U) {  // pass C grid (groups, NX * Y1): by advances
      const BatchCellDesc& d = cells[units[c].first];
      for (int y = 0; y < d.c_per; y += K)
        item((int)c, kStageC, units[c].second, y, std::min(K, d.c_per - y), cB(c), d.b_per + d.finish, -1);
    }
  }
  ncounters = (int)(1 + 2 * U);
  return INQB_OK;
}

int batch_ctas_per_sm(int precision, size_t smem, int* ctas) {
  int n = 0;
  if (precision == INQB_FP64) {
    INQB_TRY(ensure_batch_smem<double>(smem));
    INQB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_h<double>, 256, smem));
  } else {
    INQB_TRY(ensure_batch_smem<float>(smem));
    INQB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_h<float>, 256, smem));
  }
  *ctas = n;
  return n > 0 ? INQB_OK : fail(INQB_ERR_UNSUPPORTED, "persistent batch kernel does not fit on an SM");
}

template <typename T>
int launch_batch_t(const void* cells, int ncells, size_t cell_bytes, const BatchItem* items, int nitems,
                   unsigned* counters, int* err, long long wait_ns, int ctas, size_t smem, cudaStream_t st) {
  if (ncells < 1 || ncells > kMaxBatchCells || cell_bytes != sizeof(BatchCell<T>))
    return fail(INQB_ERR_INVALID, "batch cell descriptors do not match the kernel");
  INQB_TRY(ensure_batch_smem<T>(smem));
  BatchParams<T> prm;
  memcpy(prm.cells, cells, cell_bytes * (size_t)ncells);
  k_batch_h<T><<<ctas, 256, smem, st>>>(prm, items, nitems, counters, err, wait_ns);
  return INQB_OK;
}

int launch_batch(int precision, const void* cells, int ncells, size_t cell_bytes, const BatchItem* items, int nitems,
                 unsigned* counters, int ncounters, int* err, long long wait_ns, int ctas, size_t smem,
                 void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  INQB_CUDA_TRY(cudaMemsetAsync(counters, 0, sizeof(unsigned) * (size_t)ncounters, st));
  if (precision == INQB_FP64)
    INQB_TRY(launch_batch_t<double>(cells, ncells, cell_bytes, items, nitems, counters, err, wait_ns, ctas, smem, st));
  else
    INQB_TRY(launch_batch_t<float>(cells, ncells, cell_bytes, items, nitems, counters, err, wait_ns, ctas, smem, st));
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

}  // namespace inqb
