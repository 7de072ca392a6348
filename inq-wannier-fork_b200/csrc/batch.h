// The persistent launch of a batch of cells: one kernel over work items (cell,
// stage, CTA coordinates) that CTAs take from a device ticket counter.
//
// Stages per (cell, orbital group g), a "unit":
//   A       first tile pass, the (g, x-plane, half) CTAs                 -> signals cA[u]
//   finish  the fused projection's fixed-order finish for group g        waits cA, signals cB
//   B       second tile pass, the (ka, kz) CTAs of group g                 waits cA, signals cB
//   C       third tile pass, the (g, tile) CTAs                           waits cB
// An item runs a few consecutive CTAs of one pass of one unit.  Step s of the queue
// holds the A items of unit s, the finish and B items of unit s - lag and the C items
// of unit s - 2 lag; the default lag (the number of units) queues all A items, then
// all finish and B items, then all C items.  Every item therefore waits only on items
// with smaller tickets: the CTA holding the smallest unfinished ticket always has its
// inputs, and the launch needs no co-residency (no cooperative launch).  A wait gives up after a
// time limit: the CTA sets the error word, every CTA stops at its next item or wait,
// and the host reports INQB_ERR_TIMEOUT.
#pragma once

#include <cstddef>
#include <vector>

namespace inqb {

// The grids compiled into the persistent kernel (cubic NX = NY = NZ).
#define INQB_BATCH_GRIDS(X) X(0, 16) X(1, 20) X(2, 24) X(3, 32) X(4, 40) X(5, 48)

inline int batch_kind(int nx, int ny, int nz) {
  if (nx != ny || nx != nz) return -1;
#define INQB_BATCH_KIND(K, N) \
  if (nx == N) return K;
  INQB_BATCH_GRIDS(INQB_BATCH_KIND)
#undef INQB_BATCH_KIND
  return -1;
}

enum BatchStage { kStageA = 0, kStageFinish = 1, kStageB = 2, kStageC = 3 };

// One work item: count consecutive CTAs of its pass, starting at coordinates (bx,
// by) (the pass's varying coordinate advances: by for A and C, bx for B), the counter
// it waits on (-1: none) until it reaches target, and the counter it adds count to
// when done (counters count CTAs of a pass, not items).
struct BatchItem {
  int cell, stage, bx, by;
  int count, wait, target, signal;
  int kind, pad[3];  // kind: the cell's index in INQB_BATCH_GRIDS
};

// Most CTAs of a pass per work item
constexpr int kBatchTilesPerItem = 4;

// One cell as the plan sees it.  bytes holds the kernel's descriptor of the cell
// (BatchCell<T> of launch_h.cuh), filled by the grid's launcher.
struct BatchCellDesc {
  int kind = -1;      // index in INQB_BATCH_GRIDS
  int groups = 0;     // orbital groups
  int a_per = 0;      // pass A items per group (NX * ysplit)
  int b_per = 0;      // pass B items per group (Y2 * NZ)
  int c_per = 0;      // pass C items per group (NX * Y1)
  int finish = 0;     // 1: a projection finish item per group
  size_t smem = 0;    // largest dynamic shared memory of its stages
  std::vector<unsigned char> bytes;
};

// Work list for a launch of ctas CTAs: the pipelined order above, up to
// kBatchTilesPerItem CTAs of a pass per item (fewer where the batch is small, so
// every stage has items for every CTA); counters [0] = ticket, then cA, cB per unit.
// tiles_per_item / lag > 0 override the choices (tests).  Host code, no device calls.
int build_batch_items(const std::vector<BatchCellDesc>& cells, int ctas, std::vector<BatchItem>& items,
                      int& ncounters, int tiles_per_item = 0, int lag = 0);

// CTAs of k_batch_h that fit on one SM with the given dynamic shared memory.
int batch_ctas_per_sm(int precision, size_t smem, int* ctas);

// Cells one launch takes: their descriptors travel as kernel parameters (32 KB at
// most), which the kernel reads from the constant bank as a kernel of its own would.
constexpr int kMaxBatchCells = 64;

// One launch over the items: counters zeroed, then ctas CTAs of 256 threads.  cells:
// ncells host descriptors (BatchCell<T>, cell_bytes each).
int launch_batch(int precision, const void* cells, int ncells, size_t cell_bytes, const BatchItem* items, int nitems,
                 unsigned* counters, int ncounters, int* err, long long wait_ns, int ctas, size_t smem,
                 void* stream);

}  // namespace inqb
