// The work list of the persistent batch launch (build_batch_items, batch.h) against
// the protocol k_batch_h runs, on the host: every pass CTA appears in exactly one
// item, every counter's waiters wait for exactly the CTAs that signal it, every item
// waits only on items with smaller tickets, and a simulation of P CTAs (each holding
// the ticket it runs and the next one it took, steps interleaved at random) runs every
// item after its inputs and never deadlocks, for P = 1 .. 64 and 1 .. 5 CTAs of a pass
// per item.  A plan with one unreachable wait stalls: the items the kernel's time
// limit then ends.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>

#include "../../inq-wannier-fork_b200/csrc/batch.h"
#include "../../inq-wannier-fork_b200/csrc/inqb_internal.h"

using namespace inqb;

static std::vector<BatchCellDesc> random_cells(std::mt19937& rng) {
  std::uniform_int_distribution<int> ncell(1, 9), kind(0, 5), groups(1, 5), fin(0, 1), ys(1, 3);
  const int grids[6] = {16, 20, 24, 32, 40, 48};
  const int y2[6] = {4, 5, 8, 8, 8, 8};  // rows per tile of the size table's split
  std::vector<BatchCellDesc> cells(ncell(rng));
  for (auto& c : cells) {
    c.kind = kind(rng);
    const int n = grids[c.kind];
    c.groups = groups(rng);
    c.a_per = n * ys(rng);
    c.b_per = y2[c.kind] * n;
    c.c_per = n * (n / y2[c.kind]);
    c.finish = fin(rng);
  }
  return cells;
}

// P CTAs run the kernel's loop; returns the items run, or -1 on a rule violation.
static long simulate(const std::vector<BatchItem>& items, int nctr, int P, std::mt19937& rng, bool expect_stall) {
  const int n = (int)items.size();
  std::vector<int> ctr(nctr, 0), done(n, 0);
  int ticket = 0;
  struct Cta { int cur, next; bool live; };
  std::vector<Cta> ctas(P);
  for (auto& c : ctas) c = {-1, ticket++, true};
  long ran = 0;
  int live = P;
  while (live > 0) {
    // CTAs that can move: start their next item, or finish the one they wait on
    std::vector<int> movable;
    for (int p = 0; p < P; p++) {
      Cta& c = ctas[p];
      if (!c.live) continue;
      if (c.cur < 0) { movable.push_back(p); continue; }
      const BatchItem& it = items[c.cur];
      if (it.wait < 0 || ctr[it.wait] >= it.target) movable.push_back(p);
    }
    if (movable.empty()) return expect_stall ? ran : -1;
    const int p = movable[std::uniform_int_distribution<int>(0, (int)movable.size() - 1)(rng)];
    Cta& c = ctas[p];
    if (c.cur < 0) {  // take the held ticket, and the following one
      c.cur = c.next;
      if (c.cur >= n) { c.live = false; live--; continue; }
      c.next = ticket++;
      continue;
    }
    const BatchItem& it = items[c.cur];
    // inputs: every item that signals the waited counter has run
    if (it.wait >= 0)
      for (int j = 0; j < n; j++)
        if (items[j].signal == it.wait && !done[j]) return -1;
    done[c.cur] = 1;
    ran++;
    if (it.signal >= 0) ctr[it.signal] += it.count;
    c.cur = -1;
  }
  for (int j = 0; j < n; j++)
    if (!done[j]) return -1;
  return ran;
}

int main() {
  std::mt19937 rng(7);
  int bad = 0, plans = 0;
  long sims = 0;
  for (int trial = 0; trial < 40; trial++) {
    auto cells = random_cells(rng);
    // tiles per item and lag fixed (1-5, 1-3) or chosen by the builder for a launch of
    // 1-600 CTAs
    const int K0 = trial % 3 == 0 ? 0 : 1 + trial % 5, lag0 = trial % 4 == 0 ? 0 : 1 + trial % 3;
    const int ctas = 1 + (int)(rng() % 600);
    std::vector<BatchItem> items;
    int nctr = 0;
    if (build_batch_items(cells, ctas, items, nctr, K0, lag0) != 0) { bad++; continue; }
    int K = 1;
    for (auto& it : items) K = std::max(K, it.count);
    if (K > (K0 > 0 ? K0 : kBatchTilesPerItem)) bad++;
    plans++;
    // every CTA of every pass in exactly one item
    for (int c = 0; c < (int)cells.size(); c++)
      for (int stage = 0; stage < 4; stage++)
        for (int g = 0; g < cells[c].groups; g++) {
          const int per = stage == kStageA ? cells[c].a_per : stage == kStageFinish ? cells[c].finish
                          : stage == kStageB ? cells[c].b_per : cells[c].c_per;
          std::vector<int> seen(per, 0);
          for (auto& it : items) {
            if (it.cell != c || it.stage != stage) continue;
            const int grp = stage == kStageB ? it.by : it.bx;
            if (grp != g) continue;
            if (it.count < 1 || it.count > K) bad++;
            const int first = stage == kStageB ? it.bx : it.by;
            for (int t = 0; t < it.count; t++)
              if (first + t < 0 || first + t >= per) bad++;
              else seen[first + t]++;
          }
          for (int v : seen) if (v != 1) bad++;
        }
    // waiters' targets equal the CTAs that signal; waits point backward
    std::vector<int> signals(nctr, 0), last_signal(nctr, -1);
    for (int i = 0; i < (int)items.size(); i++)
      if (items[i].signal >= 0) {
        if (items[i].signal < 1 || items[i].signal >= nctr) bad++;
        else { signals[items[i].signal] += items[i].count; last_signal[items[i].signal] = i; }
      }
    for (int i = 0; i < (int)items.size(); i++) {
      const BatchItem& it = items[i];
      if (it.kind != cells[it.cell].kind) bad++;
      if (it.wait < 0) continue;
      if (it.target != signals[it.wait]) bad++;
      if (last_signal[it.wait] >= i) bad++;
    }
    for (int P : {1, 2, 7, 64}) {
      const long r = simulate(items, nctr, P, rng, false);
      if (r != (long)items.size()) bad++;
      sims++;
    }
    // one unreachable wait (the test hook): the simulation stalls, with that item and
    // only items queued after it left
    auto stalled = items;
    int k = -1;
    for (int i = 0; i < (int)stalled.size(); i++)
      if (stalled[i].stage == kStageC) { stalled[i].target += 1; k = i; break; }
    const long r = simulate(stalled, nctr, 5, rng, true);
    if (k < 0 || r < 0 || r >= (long)items.size() || r < k) bad++;
  }
  printf("plans=%d simulations=%ld bad=%d\n", plans, sims, bad);
  return bad ? 1 : 0;
}
