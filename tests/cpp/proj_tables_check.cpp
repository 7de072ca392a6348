// Invariants of the projector tables the H kernels index by (host code only; links
// libinqb200 for the table builder and the sphere construction).
#include <cstdio>
#include <vector>
#include <algorithm>
#include "../../inq-wannier-fork_b200/csrc/inqb_internal.h"
namespace inqb {
int build_proj_tables(const inqb_ctx& ctx, int nproj, int L, int smax, const int* counts, const int* coords,
                      const float* relpos, const double* beta, const double* coeff, ProjTables& t);
}
static int check(double a, int n, int reps) {
  double lat[9] = {a, 0, 0, 0, a, 0, 0, 0, a};
  int nr[3] = {n, n, n};
  inqb_ctx ctx;
  ctx.nr[0] = ctx.nr[1] = ctx.nr[2] = n;
  ctx.N = (long)n * n * n;
  ctx.cell.init(lat);
  ctx.dV = ctx.cell.volume / ctx.N;
  const double fr[8][3] = {{0,0,0},{0,.5,.5},{.5,0,.5},{.5,.5,0},{.25,.25,.25},{.25,.75,.75},{.75,.25,.75},{.75,.75,.25}};
  std::vector<std::vector<double>> pos;
  double ac = a / reps;
  for (int i = 0; i < reps; i++) for (int j = 0; j < reps; j++) for (int k = 0; k < reps; k++)
    for (auto& f : fr) pos.push_back({(f[0] + i) * ac, (f[1] + j) * ac, (f[2] + k) * ac});
  int nproj = pos.size();
  std::vector<int> counts(nproj);
  int smax = 0;
  for (int p = 0; p < nproj; p++) {
    inqb_sphere_size(lat, nr, pos[p].data(), 3.0, &counts[p]);
    smax = std::max(smax, counts[p]);
  }
  std::vector<int> coords((size_t)nproj * smax * 3, -1);
  std::vector<float> relpos((size_t)nproj * smax * 3, 0), dist((size_t)nproj * smax, 0);
  for (int p = 0; p < nproj; p++)
    inqb_sphere_points(lat, nr, pos[p].data(), 3.0, counts[p], &coords[(size_t)p * smax * 3], &dist[(size_t)p * smax],
                       &relpos[(size_t)p * smax * 3]);
  const int L = 4;
  std::vector<double> beta((size_t)nproj * L * smax, 1.0), coeff((size_t)nproj * L, 1.0);
  inqb::ProjTables t;
  int st = inqb::build_proj_tables(ctx, nproj, L, smax, counts.data(), coords.data(), relpos.data(), beta.data(),
                                   coeff.data(), t);
  if (st) { printf("build failed %d %s\n", st, inqb_last_error()); return 1; }
  int ntile = n * t.y1, bad = 0;
  if ((int)t.seg_ptr.size() != ntile + 1 || (int)t.seg_ent.size() != t.nseg + 1) bad++;
  long tot = 0;
  for (int tile = 0; tile < ntile; tile++) {
    int e0 = t.seg_ent[t.seg_ptr[tile]], e1 = t.seg_ent[t.seg_ptr[tile + 1]];
    const int* tp = &t.pt_ptr[(size_t)tile * t.pt_stride];
    if (tp[0] != 0 || tp[t.tile_pts] != e1 - e0) bad++;
    std::vector<int> seen(e1 - e0, 0);
    for (int e = e0; e < e1; e++) {
      int q = t.pt_pos[e] - e0;
      if (q < 0 || q >= e1 - e0) { bad++; continue; }
      seen[q]++;
      int off = t.ent_off[e];
      if (off < 0 || off >= t.tile_pts) bad++;
      if (!(q >= tp[off] && q < tp[off + 1])) bad++;
    }
    for (int v : seen) if (v != 1) bad++;
    for (int s = t.seg_ptr[tile]; s < t.seg_ptr[tile + 1]; s++) {
      int ix = tile / t.y1;
      int na = t.plane_ptr[ix + 1] - t.plane_ptr[ix];
      if (t.seg_local[s] < 0 || t.seg_local[s] >= na) bad++;
      if (t.plane_atom[t.plane_ptr[ix] + t.seg_local[s]] != t.seg_atom[s]) bad++;
    }
    tot += e1 - e0;
  }
  if (tot != t.nent) bad++;
  // atom-major order: atom_pos inverts atom_ent; chunks tile every atom's entries
  for (int i = 0; i < t.nent; i++)
    if (t.atom_pos[t.atom_ent[i]] != i) bad++;
  for (int a = 0; a < nproj; a++) {
    int covered = 0;
    for (int c = t.atom_chunk_ptr[a]; c < t.atom_chunk_ptr[a + 1]; c++) {
      if (t.chunk_atom[c] != a) bad++;
      covered += std::min(inqb::kNlChunk, t.atom_ptr[a + 1] - t.chunk_beg[c]);
    }
    if (covered != t.atom_ptr[a + 1] - t.atom_ptr[a]) bad++;
  }
  printf("a=%g n=%d atoms=%d nent=%d nseg=%d max_tile_ent=%d max_tile_seg=%d max_plane_atoms=%d pt_stride=%d bad=%d\n",
         a, n, nproj, t.nent, t.nseg, t.max_tile_ent, t.max_tile_seg, t.max_plane_atoms, t.pt_stride, bad);
  return bad != 0;
}
int main() { return check(10.26, 32, 1) | check(20.52, 64, 2) | check(10.26, 24, 1) | check(10.26, 40, 1); }
