// Host-side setup of libinqb200: cell geometry, atom spheres, KB tables and the
// device layout of the projector data.  This is the one-time work INQ does in
// the projector_all / spherical_grid constructors (per ion configuration); every
// per-apply operation runs in the CUDA kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>

#include "inqb_internal.h"
#include "project.h"
#include "sizes.h"

namespace inqb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}
const char* last_error() { return g_last_error.c_str(); }

// ---------------------------------------------------------------- cell
// Same floating-point operation order as src/systems/cell.hpp:35-53,146-226 so
// that the float-rounded sphere data agree bit for bit with INQ's.
static double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

void CellGeom::init(const double* lattice) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) lat[i][j] = lattice[3 * i + j];
  double c12[3], c20[3], c01[3];
  cross3(lat[1], lat[2], c12);
  cross3(lat[2], lat[0], c20);
  cross3(lat[0], lat[1], c01);
  volume = dot3(lat[0], c12);
  const double f = 2.0 * M_PI / volume;
  for (int c = 0; c < 3; c++) {
    rlat[0][c] = c12[c] * f;
    rlat[1][c] = c20[c] * f;
    rlat[2][c] = c01[c] * f;
  }
}
void CellGeom::contra_to_cart(const double v[3], double o[3]) const {
  for (int c = 0; c < 3; c++) o[c] = lat[0][c] * v[0] + lat[1][c] * v[1] + lat[2][c] * v[2];
}
void CellGeom::cov_to_cart(const double v[3], double o[3]) const {
  for (int c = 0; c < 3; c++) o[c] = (rlat[0][c] * v[0] + rlat[1][c] * v[1] + rlat[2][c] * v[2]) / (2.0 * M_PI);
}
void CellGeom::cart_to_contra(const double v[3], double o[3]) const {
  for (int d = 0; d < 3; d++) o[d] = dot3(rlat[d], v) / (2.0 * M_PI);
}
void CellGeom::cart_to_cov(const double v[3], double o[3]) const {
  for (int d = 0; d < 3; d++) o[d] = dot3(lat[d], v);
}

// ---------------------------------------------------------------- device buffers
int DevBuf::ensure(size_t nbytes) {
  if (nbytes <= bytes && ptr) return INQB_OK;
  release();
  if (nbytes == 0) return INQB_OK;
  cudaError_t e = cudaMalloc(&ptr, nbytes);
  if (e != cudaSuccess) {
    ptr = nullptr;
    bytes = 0;
    return fail(INQB_ERR_NOMEM, std::string("cudaMalloc(") + std::to_string(nbytes) + "): " + cudaGetErrorString(e));
  }
  bytes = nbytes;
  return INQB_OK;
}
void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

// ---------------------------------------------------------------- spheres
// A grid with INQ's symmetric-range coordinates (src/basis/grid.hpp:111-150).
struct GridGeom {
  const CellGeom& cell;
  int nr[3];
  GridGeom(const CellGeom& c, const int n[3]) : cell(c) { std::memcpy(nr, n, sizeof(nr)); }
  int to_sym(int i, int d) const { return (i >= (nr[d] + 1) / 2) ? i - nr[d] : i; }
  int from_sym(int i, int d) const { return (i < 0) ? i + nr[d] : i; }
  void rvector_cart(const int ii[3], double o[3]) const {
    double c[3];
    for (int d = 0; d < 3; d++) c[d] = to_sym(ii[d], d) * (1.0 / nr[d]);
    cell.contra_to_cart(c, o);
  }
};

// Periodic images of an atom within the cell diagonal
// (src/ionic/periodic_replicas.hpp:27-52 with range = diagonal_length()).
static std::vector<std::array<double, 3>> replicas(const CellGeom& cell, const double pos[3]) {
  double c[3], p[3];
  cell.cart_to_contra(pos, c);
  for (int d = 0; d < 3; d++) {
    c[d] -= std::floor(c[d]);
    if (c[d] >= 0.5) c[d] -= 1.0;
  }
  cell.contra_to_cart(c, p);
  double rl[3];
  for (int d = 0; d < 3; d++) rl[d] = std::sqrt(dot3(cell.lat[d], cell.lat[d]));
  const double range = std::sqrt(dot3(rl, rl));
  int nmax[3];
  for (int d = 0; d < 3; d++) nmax[d] = 1 + (int)std::lround(range / std::sqrt(dot3(cell.lat[d], cell.lat[d])));
  std::vector<std::array<double, 3>> out;
  out.push_back({p[0], p[1], p[2]});
  for (int i = -nmax[0]; i <= nmax[0]; i++)
    for (int j = -nmax[1]; j <= nmax[1]; j++)
      for (int k = -nmax[2]; k <= nmax[2]; k++) {
        if (i == 0 && j == 0 && k == 0) continue;
        std::array<double, 3> r;
        for (int c2 = 0; c2 < 3; c2++)
          r[c2] = ((p[c2] + (double)i * cell.lat[0][c2]) + (double)j * cell.lat[1][c2]) + (double)k * cell.lat[2][c2];
        out.push_back(r);
      }
  return out;
}

struct SpherePt {
  int c[3];
  float dist;
  float rel[3];
};

// spherical_grid::initialize (src/basis/spherical_grid.hpp:59-158): for every
// replica, walk its containing cube (src/basis/containing_cube.hpp:20-43) in
// x, y, z order and keep the points within the radius.
static std::vector<SpherePt> sphere(const GridGeom& g, const double center[3], double radius) {
  std::vector<SpherePt> pts;
  for (const auto& re : replicas(g.cell, center)) {
    int lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
      const double* rec = g.cell.rlat[d];
      const double s = radius / std::sqrt(dot3(rec, rec));
      double lop[3], hip[3], cl[3], ch[3];
      for (int c = 0; c < 3; c++) {
        lop[c] = re[c] - s * rec[c];
        hip[c] = re[c] + s * rec[c];
      }
      g.cell.cart_to_contra(lop, cl);
      g.cell.cart_to_contra(hip, ch);
      const double sp = 1.0 / g.nr[d];
      lo[d] = (int)std::lround(std::floor(cl[d] / sp));
      hi[d] = (int)std::lround(std::ceil(ch[d] / sp)) + 1;
      const int b = -g.nr[d] / 2, e = g.nr[d] / 2 + g.nr[d] % 2;
      lo[d] = std::min(std::max(lo[d], b), e);
      hi[d] = std::min(std::max(hi[d], b), e);
    }
    for (int i = lo[0]; i < hi[0]; i++)
      for (int j = lo[1]; j < hi[1]; j++)
        for (int k = lo[2]; k < hi[2]; k++) {
          const int ii[3] = {g.from_sym(i, 0), g.from_sym(j, 1), g.from_sym(k, 2)};
          double r[3], dr[3];
          g.rvector_cart(ii, r);
          for (int c = 0; c < 3; c++) dr[c] = r[c] - re[c];
          const double n2 = dot3(dr, dr);
          if (n2 > radius * radius) continue;
          SpherePt sp;
          std::memcpy(sp.c, ii, sizeof(ii));
          sp.dist = (float)std::sqrt(n2);
          double cc[3];
          g.cell.cart_to_contra(dr, cc);
          for (int c = 0; c < 3; c++) sp.rel[c] = (float)cc[c];
          pts.push_back(sp);
        }
  }
  return pts;
}

// ---------------------------------------------------------------- twiddles
// tw[k1 * N2 + j2] = exp(-2 pi i j2 k1 / N) for the four-step split N = N1 N2,
// evaluated in extended precision and rounded once.
void twiddle_table(int n, int n1, int n2, std::vector<double>& re, std::vector<double>& im) {
  re.assign(n, 0.0);
  im.assign(n, 0.0);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k1 = 0; k1 < n1; k1++)
    for (int j2 = 0; j2 < n2; j2++) {
      const long t = ((long)j2 * k1) % n;
      const long double a = -2.0L * pi * (long double)t / (long double)n;
      re[k1 * n2 + j2] = (double)cosl(a);
      im[k1 * n2 + j2] = (double)sinl(a);
    }
}

int split_of(int n, int* n1, int* n2) {
#define INQB_ROW(N, A, B) {N, A, B},
  static const int table[][3] = {INQB_FFT_SIZES(INQB_ROW)};
#undef INQB_ROW
  for (const auto& r : table)
    if (r[0] == n) {
      *n1 = r[1];
      *n2 = r[2];
      return INQB_OK;
    }
  return INQB_ERR_UNSUPPORTED;
}

// ---------------------------------------------------------------- projector tables
int build_proj_tables(const inqb_ctx& ctx, int nproj, int L, int smax, const int* counts, const int* coords,
                      const float* relpos, const double* beta, const double* coeff, ProjTables& t) {
  const int nx = ctx.nr[0], ny = ctx.nr[1], nz = ctx.nr[2];
  t.nproj = nproj;
  t.L = L;
  // The H kernels tile plane ix into Y1 row classes: tile (ix, y1) holds the rows
  // y = y1 + Y1 * r, r = 0..NY/Y1-1, where NY = Y2 * Y1 is the four-step split of
  // the y axis.  Entries are bucketed by tile, keeping (atom, point) order inside.
  int y2n = 0, y1n = 0;
  if (split_of(ny, &y2n, &y1n) != INQB_OK) return fail(INQB_ERR_UNSUPPORTED, "unsupported y grid size");
  const int ntile = nx * y1n;
  std::vector<std::vector<std::pair<int, int>>> by_tile(ntile);
  long total = 0;
  for (int a = 0; a < nproj; a++) {
    if (counts[a] < 0 || counts[a] > smax) return fail(INQB_ERR_INVALID, "sphere count out of range");
    for (int p = 0; p < counts[a]; p++) {
      const int* c = coords + ((long)a * smax + p) * 3;
      if (c[0] < 0 || c[0] >= nx || c[1] < 0 || c[1] >= ny || c[2] < 0 || c[2] >= nz)
        return fail(INQB_ERR_INVALID, "sphere point outside the grid");
      by_tile[c[0] * y1n + c[1] % y1n].push_back({a, p});
      total++;
    }
  }
  if (total > 0x7fffffff) return fail(INQB_ERR_UNSUPPORTED, "too many sphere points");
  t.nent = (int)total;
  t.y1 = y1n;
  t.seg_ptr.assign(ntile + 1, 0);
  t.seg_atom.clear();
  t.seg_ent.clear();
  t.seg_local.clear();
  t.plane_ptr.assign(nx + 1, 0);
  t.plane_atom.clear();
  t.ent_off.resize(total);
  t.ent_atom.resize(total);
  t.ent_beta.resize(total * L);
  t.ent_relpos.resize(total * 3);
  t.max_plane_atoms = 0;
  std::vector<int> local_of(nproj, -1);
  int e = 0;
  for (int ix = 0; ix < nx; ix++) {
    // atoms of plane ix in increasing order: the plane-local accumulator index
    t.plane_ptr[ix] = (int)t.plane_atom.size();
    std::vector<char> in_plane(nproj, 0);
    for (int y1 = 0; y1 < y1n; y1++)
      for (auto [a, p] : by_tile[ix * y1n + y1]) in_plane[a] = 1;
    for (int a = 0; a < nproj; a++)
      if (in_plane[a]) {
        local_of[a] = (int)t.plane_atom.size() - t.plane_ptr[ix];
        t.plane_atom.push_back(a);
      }
    t.max_plane_atoms = std::max(t.max_plane_atoms, (int)t.plane_atom.size() - t.plane_ptr[ix]);
    for (int y1 = 0; y1 < y1n; y1++) {
      const int tile = ix * y1n + y1;
      t.seg_ptr[tile] = (int)t.seg_atom.size();
      int cur = -1;
      for (auto [a, p] : by_tile[tile]) {
        if (a != cur) {
          t.seg_atom.push_back(a);
          t.seg_ent.push_back(e);
          t.seg_local.push_back(local_of[a]);
          cur = a;
        }
        const int* c = coords + ((long)a * smax + p) * 3;
        t.ent_off[e] = (c[1] / y1n) * nz + c[2];  // tile-local row, z
        t.ent_atom[e] = a;
        for (int l = 0; l < L; l++) t.ent_beta[(long)e * L + l] = beta[((long)a * L + l) * smax + p];
        for (int d = 0; d < 3; d++) t.ent_relpos[(long)e * 3 + d] = relpos[((long)a * smax + p) * 3 + d];
        e++;
      }
    }
  }
  t.seg_ptr[ntile] = (int)t.seg_atom.size();
  t.plane_ptr[nx] = (int)t.plane_atom.size();
  t.seg_ent.push_back(e);
  t.nseg = (int)t.seg_atom.size();
  t.max_tile_ent = 0;
  t.max_tile_seg = 0;
  for (int tile = 0; tile < ntile; tile++) {
    t.max_tile_ent = std::max(t.max_tile_ent, (int)by_tile[tile].size());
    t.max_tile_seg = std::max(t.max_tile_seg, t.seg_ptr[tile + 1] - t.seg_ptr[tile]);
  }
  // point order inside each tile: stable sort of the tile's entries by offset
  t.tile_pts = y2n * nz;
  t.pt_stride = (t.tile_pts + 1 + 3) / 4 * 4;
  t.pt_pos.assign(total, 0);
  t.pt_ptr.assign((size_t)ntile * t.pt_stride, 0);
  for (int tile = 0; tile < ntile; tile++) {
    const int e0 = t.seg_ent[t.seg_ptr[tile]], e1 = t.seg_ent[t.seg_ptr[tile + 1]];
    int* tp = &t.pt_ptr[(size_t)tile * t.pt_stride];
    for (int e = e0; e < e1; e++) tp[t.ent_off[e] + 1]++;
    for (int q = 0; q < t.tile_pts; q++) tp[q + 1] += tp[q];
    std::vector<int> fill(tp, tp + t.tile_pts);
    for (int e = e0; e < e1; e++) t.pt_pos[e] = e0 + fill[t.ent_off[e]]++;
  }
  // grid point of every entry, in entry order
  std::vector<long> pt_of(total);
  {
    int ee = 0;
    for (int tile = 0; tile < ntile; tile++)
      for (auto [a, p] : by_tile[tile]) {
        const int* c = coords + ((long)a * smax + p) * 3;
        pt_of[ee++] = ((long)c[0] * ny + c[1]) * nz + c[2];
      }
  }
  // atom-major entry lists, grid points and cartesian relative positions
  t.ent_pt.resize(total);
  t.ent_xyz.resize(total * 3);
  for (long i = 0; i < total; i++) {
    t.ent_pt[i] = (int)pt_of[i];
    const double rc[3] = {(double)t.ent_relpos[3 * i], (double)t.ent_relpos[3 * i + 1],
                          (double)t.ent_relpos[3 * i + 2]};
    ctx.cell.contra_to_cart(rc, &t.ent_xyz[3 * i]);
  }
  t.atom_ptr.assign(nproj + 1, 0);
  for (long i = 0; i < total; i++) t.atom_ptr[t.ent_atom[i] + 1]++;
  for (int a = 0; a < nproj; a++) t.atom_ptr[a + 1] += t.atom_ptr[a];
  t.atom_ent.assign(total, 0);
  {
    std::vector<int> fill(t.atom_ptr.begin(), t.atom_ptr.end() - 1);
    for (long i = 0; i < total; i++) t.atom_ent[fill[t.ent_atom[i]]++] = (int)i;
  }
  t.atom_pos.assign(total, 0);
  for (long i = 0; i < total; i++) t.atom_pos[t.atom_ent[i]] = (int)i;
  t.chunk_atom.clear();
  t.chunk_beg.clear();
  t.atom_chunk_ptr.assign(nproj + 1, 0);
  for (int a = 0; a < nproj; a++) {
    t.atom_chunk_ptr[a] = (int)t.chunk_atom.size();
    for (int i = t.atom_ptr[a]; i < t.atom_ptr[a + 1]; i += kNlChunk) {
      t.chunk_atom.push_back(a);
      t.chunk_beg.push_back(i);
    }
  }
  t.atom_chunk_ptr[nproj] = (int)t.chunk_atom.size();
  // chunks of the projection kernels, in atom-major entry order
  t.pc_ptr.assign(nproj + 1, 0);
  for (int a = 0; a < nproj; a++)
    t.pc_ptr[a + 1] = t.pc_ptr[a] + (t.atom_ptr[a + 1] - t.atom_ptr[a] + kProjChunk - 1) / kProjChunk;
  t.pc_chunks = t.pc_ptr[nproj];
  const size_t pcn = (size_t)t.pc_chunks * kProjChunk;
  t.pc_pt.assign(pcn, -1);
  t.pc_beta.assign(pcn * 4, 0.0);
  t.pc_relpos.assign(pcn * 3, 0.0f);
  for (int a = 0; a < nproj; a++)
    for (int i = t.atom_ptr[a]; i < t.atom_ptr[a + 1]; i++) {
      const size_t q = (size_t)t.pc_ptr[a] * kProjChunk + (i - t.atom_ptr[a]);
      const int ee = t.atom_ent[i];
      t.pc_pt[q] = t.ent_pt[ee];
      for (int l = 0; l < L && l < 4; l++) t.pc_beta[4 * q + l] = t.ent_beta[(size_t)ee * L + l];
      for (int d = 0; d < 3; d++) t.pc_relpos[3 * q + d] = t.ent_relpos[3 * (size_t)ee + d];
    }
  // each atom's slots of the fused projection's partial sums, in plane order
  {
    std::vector<std::vector<int>> lists(nproj);
    for (int ix = 0; ix < nx; ix++)
      for (int q = t.plane_ptr[ix]; q < t.plane_ptr[ix + 1]; q++) lists[t.plane_atom[q]].push_back(q);
    t.aslot_ptr.assign(nproj + 1, 0);
    t.aslot.clear();
    for (int a = 0; a < nproj; a++) {
      t.aslot.insert(t.aslot.end(), lists[a].begin(), lists[a].end());
      t.aslot_ptr[a + 1] = (int)t.aslot.size();
    }
  }
  t.scale.resize((size_t)nproj * L);
  for (int a = 0; a < nproj; a++)
    for (int l = 0; l < L; l++) t.scale[(size_t)a * L + l] = ctx.dV * coeff[(size_t)a * L + l];
  return INQB_OK;
}

template <typename T>
static int upload(DevBuf& b, const std::vector<T>& v) {
  INQB_TRY(b.ensure(std::max<size_t>(sizeof(T) * v.size(), 16)));
  if (!v.empty()) INQB_CUDA_TRY(cudaMemcpy(b.ptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  return INQB_OK;
}

// Entry records with zero phases (the phase kernel fills them for each k + A).
// point_order: record e goes to pt_pos[e] instead of e.
template <typename T>
static std::vector<EntRec<T>> ent_records(const ProjTables& t, bool point_order = false) {
  std::vector<EntRec<T>> rec((size_t)t.nent);
  for (int tile = 0; tile + 1 < (int)t.seg_ptr.size(); tile++)
    for (int s = t.seg_ptr[tile]; s < t.seg_ptr[tile + 1]; s++)
      for (int e = t.seg_ent[s]; e < t.seg_ent[s + 1]; e++) {
        EntRec<T>& r = rec[point_order ? t.pt_pos[e] : e];
        r.ph[0] = r.ph[1] = (T)0;
        for (int l = 0; l < 4; l++) r.beta[l] = (l < t.L) ? (T)t.ent_beta[(size_t)e * t.L + l] : (T)0;
        r.off = t.ent_off[e];
        r.tseg = s - t.seg_ptr[tile];
      }
  return rec;
}

// Atom-major adjoint records with zero phases (the phase kernel fills them).
template <typename T>
static std::vector<AdjRec<T>> adj_records(const ProjTables& t) {
  std::vector<AdjRec<T>> rec((size_t)t.nent);
  for (int i = 0; i < t.nent; i++) {
    const int e = t.atom_ent[i];
    AdjRec<T>& r = rec[i];
    r.ph[0] = r.ph[1] = (T)0;
    for (int l = 0; l < 4; l++) r.beta[l] = (l < t.L) ? (T)t.ent_beta[(size_t)e * t.L + l] : (T)0;
    for (int d = 0; d < 3; d++) r.xyz[d] = t.ent_xyz[3 * (size_t)e + d];
    r.pt = t.ent_pt[e];
  }
  return rec;
}

int upload_proj_tables(const inqb_ctx& ctx, ProjTables& t) {
  INQB_TRY(upload(t.d_seg_ptr, t.seg_ptr));
  INQB_TRY(upload(t.d_seg_atom, t.seg_atom));
  INQB_TRY(upload(t.d_seg_ent, t.seg_ent));
  INQB_TRY(upload(t.d_ent_off, t.ent_off));
  INQB_TRY(upload(t.d_ent_atom, t.ent_atom));
  INQB_TRY(upload(t.d_seg_local, t.seg_local));
  INQB_TRY(upload(t.d_plane_ptr, t.plane_ptr));
  INQB_TRY(upload(t.d_plane_atom, t.plane_atom));
  INQB_TRY(upload(t.d_ent_relpos, t.ent_relpos));
  INQB_TRY(upload(t.d_scale, t.scale));
  INQB_TRY(upload(t.d_atom_ptr, t.atom_ptr));
  INQB_TRY(upload(t.d_atom_ent, t.atom_ent));
  INQB_TRY(upload(t.d_ent_pt, t.ent_pt));
  INQB_TRY(upload(t.d_ent_xyz, t.ent_xyz));
  INQB_TRY(upload(t.d_chunk_atom, t.chunk_atom));
  INQB_TRY(upload(t.d_chunk_beg, t.chunk_beg));
  INQB_TRY(upload(t.d_atom_chunk_ptr, t.atom_chunk_ptr));
  if (ctx.precision == INQB_FP64) {
    INQB_TRY(upload(t.d_ent_beta, t.ent_beta));
  } else {
    std::vector<float> bf(t.ent_beta.begin(), t.ent_beta.end());
    INQB_TRY(upload(t.d_ent_beta, bf));
  }
  INQB_TRY(t.d_ent_phase.ensure(std::max<size_t>((size_t)t.nent * ctx.elem_bytes(), 16)));
  if (ctx.precision == INQB_FP64) {
    INQB_TRY(upload(t.d_ent_rec, ent_records<double>(t)));
    INQB_TRY(upload(t.d_ent_rec_pt, ent_records<double>(t, true)));
  } else {
    INQB_TRY(upload(t.d_ent_rec, ent_records<float>(t)));
    INQB_TRY(upload(t.d_ent_rec_pt, ent_records<float>(t, true)));
  }
  INQB_TRY(upload(t.d_pt_pos, t.pt_pos));
  INQB_TRY(upload(t.d_atom_pos, t.atom_pos));
  if (ctx.precision == INQB_FP64) {
    INQB_TRY(upload(t.d_adj_rec, adj_records<double>(t)));
  } else {
    INQB_TRY(upload(t.d_adj_rec, adj_records<float>(t)));
  }
  INQB_TRY(upload(t.d_pt_ptr, t.pt_ptr));
  INQB_TRY(upload(t.d_aslot_ptr, t.aslot_ptr));
  INQB_TRY(upload(t.d_aslot, t.aslot));
  INQB_TRY(upload(t.d_pc_ptr, t.pc_ptr));
  INQB_TRY(upload(t.d_pc_pt, t.pc_pt));
  INQB_TRY(upload(t.d_pc_beta, t.pc_beta));
  INQB_TRY(upload(t.d_pc_relpos, t.pc_relpos));
  INQB_TRY(t.d_pc_table.ensure(std::max<size_t>(project_table_bytes(ctx.precision, t.pc_chunks), 16)));
  return INQB_OK;
}

// ---------------------------------------------------------------- C ABI helpers (setup)
int sphere_points(const CellGeom& cell, const int nr[3], const double center[3], double radius, int npts, int* coords,
                  float* dist, float* relpos, int* count_out) {
  GridGeom g(cell, nr);
  auto pts = sphere(g, center, radius);
  if (count_out) *count_out = (int)pts.size();
  if (coords) {
    if (npts != (int)pts.size()) return fail(INQB_ERR_INVALID, "npts does not match the sphere size");
    for (size_t i = 0; i < pts.size(); i++) {
      for (int d = 0; d < 3; d++) {
        coords[3 * i + d] = pts[i].c[d];
        relpos[3 * i + d] = pts[i].rel[d];
      }
      dist[i] = pts[i].dist;
    }
  }
  return INQB_OK;
}

// Real spherical harmonics l = 0, 1 in the (y, z, x) order of m = -1, 0, 1.
static double ylm(int l, int m, const double r[3]) {
  if (l == 0) return 0.5 / std::sqrt(M_PI);
  const double rr = std::sqrt(dot3(r, r));
  if (rr == 0.0) return 0.0;
  const double c = std::sqrt(3.0 / (4.0 * M_PI));
  return c * (m == -1 ? r[1] : m == 0 ? r[2] : r[0]) / rr;
}

int gaussian_kb_beta(const CellGeom& cell, int npts, const float* dist, const float* relpos, double sigma,
                     double* beta) {
  if (sigma <= 0.0) return fail(INQB_ERR_INVALID, "sigma must be positive");
  for (int p = 0; p < npts; p++) {
    const double r = (double)dist[p];
    const double rc[3] = {(double)relpos[3 * p], (double)relpos[3 * p + 1], (double)relpos[3 * p + 2]};
    double cart[3];
    cell.contra_to_cart(rc, cart);
    const double gauss = std::exp(-r * r / (2.0 * sigma * sigma));
    beta[p] = gauss * ylm(0, 0, cart);
    for (int m = -1; m <= 1; m++) beta[(size_t)(m + 2) * npts + p] = r * gauss * ylm(1, m, cart);
  }
  return INQB_OK;
}

}  // namespace inqb
