// Internal state of libinqb200: the context that backs the C ABI in
// include/inqb200.h.  Host-only declarations plus the POD views that kernels get.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/inqb200.h"

namespace inqb {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);

#define INQB_CUDA_TRY(expr)                                                            \
  do {                                                                                 \
    cudaError_t err_ = (expr);                                                         \
    if (err_ != cudaSuccess)                                                           \
      return ::inqb::fail(INQB_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(err_)); \
  } while (0)

#define INQB_TRY(expr)        \
  do {                        \
    int st_ = (expr);         \
    if (st_ != INQB_OK) return st_; \
  } while (0)

// ---------------------------------------------------------------- cell
struct CellGeom {
  double lat[3][3];   // lat[i] = lattice vector a_i (cartesian, bohr)
  double rlat[3][3];  // reciprocal vectors b_i with a_i . b_j = 2 pi delta_ij
  double volume;
  void init(const double* lattice);
  void contra_to_cart(const double c[3], double out[3]) const;
  void cov_to_cart(const double c[3], double out[3]) const;
  void cart_to_contra(const double v[3], double out[3]) const;
  void cart_to_cov(const double v[3], double out[3]) const;
};

// ---------------------------------------------------------------- device buffer
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      bytes = o.bytes;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  int ensure(size_t nbytes);  // grows, never shrinks; contents not preserved
  void release();
  ~DevBuf() { release(); }
  template <typename P>
  P* as() const { return reinterpret_cast<P*>(ptr); }
};

// One sphere entry as the H tiles read it: exp(+i (k+A).r), the KB radial values
// (zero past L) and the tile-local offset (row * NZ + z), padded to whole
// 16-byte vectors so a tile's run of entries is copied with cp.async.
template <typename T>
struct alignas(16) EntRec {
  T ph[2];
  T beta[4];
  int off;
  int tseg;  // segment index within the tile (its atom's slot in the tile's projections)
};

// One sphere entry in atom-major order for the adjoint's nonlocal moments: phase,
// radial values, cartesian position relative to the atom and linear grid point.
template <typename T>
struct alignas(16) AdjRec {
  T ph[2];
  T beta[4];
  double xyz[3];
  int pt;
};

// Projector tables in the layout the fused H kernels read (built on the host
// from projector_all-style per-atom sphere tables, then uploaded).
struct ProjTables {
  int nproj = 0, L = 0;
  int nent = 0, nseg = 0;
  int y1 = 1;               // row classes per x-plane (tiles per plane)
  int max_plane_atoms = 0;  // most atoms whose spheres cut one x-plane
  int max_tile_ent = 0;     // most sphere entries in one tile
  int max_tile_seg = 0;     // most atom segments in one tile
  int tile_pts = 0;         // grid points of a tile (NY / Y1 rows x NZ)
  int pt_stride = 0;        // tile stride of pt_ptr: tile_pts + 1 rounded up to 4
  // host copies.  Tile (ix, y1) holds rows y = y1 + Y1 * r of plane ix; seg_ptr
  // [NX * Y1 + 1] lists its atom segments (seg_atom, seg_ent range, seg_local =
  // the atom's index among the atoms of plane ix, plane_ptr / plane_atom).
  std::vector<int> seg_ptr, seg_atom, seg_ent, seg_local, plane_ptr, plane_atom, ent_off, ent_atom;
  std::vector<double> ent_beta;     // [nent][L]
  std::vector<float> ent_relpos;    // [nent][3] contravariant, float as the reference stores it
  std::vector<double> scale;        // [nproj][L] = dV * kb coefficient
  // atom-major view used by the derivative kernels of the adjoint
  std::vector<int> atom_ptr, atom_ent, ent_pt;  // [nproj+1], [nent], [nent] linear grid point
  std::vector<double> ent_xyz;      // [nent][3] cartesian relative position
  // chunks of at most kNlChunk consecutive entries of one atom (atom-major order),
  // the unit of work of the nonlocal moment kernel of the adjoint
  std::vector<int> chunk_atom, chunk_beg, atom_chunk_ptr;
  std::vector<int> atom_pos;        // [nent] position of entry e in atom-major order
  // per-atom chunks of kProjChunk entries (atom-major, the last chunk of an atom padded)
  // for the projection kernels: pc_ptr [nproj+1] chunk offsets, pc_pt [chunks * 32]
  // linear grid point (-1 = padding), pc_beta [chunks * 32][4] (zero past L and for
  // padding), pc_relpos [chunks * 32][3] contravariant float relative position
  int pc_chunks = 0;
  std::vector<int> pc_ptr, pc_pt;
  std::vector<double> pc_beta;
  std::vector<float> pc_relpos;
  DevBuf d_pc_ptr, d_pc_pt, d_pc_beta, d_pc_relpos;
  DevBuf d_pc_table;                // coefficient table beta exp(+i (k+A).r) for the current k + A
  // each atom's (plane, atom) slots of the fused projection, in plane order
  std::vector<int> aslot_ptr, aslot;
  DevBuf d_aslot_ptr, d_aslot;
  DevBuf d_adj_rec, d_atom_pos;     // [nent] AdjRec<T> in atom-major order
  // device copies
  DevBuf d_seg_ptr, d_seg_atom, d_seg_ent, d_seg_local, d_plane_ptr, d_plane_atom, d_ent_off, d_ent_atom;
  DevBuf d_ent_beta;                // [nent][L] in the context precision
  DevBuf d_ent_relpos;              // [nent][3] float
  DevBuf d_ent_phase;               // [nent] complex, exp(+i (k+A).r), context precision
  DevBuf d_ent_rec;                 // [nent] EntRec<T>, phases filled with d_ent_phase
  // the same records in point order inside each tile (for the owner-computes
  // nonlocal scatter): rec_pt[pt_pos[e]] is entry e; pt_ptr[tile * pt_stride + q]
  // is the first record of tile-local point q relative to the tile's first entry
  std::vector<int> pt_pos, pt_ptr;
  DevBuf d_ent_rec_pt, d_pt_pos, d_pt_ptr;
  DevBuf d_scale;                   // [nproj][L] double
  DevBuf d_atom_ptr, d_atom_ent, d_ent_pt, d_ent_xyz;
  DevBuf d_chunk_atom, d_chunk_beg, d_atom_chunk_ptr;
};

// Kernel view of the projector tables (T = float or double).
template <typename T>
struct ProjView {
  int nproj, L, max_plane_atoms, max_tile_ent, max_tile_seg, pt_stride;
  const int* seg_ptr;     // [NX * Y1 + 1] segments of tile (ix, y1)
  const int* seg_atom;
  const int* seg_ent;     // [nseg + 1] entry ranges
  const int* seg_local;   // plane-local atom index of a segment
  const int* plane_ptr;   // [NX + 1] atoms of plane ix
  const int* plane_atom;
  const int* ent_off;     // tile-local (row * NZ + z)
  const int* ent_atom;
  const T* ent_beta;
  const void* ent_phase;  // cplx<T>*
  const EntRec<T>* ent_rec;     // segment (atom) order
  const EntRec<T>* ent_rec_pt;  // point order inside each tile
  const int* pt_ptr;            // [tiles][pt_stride]
  const double* scale;
  double2* proj;          // [nproj][L][M] accumulators (FP64 in both precisions)
  // the projection kernels' chunk tables (project.h)
  const int* pc_ptr;
  const int* pc_pt;
  const void* pc_table;
  int* err;               // device error word (a device-side wait gave up)
  int proj_mode;          // 0: fused into the first tile pass; 1: projection kernel
  // the fused projection's partial sums: slot (plane_ptr[ix] + local atom) * ysplit + half
  // holds [LMAX][M]; aslot_ptr / aslot list each atom's slots in plane order
  double2* slots;         // null: flush with atomics instead
  const int* aslot_ptr;
  const int* aslot;
};

constexpr int kNlChunk = 64;  // sphere entries per chunk of the adjoint's nonlocal moments

struct Plan;  // kernel launch plan for one (precision, grid) pair

}  // namespace inqb

struct inqb_ctx {
  int device = 0;
  int precision = INQB_FP64;
  int nr[3] = {0, 0, 0};
  long N = 0;
  inqb::CellGeom cell;
  double dV = 0.0;
  double kA_cov[3] = {0, 0, 0};
  const inqb::Plan* plan = nullptr;
  bool proj_phases_valid = false;  // device phases match kA_cov
  int fourier_mask = 0;            // zero_outside_sphere on the kinetic term

  std::vector<double> V_host;
  // the projector inputs as set (inqb_ctx_clone rebuilds the tables from them)
  struct ProjSource {
    int nproj = 0, L = 0, smax = 0;
    std::vector<int> counts, coords;
    std::vector<float> relpos;
    std::vector<double> beta, coeff;
  } proj_src;
  inqb::DevBuf d_V;       // [N] in context precision
  inqb::DevBuf d_tw;      // twiddles for x, y, z (context precision), N_d entries each
  inqb::ProjTables proj;

  // workspace (grown on demand)
  inqb::DevBuf d_tmp;     // Fourier-space intermediate, [groups][N][G]
  inqb::DevBuf d_projacc; // projection accumulators
  inqb::DevBuf d_work;    // one orbital block for propagators
  inqb::DevBuf d_work2;
  inqb::DevBuf d_red;     // small reduction buffers
  inqb::DevBuf d_band;    // band-energy sums, 3 doubles per orbital
  inqb::DevBuf d_adjU, d_adjW;  // Fourier transforms for the dH/dA inner products
  inqb::DevBuf d_nlpart;        // per-chunk nonlocal moments of the dH/dA inner products
  inqb::DevBuf d_adjL;          // adjoint step: H^j lambda (4 blocks), Xi, spare
  inqb::DevBuf d_cn;            // Crank-Nicolson: rhs, residual, (1 + i dt/2 H) residual
  inqb::DevBuf d_cnred;         // Crank-Nicolson: 4 sums and the residual norm per orbital
  inqb::DevBuf d_scf;           // ETRS with self-consistency: the saved half step, H^k phi
  inqb_density_reduce_fn density_reduce = nullptr;  // cross-rank density sum (orbital sharding)
  void* density_reduce_user = nullptr;
  inqb::DevBuf d_io;            // checkpoint staging (complex128 rows of a chunk of states)
  inqb::DevBuf d_mlwf;          // TD-MLWF: the six matrices, u, adiag, sums, slabs, pairs, deltas
  inqb::DevBuf d_pot;           // density -> potential: V_H field [N] (complex), previous
                                // density [N], partial sums, sums
  inqb::DevBuf d_err;           // one int: set by a kernel whose bounded device-side wait gave up
  int proj_mode = 0;            // INQB_PROJECTION_FUSED (0) or INQB_PROJECTION_KERNEL (1)
  inqb::DevBuf d_slots;         // the fused projection's per-(plane, half) partial sums
  inqb::DevBuf d_mix;           // Crank-Nicolson with self-consistency: Broyden ring df, dv [4][N],
                                // f_old, vin_old, the new density [N], partial sums, dot products
  size_t elem_bytes() const { return precision == INQB_FP64 ? 16 : 8; }

  // launch schedules per orbital count (ysplit, threads of the three passes), set
  // by inqb_autotune or inqb_set_schedule; absent counts use the compiled default
  std::map<int, std::array<int, 4>> schedules;

  // host-buffer applies: copy-in, compute and copy-out streams and chunk events
  cudaStream_t host_streams[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t host_events[8] = {};

  // optional per-pass CUDA-event timing of H applications
  std::vector<cudaEvent_t> timing_events;  // 5 per recorded application
  int timing_capacity = 0, timing_count = 0;
  bool timing_on = false;
};
