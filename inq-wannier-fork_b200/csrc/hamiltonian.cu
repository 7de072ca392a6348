// Kohn-Sham Hamiltonian application and the plain 3-D FFTs on sm_100a: the phase
// kernel of the projector records and the registry of compiled grids.  The tile
// kernels and their launcher are in tiles.cuh / launch_h.cuh; the grids are
// instantiated in groups by grids_*.cu so that they compile in parallel.
//
// H|psi> (src/hamiltonian/ks_hamiltonian.hpp:132-152): k_tile_fwd (z FFT, inner
// y stage, KB projection) -> k_tile_x (outer y stage, x FFT, kinetic, inverse) ->
// k_tile_inv (inverse stages, epilogue with V psi and the nonlocal term).
// to_fourier: k_tile_fwd without projection -> k_tile_x_fft<0>.
// to_real: k_tile_x_fft<1> -> k_tile_inv<MODE_H = 0> with the 1/N.
#include <cuda_runtime.h>

#include <map>
#include <tuple>

#include "dft.cuh"
#include "inqb_internal.h"
#include "plan.h"

namespace inqb {

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
using GridRegistry = std::map<std::tuple<int, int, int, int>, Plan>;
void register_grids_small(GridRegistry& reg);
void register_grids_mid(GridRegistry& reg);
void register_grids_64(GridRegistry& reg);
void register_grids_72(GridRegistry& reg);
void register_grids_96(GridRegistry& reg);
void register_grids_128(GridRegistry& reg);
void register_grids_144(GridRegistry& reg);

static const GridRegistry& registry() {
  static const GridRegistry reg = [] {
    GridRegistry r;
    register_grids_small(r);
    register_grids_mid(r);
    register_grids_64(r);
    register_grids_72(r);
    register_grids_96(r);
    register_grids_128(r);
    register_grids_144(r);
    return r;
  }();
  return reg;
}

const Plan* find_plan(int nx, int ny, int nz, int precision) {
  const auto& reg = registry();
  auto it = reg.find(std::make_tuple(nx, ny, nz, precision == INQB_FP64 ? 0 : 1));
  return it == reg.end() ? nullptr : &it->second;
}

}  // namespace inqb
