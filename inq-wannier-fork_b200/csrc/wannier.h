// Launchers of the TD-MLWF kernels (wannier.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace inqb {

// Bytes of the Gram kernel's per-slab partial sums for M states (either precision).
size_t mlwf_partial_bytes(long N, int M);
// a [6][M][M] complex128: the six matrices of tdmlwf_trans::update from psi; sums[3 m + 2]
// = sum_p |psi_m|^2 (band sums); partial: mlwf_partial_bytes.
int launch_mlwf_gram(int precision, const void* psi, long ld, int M, long N, const int nr[3], const double lat[3][3],
                     const double* sums, void* partial, double2* a, void* stream);
int launch_identity(double2* u, int M, void* stream);
// one JADE rotation step over np pairs (int2 top, bottom; indices >= M are skipped);
// delta[np] receives each pair's change of sum_k trace(a_k)
int launch_jade_step(double2* a, double2* u, int M, const int2* pairs, int np, double* delta, void* stream);
int launch_jade_change(const double* delta, int nsteps, int np, double* out, void* stream);
int launch_jade_adiag(const double2* a, const double2* u, int M, double2* adiag, void* stream);
// out = psi u^H (out must not alias psi)
int launch_mlwf_rotate(int precision, const void* psi, long ld, int M, long N, const double2* u, void* out, long ldo,
                       void* stream);

}  // namespace inqb
