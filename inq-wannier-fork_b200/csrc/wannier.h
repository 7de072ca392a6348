// Launchers of the TD-MLWF kernels (wannier.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace inqb {

// Bytes of the Gram kernel's per-slab partial sums and their FP64 sum, for M states or
// an Ma x Mb block (either precision).
size_t mlwf_partial_bytes(long N, int M);
size_t mlwf_partial_bytes(long N, int Ma, int Mb);
// Z [3][Ma][Mb] (device, complex128) = sum_p conj(a_m) e^{i theta_d} b_n: one block of the
// three weighted Gram matrices (orbital-sharded TD-MLWF); partial: mlwf_partial_bytes(N, Ma, Mb)
int launch_mlwf_gram_block(int precision, const void* pa, long lda, int Ma, const void* pb, long ldb, int Mb, long N,
                           const int nr[3], const double lat[3][3], void* partial, double2* Z, void* stream);
// a [6][M][M] from Z [3][M][M] and norms[ns m + ns - 1] = sum_p |psi_m|^2
int launch_mlwf_finish(const double2* Z, int M, const double* norms, int norm_stride, double2* a, void* stream);
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
