// Launchers of the observable and orbital linear-algebra kernels.
#pragma once

#include <cuda_runtime.h>

namespace inqb {

int launch_density(int precision, const void* psi, long ld, int M, long N, const double* occ, double* rho,
                   void* stream);
// acc[3 m + {0,1,2}] = (Re, Im) sum_p conj(hpsi) psi, sum_p |psi|^2 (FP64)
int launch_band_sums(int precision, const void* psi, const void* hpsi, long ld, int M, long N, double* acc,
                     void* stream);
int launch_dipole(const double* rho, long N, const double lat[3][3], const int nr[3], double* out_dev, void* stream);
int launch_orthonormalize(int precision, void* psi, long ld, int M, long N, double dV, double2* S, double2* X,
                          int* info, void* stream);
// orbital-sharded orthonormalisation: S (Ma x Mb, row stride lds) = dV a^H b; S (M x M)
// <- U^-1 with S = U^H U (X: M x M scratch, info: one int); out = a R (Ma x Mo block)
int launch_overlap_block(int precision, const void* a, long lda, int Ma, const void* b, long ldb, int Mb, long N,
                         double dV, double2* S, long lds, void* stream);
int launch_cholesky_inverse(double2* S, int M, long lds, double2* X, int* info, void* stream);
int launch_rotate_block(int precision, const void* a, long lda, int Ma, const double2* R, long ldr, int Mo,
                        void* out, long ldo, long N, void* stream);
// Largest orbital count of the allocation-free orthonormalisation (fixed device scratch).
constexpr int kOrthoNoAllocMaxStates = 256;
int orthonormalize_noalloc(int precision, int device, void* psi, long ld, int M, long N, double dV, void* stream);

}  // namespace inqb
