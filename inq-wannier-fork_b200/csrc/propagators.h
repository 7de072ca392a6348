// Launchers of the Crank-Nicolson solver kernels (propagators.cu).
#pragma once

namespace inqb {

// acc[4 m ..] = sum_p (|hsd|^2, Re conj(r) hsd, Im conj(r) hsd, |r|^2), FP64, without dV
int launch_sd_sums(int precision, const void* r, const void* hsd, long ld, int M, long N, double* acc, void* stream);
// phi += lambda_m r with the steepest-descent step length from acc (dV applied here);
// normres[m] = dV sum_p |r|^2
int launch_sd_update(int precision, void* phi, long ldp, const void* r, long ldr, int M, long N, const double* acc,
                     double dV, double* normres, void* stream);

}  // namespace inqb
