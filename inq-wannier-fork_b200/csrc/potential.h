// Launchers of the density -> potential kernels (potential.cu).
#pragma once

namespace inqb {

// Number of per-block partial sums the reductions below write (grid size of their
// launches): partial buffers hold kPotBlocks * 4 doubles.
constexpr int kPotBlocks = 592;

// out[p] = (rho[p], 0) in the context precision
int launch_pack_density(int precision, const double* rho, void* out, long N, void* stream);
// V (context precision) = vion + Re vh + v_xc, by theory (0 none, 1 Hartree, 2 LDA);
// vion and vh may be null (zero).  sums[4] (device) = {sum rho vion, sum rho Re vh,
// sum e_xc max(rho, 0), sum rho v_xc} without dV.  partial: kPotBlocks * 4 doubles.
int launch_ks_potential(int precision, const double* rho, const double* vion, const void* vh, int theory, long N,
                        void* V, double* partial, double* sums, void* stream);
// *sum (device) = sum_i |a[i] - b[i]|, without dV.  partial: kPotBlocks doubles.
int launch_absdiff(const double* a, const double* b, long N, double* partial, double* sum, void* stream);
// a1 += c1 y and a2 += c2 y on [N][M] blocks (exponential_2_for_1's accumulators)
int launch_shift2(int precision, const void* y, long ldy, void* a1, long ld1, void* a2, long ld2, int M, long N,
                  const double c1[2], const double c2[2], void* stream);

}  // namespace inqb
