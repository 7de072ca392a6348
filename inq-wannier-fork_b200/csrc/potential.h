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


// ---- Broyden density mixer (src/mixers/broyden.hpp:26-160) on FP64 device vectors of
// n values.  The ring bookkeeping and the small solve are on the host
// (broyden_host.h).
constexpr int kMaxDots = 16;    // dot products per launch_dots call
constexpr int kMaxBroyden = 8;  // ring slots the update kernel takes
struct DotList {
  const double* a[kMaxDots];
  const double* b[kMaxDots];
};
struct BroydenCoef {
  double c[kMaxBroyden];
};
// f_old = vout - vin and vin_old = vin; when df and dv are not null, first
// df = (vout - vin) - f_old and dv = vin - vin_old.
int launch_broyden_diff(const double* vin, const double* vout, double* f_old, double* vin_old, double* df,
                        double* dv, long n, void* stream);
// out[k] (device) = sum_i a_k[i] b_k[i] for k < nd <= kMaxDots, each in a fixed order.
// partial: kPotBlocks * kMaxDots doubles.
int launch_dots(const DotList& d, int nd, long n, double* partial, double* out, void* stream);
// x *= s and y *= s
int launch_scale2(double* x, double* y, double s, long n, void* stream);
// vin += mix ff - sum_{k < used} c_k (mix df_k + dv_k), df and dv [used][n]; *sum (device)
// = the sum of the new vin.  partial: kPotBlocks doubles.
int launch_broyden_update(double* vin, const double* ff, const double* df, const double* dv, long n, int used,
                          const BroydenCoef& c, double mix, double* partial, double* sum, void* stream);
// x *= s
int launch_scale(double* x, double s, long n, void* stream);

}  // namespace inqb
