// Launchers of the adjoint building blocks (adjoint.cu).
#pragma once

struct inqb_ctx;

namespace inqb {

int launch_axpby(int precision, long N, int M, const double a[2], const void* x, long ldx, const double b[2], void* y,
                 long ldy, void* stream);
// y = sum_k a_k x_k, 1 <= K <= 5 blocks; y may alias an x_k with the same leading dimension
int launch_lincomb(int precision, long N, int M, int K, const double (*a)[2], const void* const* x, const long* ldx,
                   void* y, long ldy, void* stream);
int launch_position_scale(int precision, const inqb_ctx& ctx, const void* psi, long ld, void* out, long ldo, int M,
                          int dir, const double* occ, double s, void* stream);
// psi *= exp(-i kick . r) (the length-gauge kick)
int launch_phase_kick(int precision, const inqb_ctx& ctx, void* psi, long ld, int M, const double kick[3],
                      void* stream);
int launch_vgrad(int precision, long N, int M, const void* u, const void* w, long ld, double cre, double cim,
                 double* gV, void* stream);
// gA += Re(c <u| dH/dA |w>) from the forward coefficients U, W of u, w: natural order
// [N][M] (tiles = false) or the tile layout the H passes emit (tiles = true)
int launch_agrad(const inqb_ctx& ctx, const void* U, const void* W, const void* u, const void* w, long ld, int M,
                 double* acc, double cre, double cim, double* gA, void* stream, bool tiles = false);

// The V and A gradient of one backward ETRS half step: Lam[0..3] (leading dimensions
// ldL), Phi[0..3] (ldP), their forward coefficients FL, FP in the tile layout,
// weights w[i][j] = conj(c_{i+j+1}) (i + j <= 3); with Xi_i = sum_j w[i][j] Lam_j,
// gV += 2 Re sum_i conj(Xi_i) Phi_i and gA += 2 Re sum_i <Xi_i| dH/dA |Phi_i>.
int launch_half_grad(const inqb_ctx& ctx, const void* const Lam[4], const long ldL[4], const void* const Phi[4],
                     long ldP, const void* const FL[4], const void* const FP[4], const double w[4][4][2], int M,
                     double* gV, double* gA, void* stream);

}  // namespace inqb
