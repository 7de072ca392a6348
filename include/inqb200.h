/*
 * inqb200.h — C ABI of libinqb200, the B200 (sm_100a) implementation of INQ's
 * Kohn-Sham Hamiltonian application H|psi> and the real-time propagators built
 * on it.
 *
 * Conventions (identical to INQ; paths relative to the reference project root):
 *   - An orbital block is [N][ld] interleaved complex, orbital index fastest:
 *     element (point p, orbital m) at psi[p*ld + m], p = (ix*ny + iy)*nz + iz
 *     (src/basis/field_set.hpp:51, :188-194).  complex128 for INQB_FP64,
 *     complex64 for INQB_MIXED.  Device pointers are caller owned and 16-byte
 *     aligned; ld >= M.
 *   - The lattice is given as 9 doubles, row i = lattice vector a_i in bohr.
 *   - Vectors called "cov" are covariant components (k . a_i), as INQ stores
 *     the k-point plus vector potential (src/hamiltonian/self_consistency.hpp:152-160).
 *   - Every function returns an inqb_status; inqb_last_error() describes the
 *     last failure of the calling thread.  Functions taking a `stream`
 *     (a cudaStream_t, NULL = legacy default stream) are asynchronous unless
 *     stated otherwise.
 */
#ifndef INQB200_H
#define INQB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct inqb_ctx inqb_ctx;

enum inqb_status {
  INQB_OK = 0,
  INQB_ERR_INVALID = 1,       /* bad argument or call order */
  INQB_ERR_UNSUPPORTED = 2,   /* grid size / projector count not compiled in */
  INQB_ERR_CUDA = 3,          /* CUDA runtime error */
  INQB_ERR_NOMEM = 4,         /* device allocation failed */
  INQB_ERR_NONFINITE = 5,     /* NaN or Inf found in an input */
  INQB_ERR_NOT_POSITIVE_DEFINITE = 6, /* overlap matrix failed Cholesky */
  INQB_ERR_TIMEOUT = 7,       /* a bounded device-side wait gave up */
  INQB_ERR_IO = 8             /* a checkpoint file is missing, short or unwritable */
};

enum inqb_precision {
  INQB_FP64 = 0,   /* complex128 storage, FP64 arithmetic */
  INQB_MIXED = 1   /* complex64 storage and FFT/pointwise, FP64 reductions */
};

/* ---------------------------------------------------------------- library */
int inqb_version(void);
const char* inqb_status_string(int status);
const char* inqb_last_error(void);
/* 1 if an (nx, ny, nz) grid has compiled kernels for `precision`, else 0. */
int inqb_grid_supported(int nx, int ny, int nz, int precision);

/* ---------------------------------------------------------------- context
 * Replaces the construction of basis::real_space + hamiltonian::ks_hamiltonian
 * (src/basis/real_space.hpp:29-32, src/hamiltonian/ks_hamiltonian.hpp:79-90).
 * The grid is given explicitly (INQ derives it as round(|a_i| / spacing)). */
int inqb_ctx_create(const double lattice[9], int nx, int ny, int nz, int precision, int device,
                    inqb_ctx** out);
int inqb_ctx_destroy(inqb_ctx* ctx);
/* A second context with src's cell, grid, precision, device, local potential (as it is
 * on the device now, including a self-consistent update), vector potential, Fourier
 * mask, projectors, projection form and launch schedules, and a workspace of its own:
 * for work on another stream beside src (two calls on one context must not overlap).
 * The density-reduce hook is not copied.  No counterpart in the reference, whose
 * Hamiltonian is copied with its C++ copy constructor. */
int inqb_ctx_clone(const inqb_ctx* src, inqb_ctx** out);
/* Allocates the device workspace for blocks of up to M orbitals, so that the
 * later calls with M' <= M allocate nothing (INQ allocates per call from its
 * caching pool, external_libs/gpurun/include/gpu/array.hpp:66-116). */
int inqb_ctx_reserve(inqb_ctx* ctx, int M);
/* volume element dV = V_cell / N (src/basis/real_space.hpp:150-152) */
double inqb_volume_element(const inqb_ctx* ctx);
/* cartesian -> covariant components (src/systems/cell.hpp:185-187) */
int inqb_cart_to_cov(const inqb_ctx* ctx, const double cart[3], double cov[3]);

/* ---------------------------------------------------------------- Hamiltonian state
 * ks_hamiltonian::scalar_potential() (src/hamiltonian/ks_hamiltonian.hpp:200-204):
 * V[N] on the host, copied to the device. */
int inqb_set_local_potential(inqb_ctx* ctx, const double* V);
/* ks_hamiltonian::uniform_vector_potential() plus the k-point, covariant
 * (src/hamiltonian/ks_hamiltonian.hpp:214-221, used as phi.kpoint() + A). */
int inqb_set_vector_potential(inqb_ctx* ctx, const double kA_cov[3]);

/* operations::transform::zero_outside_sphere (src/operations/transform.hpp:363-364,
 * src/basis/fourier_space.hpp:87-93) applied to the kinetic term: with enable = 1
 * the kinetic energy of Fourier points with sum_d (n_d/N_d)^2 > 1/4 is zeroed, so
 * H = P K P + V + V_nl (still Hermitian).  Off by default, as in INQ; it keeps
 * Taylor propagators stable when 1/2|G_max|^2 dt/2 exceeds 2 sqrt(2). */
int inqb_set_fourier_sphere_mask(inqb_ctx* ctx, int enable);

/* ---------------------------------------------------------------- projector setup
 * Setup helpers; they need no context and no GPU.
 * basis::spherical_grid (src/basis/spherical_grid.hpp:59-158): the grid points
 * within `radius` of `center` (cartesian) including periodic replicas, with the
 * float distance and float contravariant relative position INQ stores.
 * inqb_sphere_points fills coords[npts][3], distance[npts], relpos[npts][3]. */
int inqb_sphere_size(const double lattice[9], const int nr[3], const double center[3], double radius,
                     int* npts);
int inqb_sphere_points(const double lattice[9], const int nr[3], const double center[3], double radius,
                       int npts, int* coords, float* distance, float* relpos);
/* projector::build (src/hamiltonian/projector.hpp:29-50) for Gaussian KB
 * projectors: beta[lm][p], lm = (s, p_-1, p_0, p_+1), radial r^l exp(-r^2/2s^2)
 * times real Y_lm of the relative position. */
int inqb_gaussian_kb_beta(const double lattice[9], int npts, const float* distance, const float* relpos,
                          double sigma, double* beta);
/* projector_all constructor (src/hamiltonian/projector_all.hpp:27-73): per-atom
 * tables padded to smax points: counts[nproj], coords[nproj][smax][3],
 * relpos[nproj][smax][3] (float), beta[nproj][L][smax], coeff[nproj][L]. */
int inqb_set_projectors(inqb_ctx* ctx, int nproj, int L, int smax, const int* counts, const int* coords,
                        const float* relpos, const double* beta, const double* coeff);

/* ---------------------------------------------------------------- H|psi>
 * ks_hamiltonian::operator()(orbital_set<real_space, complex> const&)
 * (src/hamiltonian/ks_hamiltonian.hpp:132-152):
 *   hpsi = IFFT(1/2|G+k+A|^2 FFT psi) + V psi + sum_a beta_a E_a beta_a^T dV psi
 * with projector phases exp(+-i (k+A).r).  hpsi may alias psi. */
int inqb_apply_h(inqb_ctx* ctx, const void* psi, void* hpsi, int M, int ld, void* stream);
/* The same on HOST buffers ([N][M], ld = M): copies in, applies, copies out,
 * synchronous.  This is the call an INQ host-memory orbital_set would use.  The
 * orbitals go in chunks of at least 32 whose copy-in, H apply and copy-out overlap on
 * three streams; page-locked host buffers let the copies run concurrently. */
int inqb_apply_h_host(inqb_ctx* ctx, const void* psi_host, void* hpsi_host, int M);
/* operations::transform::to_fourier / to_real (src/operations/transform.hpp:337-400):
 * forward unnormalised sign -1, backward sign +1 then 1/N.  out may alias in. */
int inqb_fft_forward(inqb_ctx* ctx, const void* in, void* out, int M, int ld, void* stream);
int inqb_fft_backward(inqb_ctx* ctx, const void* in, void* out, int M, int ld, void* stream);

/* ---------------------------------------------------------------- batched cells
 * Many independent cells (each its own context: grid, potential, projectors)
 * applied together as one CUDA graph with one concurrent branch per cell.  The
 * reference runs cells one after another; this has no single reference
 * counterpart (it batches ks_hamiltonian::operator(), ks_hamiltonian.hpp:132-152).
 * The first call with a given set of pointers and sizes captures and instantiates
 * the graph (it also runs each cell once, uncaptured, to set up workspace); later
 * calls with the same arguments only launch it.  The contexts must outlive the
 * batch and must not be used concurrently with it. */
typedef struct inqb_batch inqb_batch;
int inqb_batch_create(inqb_ctx* const* cells, int ncells, inqb_batch** out);
int inqb_batch_destroy(inqb_batch* batch);
int inqb_batch_apply_h(inqb_batch* batch, const void* const* psis, void* const* hpsis, const int* Ms,
                       const int* lds, void* stream);
/* The launch form of inqb_batch_apply_h.  PERSISTENT: one launch of a persistent
 * kernel whose CTAs take work items (cell, pass, tiles) from a device queue and wait,
 * with a time limit, for the items each depends on; the cells (at most 64) must share
 * one precision, have cubic grids of 16, 20, 24, 32, 40 or 48 points and use the
 * fused projection (INQB_ERR_UNSUPPORTED otherwise).  GRAPH: the CUDA graph above.
 * AUTO (the default): the form inqb_batch_autotune picked, GRAPH before it ran (and
 * where the cells do not fit the persistent kernel).  Takes effect at the next apply. */
enum inqb_batch_mode { INQB_BATCH_AUTO = 0, INQB_BATCH_GRAPH = 1, INQB_BATCH_PERSISTENT = 2 };
int inqb_batch_set_mode(inqb_batch* batch, int mode);
/* Times both forms on these arguments (2 untimed and 5 timed applies each, CUDA
 * events on stream) and makes the faster the one AUTO runs.  form (optional): the
 * pick; ms (optional, [2]): milliseconds per apply of GRAPH and PERSISTENT (-1 where
 * the cells do not fit the persistent kernel).  Synchronous; the outputs hold H psi. */
int inqb_batch_autotune(inqb_batch* batch, const void* const* psis, void* const* hpsis, const int* Ms,
                        const int* lds, void* stream, int* form, double* ms);
/* The form the last inqb_batch_apply_h set up (INQB_BATCH_GRAPH, INQB_BATCH_PERSISTENT,
 * or 0 before the first), and for the persistent form its work items and CTAs. */
int inqb_batch_info(inqb_batch* batch, int* form, int* nitems, int* ctas);
/* Synchronises stream and returns INQB_ERR_TIMEOUT when a device-side wait of a
 * persistent launch gave up since the last call (that launch stopped early and its
 * outputs are not valid; the batch and its contexts stay usable), else INQB_OK. */
int inqb_batch_status(inqb_batch* batch, void* stream);
/* Time limit of one device-side wait of the persistent launch, in (0, 60] seconds
 * (default 2). */
int inqb_batch_set_wait_limit(inqb_batch* batch, double seconds);
/* Test hook: when on, one work item of the next persistent plan waits for a count
 * that no item reaches, so that wait runs out after the limit above and the launch
 * reports INQB_ERR_TIMEOUT through inqb_batch_status. */
int inqb_batch_test_unreachable_wait(inqb_batch* batch, int on);

/* ---------------------------------------------------------------- propagation
 * operations::exponential_in_place (src/operations/exponential.hpp:21-34):
 * psi <- sum_{k<=order} (f H)^k / k! psi, f = f_re + i f_im, in place. */
int inqb_exponential(inqb_ctx* ctx, void* psi, int M, int ld, double f_re, double f_im, int order,
                     void* stream);
/* real_time::etrs (src/real_time/etrs.hpp:22-82) for a density-independent H:
 * psi <- T4(i dt/2 H(kA_tdt)) T4(i dt/2 H(kA_t)) psi, in place.  Leaves the
 * context's vector potential at kA_tdt, as self_consistency does. */
int inqb_etrs_step(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                   const double kA_tdt_cov[3], void* stream);

/* ---------------------------------------------------------------- observables
 * observables::density::calculate (src/observables/density.hpp:23-33,77-95):
 * rho[p] = sum_m occ[m] |psi[p][m]|^2; occ and rho are FP64 device arrays. */
int inqb_density(inqb_ctx* ctx, const void* psi, int M, int ld, const double* occ, double* rho,
                 void* stream);
/* observables::dipole(density) (src/observables/dipole.hpp:23-40):
 * out = dV sum_p r_p rho[p] with symmetric-range r; rho on device, out on
 * host; synchronous. */
int inqb_dipole(inqb_ctx* ctx, const double* rho, double out[3], void* stream);
/* Band energies eps[m] = Re(<Hpsi_m|psi_m>) / <psi_m|psi_m> as
 * operations::overlap_diagonal_normalized(H psi, psi, real_part) computes them
 * for hamiltonian::energy (src/operations/overlap_diagonal.hpp:118-170,
 * src/hamiltonian/energy.hpp:74-76); FP64 sums in both precisions.  eps is host
 * memory [M]; synchronous. */
int inqb_band_energies(inqb_ctx* ctx, const void* psi, const void* hpsi, int M, int ld, double* eps,
                       void* stream);
/* operations::orthogonalize (src/operations/orthogonalize.hpp:25-32): FP64
 * overlap S = dV psi^H psi, Cholesky S = U^H U, psi <- psi U^-1; synchronous. */
int inqb_orthonormalize(inqb_ctx* ctx, void* psi, int M, int ld, void* stream);
/* Orbital-sharded orthonormalisation, the pieces of operations::orthogonalize when
 * the states are split over ranks (src/operations/orthogonalize.hpp:25-32).  Each rank
 * holds a block of orbitals; the caller circulates the blocks and sums the matrices
 * (pinq_b200.parallel.sharded_orthonormalize_ does it over torch.distributed).
 * S, R: FP64 complex device matrices, interleaved (re, im), row-major with row stride
 * lds / ldr in complex elements.
 * inqb_overlap_block: S = dV a^H b for an Ma-orbital block a and an Mb-orbital block
 * b: one block of operations::overlap's set-parallel branch
 * (src/operations/overlap.hpp:47-72), which circulates the blocks and all-reduces
 * the zero-padded matrix.  S is overwritten. */
int inqb_overlap_block(inqb_ctx* ctx, const void* a, int Ma, int lda, const void* b, int Mb, int ldb, double* S,
                       int lds, void* stream);
/* matrix::cholesky then matrix::invert_triangular (src/matrix/cholesky.hpp:28-100,
 * src/operations/rotate.hpp:147-157) of the M x M Hermitian S in place: on return
 * S = U^-1, upper triangular (the strict lower part zero), where S = U^H U.
 * INQB_ERR_NOT_POSITIVE_DEFINITE when a pivot fails; synchronous. */
int inqb_cholesky_inverse(inqb_ctx* ctx, double* S, int M, int lds, void* stream);
/* out = a R: a is an Ma-orbital block, R the Ma x Mo FP64 block, out an Mo-orbital
 * block in the context precision (FP64 sums); out must not overlap a.  One term of
 * operations::rotate's set-parallel branch (src/operations/rotate.hpp:100-125), whose
 * terms are summed on the rank that owns the output orbitals. */
int inqb_rotate_block(inqb_ctx* ctx, const void* a, int Ma, int lda, const double* R, int ldr, int Mo, void* out,
                      int ldo, void* stream);
/* The same orthonormalisation without any device allocation (no counterpart in the
 * reference).  inqb_orthonormalize allocates its M x M scratch on every call; this
 * one uses a fixed array of 2 MiB compiled into the library, which every GPU that
 * loads the library holds until the process exits.  It is for callers that may not
 * call cudaMalloc: code running inside another framework's memory pool or allocator
 * hooks, or a service whose device memory budget is fixed after start-up.
 *   - M <= 256 orbitals; larger M returns INQB_ERR_UNSUPPORTED.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress); make that first call before any stream capture.  The
 *     address is kept until the process exits, so, like every context of this
 *     library, it does not survive a cudaDeviceReset of that device.
 *   - All calls on a device share the array: calls that overlap on the GPU (from
 *     different streams or threads) race.  Each call clears what it accumulates.
 *   - Synchronous, like inqb_orthonormalize; the context itself was created earlier. */
int inqb_orthonormalize_noalloc(inqb_ctx* ctx, void* psi, int M, int ld, void* stream);

/* ---------------------------------------------------------------- adjoint building blocks
 * The reverse-mode pieces of the ETRS step (the reference has no adjoint; these
 * differentiate real_time::etrs, src/real_time/etrs.hpp:22-82).  Orbital blocks
 * follow the layout above; gradients are FP64 device arrays accumulated in place.
 * y <- a x + b y  (operations::shift generalised, src/operations/shift.hpp:33-44) */
int inqb_axpby(inqb_ctx* ctx, int M, double a_re, double a_im, const void* x, int ldx, double b_re, double b_im,
               void* y, int ldy, void* stream);
/* out[p][m] = scale * occ[m] * r_dir(p) * psi[p][m], r the symmetric-range
 * cartesian position of dipole.hpp:23-30: the derivative of the dipole with
 * respect to conj(psi) for scale = dV. */
int inqb_position_scale(inqb_ctx* ctx, const void* psi, int ld, void* out, int ldo, int M, int dir,
                        const double* occ, double scale, void* stream);
/* gV[p] += Re(c sum_m conj(u[p][m]) w[p][m]) = Re(c <u| dH/dV(p) |w>) */
int inqb_accum_potential_gradient(inqb_ctx* ctx, const void* u, const void* w, int M, int ld, double c_re,
                                  double c_im, double* gV, void* stream);
/* gA[d] += Re(c <u| dH/dA_d |w>), d = x, y, z cartesian, at the context's current
 * k + A: the kinetic term (G + k + A)_d and the nonlocal position commutator of
 * projector_all::position_commutator (src/hamiltonian/projector_all.hpp:319-403). */
int inqb_accum_vector_potential_gradient(inqb_ctx* ctx, const void* u, const void* w, int M, int ld, double c_re,
                                         double c_im, double* gA, void* stream);

/* real_time::crank_nicolson for a density-independent H
 * (src/real_time/crank_nicolson.hpp:22-114): rhs = (1 - i dt/2 H(kA_t)) psi, then
 * sweeps of solvers::steepest_descent (five steps each, no preconditioner,
 * src/solvers/steepest_descent.hpp:22-80) on (1 + i dt/2 H(kA_tdt)) psi' = rhs,
 * starting from psi, until the largest residual dV <r|r> of a sweep is below tol
 * or max_sweeps ran (the reference caps its loop at 300).  The reference ends the
 * loop on the density change under Broyden mixing, which for a density-independent
 * H only sets the number of sweeps.  Solver sums and step lengths are FP64.
 * Synchronous (one read-back per sweep); sweeps and residual may be NULL. */
int inqb_crank_nicolson_step(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                             const double kA_tdt_cov[3], int max_sweeps, double tol, int* sweeps, double* residual,
                             void* stream);
/* Bytes of the powers buffer of one step of inqb_etrs_step_powers for M orbitals. */
int inqb_etrs_powers_size(inqb_ctx* ctx, int M, size_t* bytes);
/* One ETRS step (the reference's real_time::etrs step with a density-independent
 * H, src/real_time/etrs.hpp:22-82) that also keeps what its adjoint needs:
 * psi <- T(kA_tdt) T(kA_t) psi, T = sum_{k<=4} (i dt/2 H)^k / k!.  powers (16-byte
 * aligned, inqb_etrs_powers_size bytes) receives 8 [N][M] blocks, H^k psi_t at kA_t
 * (k = 0..3) then H^k phi at kA_tdt (phi the half-stepped orbitals), followed by
 * their forward 3-D coefficients as the H kernels hold them (an opaque layout the
 * adjoint step reads).  Unlike inqb_etrs_step it sums the series term by term (no
 * Horner), like the reference's exponential. */
int inqb_etrs_step_powers(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                          const double kA_tdt_cov[3], void* powers, void* stream);
/* The step of inqb_etrs_step_powers keeping nothing: the same term-by-term sums, so
 * the same orbitals bit for bit, without writing the powers or their coefficients
 * (the steps of a checkpointed forward pass whose powers the backward recomputes). */
int inqb_etrs_step_terms(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                         const double kA_tdt_cov[3], void* stream);
/* Reverse of that step for a real objective (the reference has no adjoint):
 * lambda <- U^dagger lambda, gV[p] += 2 Re sum_i conj(Xi_i) Phi_i and
 * gA_t[d], gA_tdt[d] += 2 Re sum_i <Xi_i| dH/dA_d |Phi_i> for the two half steps,
 * where Phi_i are the stored powers and Xi_i = sum_j conj(c_{i+j+1}) H^j lambda. */
int inqb_etrs_adjoint_step(inqb_ctx* ctx, void* lambda, int M, int ld, double dt, const double kA_t_cov[3],
                           const double kA_tdt_cov[3], const void* powers, double* gV, double* gA_t,
                           double* gA_tdt, void* stream);

/* perturbations::kick (src/perturbations/kick.hpp:20-61): the zero-time kick of a
 * length-gauge run, psi *= exp(-i kick . r) with kick a cartesian field and r the
 * grid point in the symmetric range.  In a periodic cell INQ uses the velocity gauge
 * instead, where the kick is the constant vector potential A = -kick (pass it as k + A
 * to the propagators) and zero_step leaves the orbitals unchanged. */
int inqb_kick(inqb_ctx* ctx, void* psi, int M, int ld, const double kick_cart[3], void* stream);

/* ---------------------------------------------------------------- density -> potential
 * solvers::poisson for a periodic cell (src/solvers/poisson.hpp:29-35,66-100,193-211),
 * the field_set form: M complex fields [N][M] of the context precision,
 * out(G) = 4 pi in(G) / |G|^2 with 0 at |G|^2 < 1e-6.  Three fused launches (the
 * factor is applied inside the x-line transform pass).  out may alias in. */
int inqb_poisson(inqb_ctx* ctx, const void* in, void* out, int M, int ld, void* stream);

/* Theories of the density -> potential step (options::theory, src/options/theory.hpp:
 * 31-62): non-interacting, Hartree only, and LDA (Hartree + XC_LDA_X + XC_LDA_C_PZ). */
enum {
  INQB_THEORY_NONE = 0,
  INQB_THEORY_HARTREE = 1,
  INQB_THEORY_LDA = 2
};
/* self_consistency::update_hamiltonian (src/hamiltonian/self_consistency.hpp:89-160)
 * for an unpolarised density with no core density, no electric field and static
 * ions: the context's local potential becomes vion + V_H[rho] + v_xc[max(rho, 0)]
 * (xc_term.hpp:63-142), on the device.  rho and vion are FP64 device arrays [N];
 * vion may be NULL (zero).  energies (host, may be NULL; non-NULL synchronises)
 * receives {external, hartree, xc, nvxc}: dV sum rho vion, dV/2 sum rho V_H,
 * dV sum e_xc n, dV sum rho v_xc, as hamiltonian::energy records them.  The
 * exchange-correlation sums are FP64 in both precisions; V_H comes from
 * inqb_poisson in the context precision. */
int inqb_ks_potential(inqb_ctx* ctx, const double* rho, const double* vion, int theory, double energies[4],
                      void* stream);
/* real_time::etrs with its self-consistency loop (src/real_time/etrs.hpp:22-82), static
 * ions, no induced vector potential, exchange off.  On entry the context's potential
 * must be the Kohn-Sham potential of rho (inqb_ks_potential) and rho (FP64 device [N])
 * the density of psi; on exit psi and rho are at t + dt and the potential is that of
 * the last update.  Steps: save = T(i dt/2 H(kA_t)) psi and psi = T(i dt H(kA_t)) psi
 * sharing the H^k psi (operations::exponential_2_for_1); rho = density(psi); update
 * the potential; then for iscf < nscf: psi = T(i dt/2 H(kA_tdt)) save, rho =
 * density(psi), delta = dV sum |rho - rho_old|, update the potential, stop when
 * delta < threshold.  occ: FP64 device [M].  The reference uses nscf = 5 and
 * threshold 5e-5.  Synchronises once per SCF iteration (delta is read back).
 * iters and energies (host) may be NULL. */
int inqb_etrs_scf_step(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                       const double kA_tdt_cov[3], const double* occ, double* rho, const double* vion, int theory,
                       int nscf, double threshold, int* iters, double energies[4], void* stream);
/* real_time::crank_nicolson with its self-consistency loop (src/real_time/crank_nicolson.hpp:41-114),
 * static ions, no induced vector potential, exchange off.  Entry conditions as for
 * inqb_etrs_scf_step: the potential is the Kohn-Sham potential of rho, the density of
 * psi at t.  rhs = (1 - i dt/2 H(kA_t)) psi; then for istep < max_iter: update the
 * potential from rho at kA_tdt; five steps of solvers::steepest_descent on
 * (1 + i dt/2 H) psi = rhs from the current psi (as in inqb_crank_nicolson_step);
 * new = density(psi); stop when dV sum |rho - new| / num_electrons < dens_tol;
 * otherwise rho becomes the Broyden mix of rho and new (mixers::broyden with 4 steps
 * and mixing 0.3, src/mixers/broyden.hpp:26-160) normalised to num_electrons
 * (observables::density::normalize, src/observables/density.hpp:100-111).  On exit
 * rho = density(psi) and the potential is updated from it.  The reference uses
 * max_iter 300 and dens_tol 1e-5; num_electrons is the total over all ranks
 * (electrons.states().num_electrons()).  The mixer's vectors are FP64 on the device;
 * its small solve runs on the host.  Synchronises a few times per iteration.  occ:
 * FP64 device [M]; vion may be NULL (zero); iters, residual (the solver's last
 * largest dV <r|r>) and energies (host) may be NULL.  Calls the density-reduce
 * callback like inqb_etrs_scf_step. */
int inqb_crank_nicolson_scf_step(inqb_ctx* ctx, void* psi, int M, int ld, double dt, const double kA_t_cov[3],
                                 const double kA_tdt_cov[3], const double* occ, double num_electrons, double* rho,
                                 const double* vion, int theory, int max_iter, double dens_tol, int* iters,
                                 double* residual, double energies[4], void* stream);
/* The exchange step of an orbital-sharded run (one block of states per GPU): INQ sums
 * the density over its states communicator (src/observables/density.hpp:77-95).  When
 * set, inqb_etrs_scf_step and inqb_crank_nicolson_scf_step call fn(rho, N, user) after
 * each density of their own orbitals,
 * with the stream synchronised; fn must leave the sum over all ranks in rho (device
 * memory) and return 0 when the reduction is complete; nonzero ends the step with
 * INQB_ERR_INVALID.  fn NULL removes it. */
typedef int (*inqb_density_reduce_fn)(double* rho, long n, void* user);
int inqb_set_density_reduce(inqb_ctx* ctx, inqb_density_reduce_fn fn, void* user);

/* ---------------------------------------------------------------- checkpoints
 * INQ's restart layout, so that runs resume from their own checkpoints and exchange
 * orbitals with INQ (operations::io::save/load, src/operations/io.hpp:42-177, as
 * systems::electrons::save/try_load arranges them, src/systems/electrons.hpp:323-375):
 *   <dir>/kpin<kpin>/states/<state>_0000000000   raw complex128 [N] per state,
 *                                                 grid order p = (ix ny + iy) nz + iz
 *   <dir>/kpin<kpin>/occupations/array           raw FP64, this block at offset first_state
 *   <dir>/spin_density/0000000000                raw FP64 [N]
 * with numbers written "%010ld" (utils::num_to_str, src/utils/num_str.hpp:20-24).
 * The files are complex128 in both precisions (a mixed context widens on save and
 * rounds on load).  psi holds states first_state .. first_state + M - 1 (a rank's
 * block when the states are sharded); occ is a host array of M values or NULL.
 * Loading a missing or short file returns INQB_ERR_IO, as io::load returns false.
 * Synchronous. */
int inqb_save_orbitals(inqb_ctx* ctx, const char* dirname, int kpin, const void* psi, int M, int ld,
                       int first_state, const double* occ, void* stream);
int inqb_load_orbitals(inqb_ctx* ctx, const char* dirname, int kpin, void* psi, int M, int ld, int first_state,
                       double* occ, void* stream);
int inqb_save_density(inqb_ctx* ctx, const char* dirname, const double* rho, void* stream);
int inqb_load_density(inqb_ctx* ctx, const char* dirname, double* rho, void* stream);

/* ---------------------------------------------------------------- TD-MLWF
 * The fork's time-dependent maximally localised Wannier functions
 * (observables::mlwf_properties::calculate, src/observables/mlwf_properties.hpp:28-44).
 * inqb_mlwf_step = tdmlwf_trans::update + compute_transform + apply_transform and the
 * centres and spreads: the six matrices a_k = <psi_m| t_k |psi_n> of the normalised
 * states (t = cos, sin of 2 pi r_d / |a_d|; tdmlwf_trans.hpp:96-172), their joint
 * diagonalisation by JADE (jade_complex.hpp:32-335; the reference calls it with
 * maxsweep 100, tol 1e-8), psi <- psi u^H (operations::rotate), then per state the
 * centre L t (t_d = atan2(Re adiag_sin, Re adiag_cos) / 2 pi, L's rows the lattice
 * vectors, as tdmlwf_trans::center writes it) and the spread
 * sqrt(sum_d (1 - |c_d|^2 - |s_d|^2) / |b_d|^2).  centres [M][3], spreads [M] and
 * sweeps are host outputs and may be NULL.  Synchronises once per JADE sweep.
 * FP64 matrices and rotations in both precisions; in the mixed precision the matrix
 * products are FP32 summed over 16 points, then FP64. */
int inqb_mlwf_step(inqb_ctx* ctx, void* psi, int M, int ld, int maxsweep, double tol, int* sweeps, double* centres,
                   double* spreads, void* stream);
/* The pieces, on device arrays of complex128: a [6][M][M] from psi
 * (tdmlwf_trans::update); jade_complex on a (rotated in place), u [M][M], adiag [6][M];
 * psi <- psi u^H. */
int inqb_mlwf_matrices(inqb_ctx* ctx, const void* psi, int M, int ld, void* a, void* stream);
int inqb_jade(inqb_ctx* ctx, int M, void* a, void* u, void* adiag, int maxsweep, double tol, int* sweeps,
              void* stream);
int inqb_mlwf_rotate(inqb_ctx* ctx, void* psi, int M, int ld, const void* u, void* stream);
/* The pieces of the TD-MLWF step over orbitals split across ranks (the reference
 * distributes the basis instead and all-reduces the matrices over it,
 * src/wannier/tdmlwf_trans.hpp:96-172).  The caller circulates the blocks and sums;
 * pinq_b200.parallel.sharded_mlwf_step_ does it over torch.distributed.
 * inqb_mlwf_gram_block: Z [3][Ma][Mb] (device complex128) = sum_p conj(a_m(p))
 *   e^{i 2 pi r_d(p) / |a_d|} b_n(p), one block of the three weighted Gram matrices.
 * inqb_mlwf_finish: a [6][M][M] of tdmlwf_trans::update from the summed Z [3][M][M] and
 *   norms[M] = sum_p |psi_m|^2 (device FP64).
 * inqb_orbital_norms: norms[M] (device FP64) of an orbital block; synchronous.
 * inqb_mlwf_centres: centres [M][3] and spreads [M] (host) from adiag [6][M] (host
 *   complex128), tdmlwf_trans::center / spread2 (tdmlwf_trans.hpp:196-312). */
int inqb_mlwf_gram_block(inqb_ctx* ctx, const void* a, int Ma, int lda, const void* b, int Mb, int ldb, void* Z,
                         void* stream);
int inqb_mlwf_finish(inqb_ctx* ctx, int M, const void* Z, const double* norms, void* a, void* stream);
int inqb_orbital_norms(inqb_ctx* ctx, const void* psi, int M, int ld, double* norms, void* stream);
int inqb_mlwf_centres(inqb_ctx* ctx, int M, const double* adiag, double* centres, double* spreads);

/* ---------------------------------------------------------------- launch schedules
 * (no counterpart in the reference; its kernels have fixed launch shapes).  A
 * schedule is {ysplit, threads of pass 1, of pass 2, of pass 3}: ysplit CTAs share
 * one x-plane in the first pass (a divisor of the tiles per plane), and each pass
 * runs 64..256 threads per CTA (multiples of 32).  Schedules are kept per orbital
 * count M; counts without one use the compiled default. */
/* Time the candidates (every ysplit with 128 and 256 threads for the first pass,
 * 128 and 256 threads for the others) on zeroed M-orbital blocks with CUDA events
 * and keep the fastest for M; schedule (may be NULL) receives it.  Allocates two
 * scratch blocks for the duration of the call; synchronous. */
int inqb_autotune(inqb_ctx* ctx, int M, void* stream, int schedule[4]);
/* Set (or with schedule NULL, clear) the schedule used for M orbitals. */
int inqb_set_schedule(inqb_ctx* ctx, int M, const int schedule[4]);

/* ---------------------------------------------------------------- profiling
 * Per-pass CUDA-event timing of the next max_applies H applications, recorded
 * on the stream the kernels run on; the counterpart of INQ's scoped timers
 * (CALI_CXX_MARK_SCOPE, src/utils/profiling.hpp:12, external_libs/kalimotxo/cali.h).
 * inqb_timing_stop waits for the recorded events and returns the summed
 * milliseconds of the three passes (KB projection + z and inner y transforms,
 * outer y and x transforms + kinetic, inverse transforms + potential/nonlocal
 * epilogue).  inqb_timing_passes returns the same with the projection kernel
 * apart: [projection, first pass, second pass, third pass]. */
int inqb_timing_start(inqb_ctx* ctx, int max_applies);
int inqb_timing_stop(inqb_ctx* ctx, double ms_per_pass[3], int* napplies);
int inqb_timing_passes(inqb_ctx* ctx, double ms[4], int* napplies);

/* ---------------------------------------------------------------- projection and device status
 * How H|psi> forms the KB projections proj[a][l][m] of projector_all::project
 * (src/hamiltonian/projector_all.hpp:98-216).  Both are deterministic: every partial
 * sum has one owner and the partials are added in a fixed order.
 *   INQB_PROJECTION_FUSED (default): summed inside the first tile pass while the tile
 *     is in shared memory (FP32 products, FP64 sums), one partial per (x-plane, half
 *     of its row classes, atom), added per atom by a small finish kernel.
 *   INQB_PROJECTION_KERNEL: a kernel of its own before the tile passes, one CTA per
 *     (atom, block of orbitals) that gathers the orbitals at the atom's sphere points.
 *     In the mixed precision it is a tcgen05 tensor-core contraction (TF32 with a
 *     split-precision correction, FP64 sums per chunk of 32 points); in FP64 it runs
 *     on the CUDA cores.  It reads the sphere points' orbitals once more from memory,
 *     and measures slower than the fused form; orbital blocks whose complex64 rows are
 *     not 16-byte aligned (odd ld) take the fused form. */
enum inqb_projection_mode { INQB_PROJECTION_FUSED = 0, INQB_PROJECTION_KERNEL = 1 };
int inqb_set_projection_mode(inqb_ctx* ctx, int mode);
/* Kernels with a bounded device-side wait record a failed wait in a device word of
 * the context instead of waiting forever.  This synchronises `stream`, returns
 * INQB_ERR_TIMEOUT (and clears the word) if one gave up since the last call, whose
 * results are then not valid, else INQB_OK.  No counterpart in the reference (its
 * gpu::run synchronises after every kernel, external_libs/gpurun/include/gpu/run.hpp:76). */
int inqb_device_status(inqb_ctx* ctx, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* INQB200_H */
