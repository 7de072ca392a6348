// inq_b200.hpp — header-only C++ host side of libinqb200.
//
// Mirrors the seam INQ's propagators use (HamiltonianType with
// `orbital_set operator()(orbital_set const&) const`, src/operations/exponential.hpp:21-69,
// src/real_time/etrs.hpp:22-24) on top of the C ABI in include/inqb200.h, so
// generic INQ-style code (Taylor exponentials, ETRS, Crank-Nicolson) drives the
// sm_100a kernels unchanged.  Errors become exceptions (INQ aborts; a library
// should let the caller decide).
//
//   inq::b200::device_orbitals   an [N][M] complex block in device memory
//   inq::b200::device_field      an [N] FP64 field in device memory (density, potential)
//   inq::b200::ks_hamiltonian    ks_hamiltonian<complex>::operator() (ks_hamiltonian.hpp:132-152)
//   inq::b200::exponential_in_place / etrs / crank_nicolson
//                                 operations / real_time counterparts
//   inq::b200::self_consistency / energy      update_hamiltonian (self_consistency.hpp:89-160)
//   inq::b200::mlwf_properties   the fork's TD-MLWF step (mlwf_properties.hpp:28-44)
//   inq::b200::io::save / load   checkpoints in INQ's restart layout (operations/io.hpp)
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstddef>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/inqb200.h"

namespace inq {
namespace b200 {

class error : public std::runtime_error {
 public:
  error(int status, const std::string& where)
      : std::runtime_error(where + ": " + inqb_last_error() + " (" + inqb_status_string(status) + ")"),
        status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int status, const char* where) {
  if (status != INQB_OK) throw error(status, where);
}

enum class precision { fp64 = INQB_FP64, mixed = INQB_MIXED };

// An [N][M] orbital block (orbital index fastest) owned in device memory:
// the storage of INQ's orbital_set (src/basis/field_set.hpp:51).
class device_orbitals {
 public:
  device_orbitals() = default;
  device_orbitals(long npoints, int nstates, precision p) : N_(npoints), M_(nstates), prec_(p) {
    const size_t bytes = (size_t)N_ * M_ * elem_bytes();
    if (cudaMalloc(&data_, bytes) != cudaSuccess) throw std::runtime_error("cudaMalloc failed for an orbital block");
  }
  device_orbitals(const device_orbitals& o) : device_orbitals(o.N_, o.M_, o.prec_) {
    if (cudaMemcpy(data_, o.data_, bytes(), cudaMemcpyDeviceToDevice) != cudaSuccess)
      throw std::runtime_error("orbital block copy failed");
  }
  device_orbitals(device_orbitals&& o) noexcept { swap(o); }
  device_orbitals& operator=(device_orbitals o) noexcept {
    swap(o);
    return *this;
  }
  ~device_orbitals() {
    if (data_) cudaFree(data_);
  }
  void swap(device_orbitals& o) noexcept {
    std::swap(data_, o.data_);
    std::swap(N_, o.N_);
    std::swap(M_, o.M_);
    std::swap(prec_, o.prec_);
  }
  // the skeleton of INQ's orbital_set: same shape, uninitialised
  device_orbitals skeleton() const { return device_orbitals(N_, M_, prec_); }

  void* data() { return data_; }
  const void* data() const { return data_; }
  long basis_size() const { return N_; }
  int set_size() const { return M_; }
  precision prec() const { return prec_; }
  size_t elem_bytes() const { return prec_ == precision::fp64 ? 16 : 8; }
  size_t bytes() const { return (size_t)N_ * M_ * elem_bytes(); }

  void upload(const std::vector<std::complex<double>>& host) {
    check_size(host.size());
    if (prec_ == precision::fp64) {
      if (cudaMemcpy(data_, host.data(), bytes(), cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("upload failed");
    } else {
      std::vector<std::complex<float>> f(host.begin(), host.end());
      if (cudaMemcpy(data_, f.data(), bytes(), cudaMemcpyHostToDevice) != cudaSuccess)
        throw std::runtime_error("upload failed");
    }
  }
  std::vector<std::complex<double>> download() const {
    std::vector<std::complex<double>> out((size_t)N_ * M_);
    if (prec_ == precision::fp64) {
      if (cudaMemcpy(out.data(), data_, bytes(), cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("download failed");
    } else {
      std::vector<std::complex<float>> f(out.size());
      if (cudaMemcpy(f.data(), data_, bytes(), cudaMemcpyDeviceToHost) != cudaSuccess)
        throw std::runtime_error("download failed");
      for (size_t i = 0; i < f.size(); i++) out[i] = f[i];
    }
    return out;
  }

 private:
  void check_size(size_t n) const {
    if (n != (size_t)N_ * M_) throw std::invalid_argument("host buffer has the wrong size");
  }
  void* data_ = nullptr;
  long N_ = 0;
  int M_ = 0;
  precision prec_ = precision::fp64;
};

// Gaussian KB projectors (s + 3 p) on a set of atoms, in projector_all layout.
struct kb_tables {
  int nproj = 0, L = 4, smax = 0;
  std::vector<int> counts, coords;
  std::vector<float> relpos;
  std::vector<double> beta, coeff;
};

inline kb_tables gaussian_kb(const std::array<double, 9>& lattice, const std::array<int, 3>& nr,
                             const std::vector<std::array<double, 3>>& atoms, double radius, double sigma,
                             double ekb_s, double ekb_p) {
  kb_tables t;
  t.nproj = (int)atoms.size();
  std::vector<std::vector<int>> c(atoms.size());
  std::vector<std::vector<float>> d(atoms.size()), r(atoms.size());
  for (size_t a = 0; a < atoms.size(); a++) {
    int n = 0;
    check(inqb_sphere_size(lattice.data(), nr.data(), atoms[a].data(), radius, &n), "inqb_sphere_size");
    c[a].resize(3 * (size_t)n);
    d[a].resize(n);
    r[a].resize(3 * (size_t)n);
    if (n > 0)
      check(inqb_sphere_points(lattice.data(), nr.data(), atoms[a].data(), radius, n, c[a].data(), d[a].data(),
                               r[a].data()),
            "inqb_sphere_points");
    t.smax = std::max(t.smax, n);
  }
  const size_t S = t.smax;
  t.counts.resize(t.nproj);
  t.coords.assign((size_t)t.nproj * S * 3, -1);
  t.relpos.assign((size_t)t.nproj * S * 3, 0.f);
  t.beta.assign((size_t)t.nproj * 4 * S, 0.0);
  t.coeff.resize((size_t)t.nproj * 4);
  for (int a = 0; a < t.nproj; a++) {
    const int n = (int)d[a].size();
    t.counts[a] = n;
    std::copy(c[a].begin(), c[a].end(), t.coords.begin() + (size_t)a * S * 3);
    std::copy(r[a].begin(), r[a].end(), t.relpos.begin() + (size_t)a * S * 3);
    std::vector<double> b(4 * (size_t)n);
    if (n > 0) check(inqb_gaussian_kb_beta(lattice.data(), n, d[a].data(), r[a].data(), sigma, b.data()), "kb beta");
    for (int l = 0; l < 4; l++)
      std::copy(b.begin() + (size_t)l * n, b.begin() + (size_t)(l + 1) * n, t.beta.begin() + ((size_t)a * 4 + l) * S);
    t.coeff[4 * a] = ekb_s;
    for (int l = 1; l < 4; l++) t.coeff[4 * a + l] = ekb_p;
  }
  return t;
}

// ks_hamiltonian<complex> on one GPU (src/hamiltonian/ks_hamiltonian.hpp:35-228).
// exchange_operator (src/hamiltonian/exchange_operator.hpp:30-231) as every theory this
// library runs has it: the exact-exchange coefficient is 0, so enabled() is false and
// the operator adds nothing to H|phi> (ks_hamiltonian.hpp:147) or to the energy
// (energy.hpp:87-91).  Exact exchange (hybrid and Hartree-Fock theories) is not
// provided; ks_hamiltonian refuses a coefficient that INQ would treat as enabled.
class exchange_operator {
 public:
  // INQ's test: |coefficient| > 1e-14 (exchange_operator.hpp:229-231)
  static bool would_enable(double coefficient) { return std::fabs(coefficient) > 1.0e-14; }
  bool enabled() const { return false; }
};

class ks_hamiltonian {
 public:
  // exchange_coefficient: the theory's exact-exchange fraction (ks_hamiltonian.hpp:80);
  // only 0 is accepted (std::invalid_argument otherwise, before any device work)
  ks_hamiltonian(const std::array<double, 9>& lattice, const std::array<int, 3>& nr, precision p, int device = 0,
                 double exchange_coefficient = 0.0)
      : lattice_(lattice), nr_(nr), prec_(p) {
    if (exchange_operator::would_enable(exchange_coefficient))
      throw std::invalid_argument("ks_hamiltonian: exact exchange is not provided (exchange coefficient " +
                                  std::to_string(exchange_coefficient) + ", only 0 is supported)");
    check(inqb_ctx_create(lattice.data(), nr[0], nr[1], nr[2], (int)p, device, &ctx_), "inqb_ctx_create");
  }
  ks_hamiltonian(const ks_hamiltonian&) = delete;
  ks_hamiltonian& operator=(const ks_hamiltonian&) = delete;
  ~ks_hamiltonian() { inqb_ctx_destroy(ctx_); }

  long basis_size() const { return (long)nr_[0] * nr_[1] * nr_[2]; }
  double volume_element() const { return inqb_volume_element(ctx_); }
  inqb_ctx* handle() const { return ctx_; }
  // exchange() (ks_hamiltonian.hpp:206-212): never enabled here
  const exchange_operator& exchange() const { return exchange_; }

  // scalar_potential() (ks_hamiltonian.hpp:200-204), one spin component
  void set_scalar_potential(const std::vector<double>& V) {
    if ((long)V.size() != basis_size()) throw std::invalid_argument("potential size");
    check(inqb_set_local_potential(ctx_, V.data()), "inqb_set_local_potential");
  }
  // uniform_vector_potential() plus the k-point, cartesian (self_consistency.hpp:152-160)
  void set_uniform_vector_potential(const std::array<double, 3>& A_cart) {
    std::array<double, 3> cov;
    check(inqb_cart_to_cov(ctx_, A_cart.data(), cov.data()), "inqb_cart_to_cov");
    check(inqb_set_vector_potential(ctx_, cov.data()), "inqb_set_vector_potential");
  }
  void set_projectors(const kb_tables& t) {
    check(inqb_set_projectors(ctx_, t.nproj, t.L, t.smax, t.counts.data(), t.coords.data(), t.relpos.data(),
                              t.beta.data(), t.coeff.data()),
          "inqb_set_projectors");
  }

  // operator(): a new orbital set H|phi>, as INQ returns by value
  device_orbitals operator()(const device_orbitals& phi) const {
    device_orbitals hphi = phi.skeleton();
    apply(phi, hphi);
    check_cuda(cudaStreamSynchronize(nullptr), "apply");
    return hphi;
  }
  // in-place form used by the propagators below (asynchronous on the default stream)
  void apply(const device_orbitals& phi, device_orbitals& hphi) const {
    check(inqb_apply_h(ctx_, phi.data(), hphi.data(), phi.set_size(), phi.set_size(), nullptr), "inqb_apply_h");
  }

 private:
  static void check_cuda(cudaError_t e, const char* where) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
  }
  std::array<double, 9> lattice_;
  std::array<int, 3> nr_;
  precision prec_;
  inqb_ctx* ctx_ = nullptr;
  exchange_operator exchange_;
};

// operations::exponential_in_place (src/operations/exponential.hpp:21-34) on the
// fused Horner-form kernels of the library.
inline void exponential_in_place(ks_hamiltonian& ham, std::complex<double> factor, device_orbitals& phi,
                                 int order = 4) {
  check(inqb_exponential(ham.handle(), phi.data(), phi.set_size(), phi.set_size(), factor.real(), factor.imag(), order,
                         nullptr),
        "inqb_exponential");
}

// real_time::etrs for a density-independent Hamiltonian (src/real_time/etrs.hpp:22-82)
inline void etrs(ks_hamiltonian& ham, double dt, const std::array<double, 3>& A_t, const std::array<double, 3>& A_tdt,
                 device_orbitals& phi) {
  std::array<double, 3> c1, c2;
  check(inqb_cart_to_cov(ham.handle(), A_t.data(), c1.data()), "inqb_cart_to_cov");
  check(inqb_cart_to_cov(ham.handle(), A_tdt.data(), c2.data()), "inqb_cart_to_cov");
  check(inqb_etrs_step(ham.handle(), phi.data(), phi.set_size(), phi.set_size(), dt, c1.data(), c2.data(), nullptr),
        "inqb_etrs_step");
}

// The generic Taylor exponential of INQ written against HamiltonianType alone:
// shows that ks_hamiltonian is a drop-in HamiltonianType (it only needs
// operator() and a shift).  Uses the library's axpby for the shift.
template <class HamiltonianType>
void exponential_generic(const HamiltonianType& ham, std::complex<double> factor, device_orbitals& phi,
                         int order = 4) {
  auto hnphi = ham(phi);
  std::complex<double> coeff = 1.0;
  for (int iter = 1; iter <= order; iter++) {
    if (iter > 1) hnphi = ham(hnphi);
    coeff *= factor / double(iter);
    check(inqb_axpby(ham.handle(), phi.set_size(), coeff.real(), coeff.imag(), hnphi.data(), phi.set_size(), 1.0, 0.0,
                     phi.data(), phi.set_size(), nullptr),
          "inqb_axpby");
  }
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) throw std::runtime_error("exponential sync");
}

// An [N] FP64 field in device memory: the density or a potential of one spin component
// (basis::field<real_space, double>).
class device_field {
 public:
  explicit device_field(long npoints) : N_(npoints) {
    if (cudaMalloc(&data_, sizeof(double) * N_) != cudaSuccess) throw std::runtime_error("cudaMalloc failed (field)");
  }
  device_field(const device_field&) = delete;
  device_field& operator=(const device_field&) = delete;
  ~device_field() {
    if (data_) cudaFree(data_);
  }
  double* data() { return data_; }
  const double* data() const { return data_; }
  long size() const { return N_; }
  void upload(const std::vector<double>& h) {
    if ((long)h.size() != N_) throw std::invalid_argument("field size");
    if (cudaMemcpy(data_, h.data(), sizeof(double) * N_, cudaMemcpyHostToDevice) != cudaSuccess)
      throw std::runtime_error("field upload failed");
  }
  std::vector<double> download() const {
    std::vector<double> h((size_t)N_);
    if (cudaMemcpy(h.data(), data_, sizeof(double) * N_, cudaMemcpyDeviceToHost) != cudaSuccess)
      throw std::runtime_error("field download failed");
    return h;
  }

 private:
  double* data_ = nullptr;
  long N_ = 0;
};

// observables::density::calculate (density.hpp:23-52): occupations on the device
inline void density(ks_hamiltonian& ham, const device_orbitals& phi, const device_field& occ, device_field& rho) {
  check(inqb_density(ham.handle(), phi.data(), phi.set_size(), phi.set_size(), occ.data(), rho.data(), nullptr),
        "inqb_density");
}

// The energy terms update_hamiltonian records (hamiltonian/energy.hpp:26-56)
struct energy {
  double external = 0.0, hartree = 0.0, xc = 0.0, nvxc = 0.0;
};

// self_consistency for static ions, an unpolarised density, no core density
// (self_consistency.hpp:28-160); theory: INQB_THEORY_NONE, _HARTREE or _LDA.
class self_consistency {
 public:
  self_consistency(int theory, const device_field* vion) : theory_(theory), vion_(vion) {}
  // update_hamiltonian (self_consistency.hpp:89-160): the potential of ham becomes
  // vion + V_H[rho] + v_xc[rho]
  void update_hamiltonian(ks_hamiltonian& ham, energy& en, const device_field& rho) const {
    double e[4];
    check(inqb_ks_potential(ham.handle(), rho.data(), vion_ ? vion_->data() : nullptr, theory_, e, nullptr),
          "inqb_ks_potential");
    en = energy{e[0], e[1], e[2], e[3]};
  }
  int theory() const { return theory_; }
  const double* vion() const { return vion_ ? vion_->data() : nullptr; }

 private:
  int theory_;
  const device_field* vion_;
};

// real_time::etrs with its self-consistency loop (etrs.hpp:22-82); rho is the density
// of phi on entry and of the propagated phi on exit.  Returns the SCF iterations.
inline int etrs(ks_hamiltonian& ham, double dt, const std::array<double, 3>& A_t, const std::array<double, 3>& A_tdt,
                device_orbitals& phi, const device_field& occ, device_field& rho, const self_consistency& sc,
                energy& en, int nscf = 5, double threshold = 5e-5) {
  std::array<double, 3> c1, c2;
  check(inqb_cart_to_cov(ham.handle(), A_t.data(), c1.data()), "inqb_cart_to_cov");
  check(inqb_cart_to_cov(ham.handle(), A_tdt.data(), c2.data()), "inqb_cart_to_cov");
  int iters = 0;
  double e[4];
  check(inqb_etrs_scf_step(ham.handle(), phi.data(), phi.set_size(), phi.set_size(), dt, c1.data(), c2.data(),
                           occ.data(), rho.data(), sc.vion(), sc.theory(), nscf, threshold, &iters, e, nullptr),
        "inqb_etrs_scf_step");
  en = energy{e[0], e[1], e[2], e[3]};
  return iters;
}

// real_time::crank_nicolson with its self-consistency loop and Broyden density mixing
// (crank_nicolson.hpp:41-114); rho is the density of phi on entry and of the
// propagated phi on exit; num_electrons is electrons.states().num_electrons().
// Returns the iterations run.
inline int crank_nicolson(ks_hamiltonian& ham, double dt, const std::array<double, 3>& A_t,
                          const std::array<double, 3>& A_tdt, device_orbitals& phi, const device_field& occ,
                          double num_electrons, device_field& rho, const self_consistency& sc, energy& en,
                          int max_iter = 300, double dens_tol = 1e-5) {
  std::array<double, 3> c1, c2;
  check(inqb_cart_to_cov(ham.handle(), A_t.data(), c1.data()), "inqb_cart_to_cov");
  check(inqb_cart_to_cov(ham.handle(), A_tdt.data(), c2.data()), "inqb_cart_to_cov");
  int iters = 0;
  double e[4];
  check(inqb_crank_nicolson_scf_step(ham.handle(), phi.data(), phi.set_size(), phi.set_size(), dt, c1.data(),
                                     c2.data(), occ.data(), num_electrons, rho.data(), sc.vion(), sc.theory(),
                                     max_iter, dens_tol, &iters, nullptr, e, nullptr),
        "inqb_crank_nicolson_scf_step");
  en = energy{e[0], e[1], e[2], e[3]};
  return iters;
}

// observables::mlwf_properties::calculate (mlwf_properties.hpp:28-44): phi rotated in
// place to the maximally localised gauge, then the reference's lines on out.
class mlwf_properties {
 public:
  explicit mlwf_properties(int maxsweep = 100, double tol = 1e-8) : maxsweep_(maxsweep), tol_(tol) {}
  void calculate(std::ostream& out, int time_step, ks_hamiltonian& ham, device_orbitals& phi) {
    const int M = phi.set_size();
    centres_.assign(3 * (size_t)M, 0.0);
    spreads_.assign((size_t)M, 0.0);
    check(inqb_mlwf_step(ham.handle(), phi.data(), M, M, maxsweep_, tol_, &sweeps_, centres_.data(), spreads_.data(),
                         nullptr),
          "inqb_mlwf_step");
    out << "Time step: " << time_step + 1 << "\n";
    out << "MLWFs:\n";
    for (int i = 0; i < M; ++i)
      out << "  WF " << i + 1 << ": " << centres_[3 * i] << "     " << centres_[3 * i + 1] << "     "
          << centres_[3 * i + 2] << "     Spread: " << spreads_[i] << std::endl;
  }
  const std::vector<double>& centres() const { return centres_; }
  const std::vector<double>& spreads() const { return spreads_; }
  int sweeps() const { return sweeps_; }

 private:
  int maxsweep_;
  double tol_;
  int sweeps_ = 0;
  std::vector<double> centres_, spreads_;
};

// Checkpoints in INQ's restart layout (operations/io.hpp:42-177,
// systems/electrons.hpp:323-375): states and occupations of one k-point block
// (first_state when the states are sharded), and the density.
namespace io {
inline void save(const std::string& dirname, ks_hamiltonian& ham, const device_orbitals& phi,
                 const std::vector<double>& occ, const device_field& rho, int first_state = 0, int kpin = 0) {
  check(inqb_save_orbitals(ham.handle(), dirname.c_str(), kpin, phi.data(), phi.set_size(), phi.set_size(),
                           first_state, occ.empty() ? nullptr : occ.data(), nullptr),
        "inqb_save_orbitals");
  check(inqb_save_density(ham.handle(), dirname.c_str(), rho.data(), nullptr), "inqb_save_density");
}
// false when a file is missing or short (io::load returns false there)
inline bool load(const std::string& dirname, ks_hamiltonian& ham, device_orbitals& phi, std::vector<double>& occ,
                 device_field& rho, int first_state = 0, int kpin = 0) {
  occ.assign((size_t)phi.set_size(), 0.0);
  int st = inqb_load_orbitals(ham.handle(), dirname.c_str(), kpin, phi.data(), phi.set_size(), phi.set_size(),
                              first_state, occ.data(), nullptr);
  if (st == INQB_ERR_IO) return false;
  check(st, "inqb_load_orbitals");
  st = inqb_load_density(ham.handle(), dirname.c_str(), rho.data(), nullptr);
  if (st == INQB_ERR_IO) return false;
  check(st, "inqb_load_density");
  return true;
}
}  // namespace io

}  // namespace b200
}  // namespace inq
