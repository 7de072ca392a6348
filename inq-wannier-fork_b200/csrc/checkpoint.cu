// Orbital and density checkpoints in INQ's restart layout, for resume and for
// exchange with INQ itself:
//
//   <dir>/kpin<k>/states/<state>_<spinor>   raw complex128 [N] per state, grid order
//                                            p = (ix ny + iy) nz + iz
//   <dir>/kpin<k>/occupations/array          raw FP64, the block's values at offset
//                                            first_state
//   <dir>/spin_density/<component>           raw FP64 [N]
//
// (operations::io::save/load of orbital_set, field_set and arrays,
// src/operations/io.hpp:42-177; systems::electrons::save/try_load,
// src/systems/electrons.hpp:323-375; numbers as utils::num_to_str writes them,
// "%010ld", src/utils/num_str.hpp:20-24.)  The files hold complex128 whatever the
// context precision: a mixed context widens complex64 on save and rounds on load.
//
// The device keeps [N][ld] orbital-fastest blocks, so a state's file is one column.
// A tiled transpose gathers a chunk of columns into contiguous complex128 rows, one
// copy brings the chunk to pinned host memory, and writer threads put one file per
// state while the next chunk is gathered (two host buffers).  Loading runs the same
// steps backwards.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <future>
#include <string>
#include <vector>

#include "checkpoint.h"
#include "dft.cuh"
#include "inqb_internal.h"

namespace inqb {

namespace {

constexpr int kTile = 32;
constexpr size_t kChunkBytes = size_t(64) << 20;  // host/device staging per chunk

// out[j][p] = psi[p][m0 + j] for j < mc, as complex128
template <typename T>
__global__ void __launch_bounds__(kTile * 8)
    k_gather_states(const cplx<T>* __restrict__ psi, long ld, int m0, int mc, long N, double2* __restrict__ out) {
  __shared__ double2 tile[kTile][kTile + 1];
  const long p0 = (long)blockIdx.x * kTile;
  const int j0 = blockIdx.y * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int i = ty; i < kTile; i += 8) {
    const long p = p0 + i;
    const int j = j0 + tx;
    if (p < N && j < mc) {
      const cplx<T> v = psi[p * ld + m0 + j];
      tile[i][tx] = make_double2((double)v.x, (double)v.y);
    }
  }
  __syncthreads();
  for (int i = ty; i < kTile; i += 8) {
    const int j = j0 + i;
    const long p = p0 + tx;
    if (p < N && j < mc) out[(long)j * N + p] = tile[tx][i];
  }
}

// psi[p][m0 + j] = in[j][p] (rounded to the context precision)
template <typename T>
__global__ void __launch_bounds__(kTile * 8)
    k_scatter_states(const double2* __restrict__ in, int mc, long N, cplx<T>* __restrict__ psi, long ld, int m0) {
  __shared__ double2 tile[kTile][kTile + 1];
  const long p0 = (long)blockIdx.x * kTile;
  const int j0 = blockIdx.y * kTile;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int i = ty; i < kTile; i += 8) {
    const int j = j0 + i;
    const long p = p0 + tx;
    if (p < N && j < mc) tile[tx][i] = in[(long)j * N + p];
  }
  __syncthreads();
  for (int i = ty; i < kTile; i += 8) {
    const long p = p0 + i;
    const int j = j0 + tx;
    if (p < N && j < mc) {
      const double2 v = tile[i][tx];
      psi[p * ld + m0 + j] = mk<T>((T)v.x, (T)v.y);
    }
  }
}

std::string num_to_str(long n) {
  char buf[32];
  std::snprintf(buf, sizeof(buf), "%010ld", n);
  return std::string(buf);
}

std::string state_file(const std::string& dir, int kpin, long state) {
  return dir + "/kpin" + num_to_str(kpin) + "/states/" + num_to_str(state) + "_" + num_to_str(0);
}

// Writes [bytes] at offset; truncate empties the file first.  Returns "" or an error.
std::string write_file(const std::string& path, const void* data, size_t bytes, size_t offset, bool truncate) {
  const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | (truncate ? O_TRUNC : 0), 0644);
  if (fd < 0) return "cannot create '" + path + "': " + std::strerror(errno);
  const char* p = static_cast<const char*>(data);
  size_t done = 0;
  while (done < bytes) {
    const ssize_t w = ::pwrite(fd, p + done, bytes - done, (off_t)(offset + done));
    if (w <= 0) {
      const std::string e = "cannot write '" + path + "': " + std::strerror(errno);
      ::close(fd);
      return e;
    }
    done += (size_t)w;
  }
  if (::close(fd) != 0) return "cannot close '" + path + "'";
  return "";
}

// Reads exactly [bytes] at offset; a missing or short file is an error.
std::string read_file(const std::string& path, void* data, size_t bytes, size_t offset) {
  const int fd = ::open(path.c_str(), O_RDONLY);
  if (fd < 0) return "cannot open '" + path + "'";
  char* p = static_cast<char*>(data);
  size_t done = 0;
  while (done < bytes) {
    const ssize_t r = ::pread(fd, p + done, bytes - done, (off_t)(offset + done));
    if (r <= 0) {
      ::close(fd);
      return "'" + path + "' is shorter than expected";
    }
    done += (size_t)r;
  }
  ::close(fd);
  return "";
}

std::string make_dirs(const std::string& d) {
  std::error_code ec;
  std::filesystem::create_directories(d, ec);
  if (ec) return "cannot create directory '" + d + "': " + ec.message();
  return "";
}

struct PinnedPair {
  void* h[2] = {nullptr, nullptr};
  ~PinnedPair() {
    for (void* p : h)
      if (p) cudaFreeHost(p);
  }
};

template <typename T>
int launch_gather(const void* psi, long ld, int m0, int mc, long N, double2* out, cudaStream_t st) {
  const dim3 grid((unsigned)((N + kTile - 1) / kTile), (unsigned)((mc + kTile - 1) / kTile));
  k_gather_states<T><<<grid, dim3(kTile, 8), 0, st>>>((const cplx<T>*)psi, ld, m0, mc, N, out);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

template <typename T>
int launch_scatter(const double2* in, int mc, long N, void* psi, long ld, int m0, cudaStream_t st) {
  const dim3 grid((unsigned)((N + kTile - 1) / kTile), (unsigned)((mc + kTile - 1) / kTile));
  k_scatter_states<T><<<grid, dim3(kTile, 8), 0, st>>>(in, mc, N, (cplx<T>*)psi, ld, m0);
  INQB_CUDA_TRY(cudaGetLastError());
  return INQB_OK;
}

}  // namespace

size_t checkpoint_staging_bytes(long N, int M) {
  const size_t per = (size_t)N * sizeof(double2);
  const size_t mc = std::max<size_t>(1, std::min<size_t>((size_t)M, kChunkBytes / per));
  return mc * per;
}

int save_states(int precision, const std::string& dir, int kpin, const void* psi, long ld, int M, long N,
                int first_state, const double* occ, void* staging, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const std::string kdir = dir + "/kpin" + num_to_str(kpin);
  std::string err = make_dirs(kdir + "/states");
  if (err.empty() && occ) err = make_dirs(kdir + "/occupations");
  if (!err.empty()) return fail(INQB_ERR_IO, err);
  const size_t per = (size_t)N * sizeof(double2);
  const int mc = (int)(checkpoint_staging_bytes(N, M) / per);
  PinnedPair host;
  for (int b = 0; b < 2; b++) INQB_CUDA_TRY(cudaHostAlloc(&host.h[b], (size_t)mc * per, cudaHostAllocDefault));
  std::vector<std::future<std::string>> pending[2];
  auto drain = [&](int b) {
    std::string e;
    for (auto& f : pending[b]) {
      const std::string r = f.get();
      if (e.empty()) e = r;
    }
    pending[b].clear();
    return e;
  };
  int chunk = 0;
  for (int m0 = 0; m0 < M; m0 += mc, chunk++) {
    const int n = std::min(mc, M - m0);
    const int b = chunk & 1;
    err = drain(b);
    if (!err.empty()) break;
    double2* dst = static_cast<double2*>(staging);
    INQB_TRY(precision == INQB_FP64 ? launch_gather<double>(psi, ld, m0, n, N, dst, st)
                                    : launch_gather<float>(psi, ld, m0, n, N, dst, st));
    INQB_CUDA_TRY(cudaMemcpyAsync(host.h[b], dst, (size_t)n * per, cudaMemcpyDeviceToHost, st));
    INQB_CUDA_TRY(cudaStreamSynchronize(st));
    for (int j = 0; j < n; j++) {
      const char* src = static_cast<const char*>(host.h[b]) + (size_t)j * per;
      const std::string path = state_file(dir, kpin, (long)first_state + m0 + j);
      pending[b].push_back(std::async(std::launch::async, [path, src, per] { return write_file(path, src, per, 0, true); }));
    }
  }
  for (int b = 0; b < 2; b++) {
    const std::string e = drain(b);
    if (err.empty()) err = e;
  }
  if (err.empty() && occ)
    err = write_file(kdir + "/occupations/array", occ, sizeof(double) * (size_t)M, sizeof(double) * (size_t)first_state,
                     false);
  if (!err.empty()) return fail(INQB_ERR_IO, err);
  return INQB_OK;
}

int load_states(int precision, const std::string& dir, int kpin, void* psi, long ld, int M, long N, int first_state,
                double* occ, void* staging, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const std::string kdir = dir + "/kpin" + num_to_str(kpin);
  const size_t per = (size_t)N * sizeof(double2);
  const int mc = (int)(checkpoint_staging_bytes(N, M) / per);
  PinnedPair host;
  INQB_CUDA_TRY(cudaHostAlloc(&host.h[0], (size_t)mc * per, cudaHostAllocDefault));
  for (int m0 = 0; m0 < M; m0 += mc) {
    const int n = std::min(mc, M - m0);
    std::vector<std::future<std::string>> reads;
    for (int j = 0; j < n; j++) {
      char* dst = static_cast<char*>(host.h[0]) + (size_t)j * per;
      const std::string path = state_file(dir, kpin, (long)first_state + m0 + j);
      reads.push_back(std::async(std::launch::async, [path, dst, per] { return read_file(path, dst, per, 0); }));
    }
    std::string err;
    for (auto& f : reads) {
      const std::string r = f.get();
      if (err.empty()) err = r;
    }
    if (!err.empty()) return fail(INQB_ERR_IO, err);
    double2* src = static_cast<double2*>(staging);
    INQB_CUDA_TRY(cudaMemcpyAsync(src, host.h[0], (size_t)n * per, cudaMemcpyHostToDevice, st));
    INQB_TRY(precision == INQB_FP64 ? launch_scatter<double>(src, n, N, psi, ld, m0, st)
                                    : launch_scatter<float>(src, n, N, psi, ld, m0, st));
    // the host buffer is refilled by the next chunk's reads
    INQB_CUDA_TRY(cudaStreamSynchronize(st));
  }
  if (occ) {
    const std::string err = read_file(kdir + "/occupations/array", occ, sizeof(double) * (size_t)M,
                                      sizeof(double) * (size_t)first_state);
    if (!err.empty()) return fail(INQB_ERR_IO, err);
  }
  return INQB_OK;
}

int save_density(const std::string& dir, const double* rho, long N, void* stream) {
  const std::string d = dir + "/spin_density";
  std::string err = make_dirs(d);
  if (!err.empty()) return fail(INQB_ERR_IO, err);
  std::vector<double> h((size_t)N);
  INQB_CUDA_TRY(cudaMemcpyAsync(h.data(), rho, sizeof(double) * N, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
  INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  err = write_file(d + "/" + num_to_str(0), h.data(), sizeof(double) * N, 0, true);
  if (!err.empty()) return fail(INQB_ERR_IO, err);
  return INQB_OK;
}

int load_density(const std::string& dir, double* rho, long N, void* stream) {
  std::vector<double> h((size_t)N);
  const std::string err = read_file(dir + "/spin_density/" + num_to_str(0), h.data(), sizeof(double) * N, 0);
  if (!err.empty()) return fail(INQB_ERR_IO, err);
  INQB_CUDA_TRY(cudaMemcpyAsync(rho, h.data(), sizeof(double) * N, cudaMemcpyHostToDevice, (cudaStream_t)stream));
  INQB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return INQB_OK;
}

}  // namespace inqb
