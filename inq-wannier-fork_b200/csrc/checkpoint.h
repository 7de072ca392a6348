// Checkpoint files in INQ's restart layout (checkpoint.cu).
#pragma once

#include <cstddef>
#include <string>

namespace inqb {

// Device staging a save or load of M states of N points uses (complex128 rows).
size_t checkpoint_staging_bytes(long N, int M);
// dir is the electrons directory; states first_state .. first_state + M - 1 of k-point
// block kpin.  occ (host, may be null) is written to / read from the occupations array.
int save_states(int precision, const std::string& dir, int kpin, const void* psi, long ld, int M, long N,
                int first_state, const double* occ, void* staging, void* stream);
int load_states(int precision, const std::string& dir, int kpin, void* psi, long ld, int M, long N, int first_state,
                double* occ, void* staging, void* stream);
int save_density(const std::string& dir, const double* rho, long N, void* stream);
int load_density(const std::string& dir, double* rho, long N, void* stream);

}  // namespace inqb
