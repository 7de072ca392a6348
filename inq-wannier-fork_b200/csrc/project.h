// The KB projection kernels (project.cu): proj[a][l][m] for every atom and orbital,
// from per-atom chunks of sphere entries.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace inqb {

constexpr int kProjChunk = 32;  // sphere entries per chunk (one K block of the contraction)
constexpr int kProjOrbTC = 64;  // orbitals per CTA of the tensor-core kernel

// bytes of the coefficient table of nchunks chunks in the context precision
size_t project_table_bytes(int precision, int nchunks);
// rebuild the coefficient table for covariant k + A (after every phase change)
int launch_project_table(int precision, int nchunks, const float* relpos, const double* beta, const double kA[3],
                         void* table, void* stream);
// whether an orbital block can use the projection kernel (16-byte gathers)
bool project_supported(int precision, const void* in, long ld);
// proj[a][l][m] = scale[a][l] sum_s B[a][l][s] psi[pt(a, s)][m], written (no accumulation);
// err (device int) is set if a device-side wait gave up
int launch_project(int precision, const void* in, long ld, int M, int nproj, int L, const int* pc_ptr,
                   const int* pc_pt, const void* table, const double* scale, double2* proj, int* err, void* stream);

}  // namespace inqb
