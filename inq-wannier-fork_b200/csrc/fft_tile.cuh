// Shared-memory tile FFTs: one axis of a tile of lines, transformed in place by
// the four-step factorisation N = N1 * N2 with one smem round trip per step.
//
// Element n = j2 + N2 j1 of a line lives at slot(j1, j2) = j1 (N2 + PAD) + j2
// (times the element stride of the line).  PAD = 1 for even N2 makes both the
// column walk of step 1 and the row walk of step 2 bank-conflict free.
//
//   forward  step 1: thread j2 : DFT_N1 over j1, twiddle w_N^{j2 k1}, same slots
//   forward  step 2: thread k1 : DFT_N2 over j2, same slots
//     -> slot(k1, k2) holds X[k1 + N1 k2]        ("transposed" order)
//   inverse from transposed (step 2' then step 1'): exact reverse, natural out
//   inverse from natural: the forward steps with conjugate roots -> transposed
//
// Every thread writes only the slots it read, so no barrier is needed inside a
// step; the caller puts __syncthreads() between steps.
#pragma once

#include "dft.cuh"

namespace inqb {

// PAD_ < 0 selects the default: pad rows of even N2 by one slot.
template <int N1_, int N2_, int PAD_ = -1>
struct Axis {
  static constexpr int N1 = N1_;
  static constexpr int N2 = N2_;
  static constexpr int N = N1 * N2;
  static constexpr int PAD = PAD_ >= 0 ? PAD_ : ((N2 % 2 == 0 && N2 > 1) ? 1 : 0);
  static constexpr int ROW = N2 + PAD;
  static constexpr int SLOTS = N1 * ROW;  // slots used by one padded line
  // slot of row j1, column j2 of the N1 x N2 four-step view
  __host__ __device__ static constexpr int at(int j1, int j2) { return j1 * ROW + j2; }
  // slot of natural element n
  __host__ __device__ static constexpr int slot(int n) { return at(n / N2, n % N2); }
  // slot holding frequency k after a forward (or inverse-from-natural) transform
  __host__ __device__ static constexpr int slot_of_freq(int k) { return at(k % N1, k / N1); }
};

// Twiddle table layout in shared memory: tw[k1 * N2 + j2] = exp(-2 pi i j2 k1 / N).
template <typename A, bool INV, typename T>
__device__ __forceinline__ cplx<T> twiddle(cplx<T> v, const cplx<T>* tw, int k1, int j2) {
  cplx<T> w = tw[k1 * A::N2 + j2];
  return INV ? mul_conj(v, w) : v * w;
}

// Step 1 (forward or inverse-from-natural when INV): items map to (base, es, j2).
template <typename A, bool INV, typename T, typename Map>
__device__ __forceinline__ void step1(cplx<T>* S, int nitems, const cplx<T>* tw, Map map) {
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    int base, es, j2;
    map(it, base, es, j2);
    cplx<T> v[A::N1];
#pragma unroll
    for (int j1 = 0; j1 < A::N1; ++j1) v[j1] = S[base + A::at(j1, j2) * es];
    DFT<A::N1, INV, T>::run(v);
    if (A::N2 > 1) {
#pragma unroll
      for (int k1 = 1; k1 < A::N1; ++k1) v[k1] = twiddle<A, INV>(v[k1], tw, k1, j2);
    }
#pragma unroll
    for (int k1 = 0; k1 < A::N1; ++k1) S[base + A::at(k1, j2) * es] = v[k1];
  }
}

// Step 2 (forward / inverse-from-natural): items map to (base, es, k1).
template <typename A, bool INV, typename T, typename Map>
__device__ __forceinline__ void step2(cplx<T>* S, int nitems, Map map) {
  if (A::N2 == 1) return;
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    int base, es, k1;
    map(it, base, es, k1);
    cplx<T> v[A::N2];
#pragma unroll
    for (int j2 = 0; j2 < A::N2; ++j2) v[j2] = S[base + A::at(k1, j2) * es];
    DFT<A::N2, INV, T>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < A::N2; ++k2) S[base + A::at(k1, k2) * es] = v[k2];
  }
}

// Step 2' of the inverse from transposed order: inverse DFT_N2 over k2 then the
// conjugate twiddle; `pre` is applied to the frequency-domain values first
// (pre(k, value) with k = k1 + N1 k2), which fuses a pointwise operator.
template <typename A, typename T, typename Map, typename Pre>
__device__ __forceinline__ void step2_inv_transposed(cplx<T>* S, int nitems, const cplx<T>* tw, Map map,
                                                     Pre pre) {
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    int base, es, k1;
    map(it, base, es, k1);
    cplx<T> v[A::N2];
#pragma unroll
    for (int k2 = 0; k2 < A::N2; ++k2) v[k2] = pre(it, k1 + A::N1 * k2, S[base + A::at(k1, k2) * es]);
    DFT<A::N2, true, T>::run(v);
    if (A::N2 > 1) {
#pragma unroll
      for (int j2 = 0; j2 < A::N2; ++j2)
        if (k1 > 0) v[j2] = twiddle<A, true>(v[j2], tw, k1, j2);
    }
#pragma unroll
    for (int j2 = 0; j2 < A::N2; ++j2) S[base + A::at(k1, j2) * es] = v[j2];
  }
}

// Forward step 2 fused with a pointwise operator and the inverse step 2'
// (the kinetic multiply of H between a forward and an inverse transform).
template <typename A, typename T, typename Map, typename Op>
__device__ __forceinline__ void step2_fwd_op_inv(cplx<T>* S, int nitems, const cplx<T>* tw, Map map, Op op) {
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    int base, es, k1;
    map(it, base, es, k1);
    cplx<T> v[A::N2];
#pragma unroll
    for (int j2 = 0; j2 < A::N2; ++j2) v[j2] = S[base + A::at(k1, j2) * es];
    DFT<A::N2, false, T>::run(v);
#pragma unroll
    for (int k2 = 0; k2 < A::N2; ++k2) v[k2] = op(it, k1 + A::N1 * k2, v[k2]);
    DFT<A::N2, true, T>::run(v);
    if (A::N2 > 1) {
#pragma unroll
      for (int j2 = 0; j2 < A::N2; ++j2)
        if (k1 > 0) v[j2] = twiddle<A, true>(v[j2], tw, k1, j2);
    }
#pragma unroll
    for (int j2 = 0; j2 < A::N2; ++j2) S[base + A::at(k1, j2) * es] = v[j2];
  }
}

// Step 1' of the inverse from transposed order: inverse DFT_N1 over k1, natural out.
template <typename A, typename T, typename Map>
__device__ __forceinline__ void step1_inv_transposed(cplx<T>* S, int nitems, Map map) {
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    int base, es, j2;
    map(it, base, es, j2);
    cplx<T> v[A::N1];
#pragma unroll
    for (int k1 = 0; k1 < A::N1; ++k1) v[k1] = S[base + A::at(k1, j2) * es];
    DFT<A::N1, true, T>::run(v);
#pragma unroll
    for (int j1 = 0; j1 < A::N1; ++j1) S[base + A::at(j1, j2) * es] = v[j1];
  }
}

}  // namespace inqb
