// Complex arithmetic and fully unrolled in-register DFTs for the plane/line FFT
// kernels.  Forward transforms use exp(-2 pi i / R) (FFTW sign -1, the sign of
// INQ's to_fourier); inverse transforms use exp(+2 pi i / R) and are unscaled.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>
#include <utility>

#include "twiddles.cuh"

namespace inqb {

template <typename T>
struct alignas(2 * sizeof(T)) cplx {
  T x, y;
};

template <typename T>
__host__ __device__ __forceinline__ cplx<T> mk(T a, T b) {
  return cplx<T>{a, b};
}
template <typename T>
__device__ __forceinline__ cplx<T> operator+(cplx<T> a, cplx<T> b) {
  return {a.x + b.x, a.y + b.y};
}
template <typename T>
__device__ __forceinline__ cplx<T> operator-(cplx<T> a, cplx<T> b) {
  return {a.x - b.x, a.y - b.y};
}
template <typename T>
__device__ __forceinline__ cplx<T> operator*(cplx<T> a, cplx<T> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ cplx<T> operator*(T s, cplx<T> a) {
  return {s * a.x, s * a.y};
}
template <typename T>
__device__ __forceinline__ cplx<T> conj(cplx<T> a) {
  return {a.x, -a.y};
}
// a * conj(b)
template <typename T>
__device__ __forceinline__ cplx<T> mul_conj(cplx<T> a, cplx<T> b) {
  return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
// acc += a * b
template <typename T>
__device__ __forceinline__ void fma_acc(cplx<T>& acc, cplx<T> a, cplx<T> b) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
// multiply by +i / -i
template <typename T>
__device__ __forceinline__ cplx<T> mul_i(cplx<T> a) {
  return {-a.y, a.x};
}
template <typename T>
__device__ __forceinline__ cplx<T> mul_mi(cplx<T> a) {
  return {a.y, -a.x};
}

// Compile-time loop: f(std::integral_constant<int, I>{}) for I in [0, N).
template <typename F, int... Is>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// a * exp(-+ 2 pi i K / R) with K, R compile time (forward: minus sign).
template <int R, int K, bool INV, typename T>
__device__ __forceinline__ cplx<T> rot(cplx<T> a) {
  constexpr int k = K % R;
  if constexpr (k == 0) {
    return a;
  } else if constexpr (2 * k == R) {
    return {-a.x, -a.y};
  } else if constexpr (4 * k == R) {
    return INV ? mul_i(a) : mul_mi(a);
  } else if constexpr (4 * k == 3 * R) {
    return INV ? mul_mi(a) : mul_i(a);
  } else {
    constexpr T c = (T)RootsOfUnity<R>::re[k];
    constexpr T s = (T)(INV ? RootsOfUnity<R>::im[k] : -RootsOfUnity<R>::im[k]);
    return {a.x * c - a.y * s, a.x * s + a.y * c};
  }
}

constexpr int first_factor(int r) {
  return (r % 4 == 0 && r != 8) ? 4 : (r % 2 == 0) ? 2 : (r % 3 == 0) ? 3 : (r % 5 == 0) ? 5 : r;
}

// In-place DFT of R values held in registers, natural order in and out.
template <int R, bool INV, typename T>
struct DFT {
  static_assert(first_factor(R) != R, "prime radix without a specialisation");
  static constexpr int A = first_factor(R);
  static constexpr int B = R / A;
  __device__ __forceinline__ static void run(cplx<T>* v) {
    // n = b + B a ; k = k1 + A k2 (four-step inside the registers)
    cplx<T> y[R];
    static_for<B>([&](auto bI) {
      constexpr int b = decltype(bI)::value;
      cplx<T> u[A];
#pragma unroll
      for (int a = 0; a < A; ++a) u[a] = v[b + B * a];
      DFT<A, INV, T>::run(u);
      static_for<A>([&](auto kI) {
        constexpr int k1 = decltype(kI)::value;
        y[b * A + k1] = rot<R, b * k1, INV>(u[k1]);
      });
    });
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      cplx<T> w[B];
#pragma unroll
      for (int b = 0; b < B; ++b) w[b] = y[b * A + k1];
      DFT<B, INV, T>::run(w);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = w[k2];
    }
  }
};

template <bool INV, typename T>
struct DFT<1, INV, T> {
  __device__ __forceinline__ static void run(cplx<T>*) {}
};

template <bool INV, typename T>
struct DFT<2, INV, T> {
  __device__ __forceinline__ static void run(cplx<T>* v) {
    cplx<T> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  }
};

template <bool INV, typename T>
struct DFT<3, INV, T> {
  __device__ __forceinline__ static void run(cplx<T>* v) {
    constexpr T c = (T)-0.5;
    constexpr T s = (T)(INV ? 0.8660254037844386 : -0.8660254037844386);  // sin(+-2 pi / 3)
    cplx<T> a = v[1] + v[2], d = v[1] - v[2];
    cplx<T> m = {v[0].x + c * a.x, v[0].y + c * a.y};
    cplx<T> r = {-s * d.y, s * d.x};  // i s d
    v[0] = v[0] + a;
    v[1] = m + r;
    v[2] = m - r;
  }
};

template <bool INV, typename T>
struct DFT<4, INV, T> {
  __device__ __forceinline__ static void run(cplx<T>* v) {
    cplx<T> t0 = v[0] + v[2], t1 = v[0] - v[2], t2 = v[1] + v[3], t3 = v[1] - v[3];
    cplx<T> r = INV ? mul_i(t3) : mul_mi(t3);
    v[0] = t0 + t2;
    v[2] = t0 - t2;
    v[1] = t1 + r;
    v[3] = t1 - r;
  }
};

template <bool INV, typename T>
struct DFT<5, INV, T> {
  __device__ __forceinline__ static void run(cplx<T>* v) {
    constexpr T c1 = (T)0.30901699437494745;   // cos(2 pi / 5)
    constexpr T c2 = (T)-0.80901699437494734;  // cos(4 pi / 5)
    constexpr T s1 = (T)(INV ? 0.95105651629515353 : -0.95105651629515353);
    constexpr T s2 = (T)(INV ? 0.58778525229247314 : -0.58778525229247314);
    cplx<T> a1 = v[1] + v[4], b1 = v[1] - v[4], a2 = v[2] + v[3], b2 = v[2] - v[3];
    cplx<T> m1 = {v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y};
    cplx<T> m2 = {v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y};
    // n1 = i (s1 b1 + s2 b2), n2 = i (s2 b1 - s1 b2)
    cplx<T> n1 = {-(s1 * b1.y + s2 * b2.y), s1 * b1.x + s2 * b2.x};
    cplx<T> n2 = {-(s2 * b1.y - s1 * b2.y), s2 * b1.x - s1 * b2.x};
    v[0] = v[0] + a1 + a2;
    v[1] = m1 + n1;
    v[4] = m1 - n1;
    v[2] = m2 + n2;
    v[3] = m2 - n2;
  }
};

// ---------------------------------------------------------------- radix 8, complex64
// Sum and difference of two complex64 values, each as one packed f32x2 instruction
// (sm_100; round to nearest like the scalar adds, so every value is rounded once, as
// in the scalar form).
__device__ __forceinline__ cplx<float> padd(cplx<float> a, cplx<float> b) {
  const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  return {r.x, r.y};
}
__device__ __forceinline__ cplx<float> psub(cplx<float> a, cplx<float> b) {
  unsigned long long r;
  asm("{\n\t.reg .b64 pa, pb;\n\tmov.b64 pa, {%1, %2};\n\tmov.b64 pb, {%3, %4};\n\t"
      "sub.rn.f32x2 %0, pa, pb;\n\t}"
      : "=l"(r)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return {v.x, v.y};
}
__device__ __forceinline__ cplx<float> pscale(float s, cplx<float> a) {
  const float2 r = __fmul2_rn(make_float2(s, s), make_float2(a.x, a.y));
  return {r.x, r.y};
}

// DFT_8 of complex64 values written out as the split 8 = 2 x 4 (the generic form
// above with the same factors): a_n = v_n + v_{n+4} gives the even outputs as a DFT_4,
// b_n = v_n - v_{n+4} twiddled by w^n the odd ones, w = exp(-+ 2 pi i / 8).  Sums
// and differences of values in natural (re, im) order take one packed instruction;
// those with a factor +-i stay two scalar adds (the swap is free there).
template <bool INV>
struct DFT<8, INV, float> {
  __device__ __forceinline__ static void run(cplx<float>* v) {
    constexpr float h = 0.70710678118654752f;  // 1/sqrt(2)
    cplx<float> a[4], b[4];
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      a[n] = padd(v[n], v[n + 4]);
      b[n] = psub(v[n], v[n + 4]);
    }
    // even outputs: DFT_4 of a
    const cplx<float> t0 = padd(a[0], a[2]), t1 = psub(a[0], a[2]);
    const cplx<float> t2 = padd(a[1], a[3]), t3 = psub(a[1], a[3]);
    v[0] = padd(t0, t2);
    v[4] = psub(t0, t2);
    // X2 = t1 -+ i t3, X6 = t1 +- i t3 (upper signs forward)
    if (INV) {
      v[2] = {t1.x - t3.y, t1.y + t3.x};
      v[6] = {t1.x + t3.y, t1.y - t3.x};
    } else {
      v[2] = {t1.x + t3.y, t1.y - t3.x};
      v[6] = {t1.x - t3.y, t1.y + t3.x};
    }
    // odd outputs: DFT_4 of c_n = b_n w^n.  e = c0 + c2, f = c0 - c2 (c2 = -+ i b2);
    // p1 sqrt(1/2) = c1 and p3 sqrt(1/2) = c3, so s = c1 + c3, d = c1 - c3.
    cplx<float> e, f, p1, p3;
    if (INV) {
      e = {b[0].x - b[2].y, b[0].y + b[2].x};
      f = {b[0].x + b[2].y, b[0].y - b[2].x};
      p1 = {b[1].x - b[1].y, b[1].x + b[1].y};      // b1 (1 + i)
      p3 = {-b[3].x - b[3].y, b[3].x - b[3].y};     // b3 (-1 + i)
    } else {
      e = {b[0].x + b[2].y, b[0].y - b[2].x};
      f = {b[0].x - b[2].y, b[0].y + b[2].x};
      p1 = {b[1].x + b[1].y, b[1].y - b[1].x};      // b1 (1 - i)
      p3 = {b[3].y - b[3].x, -b[3].x - b[3].y};     // b3 (-1 - i)
    }
    const cplx<float> s = pscale(h, padd(p1, p3)), d = pscale(h, psub(p1, p3));
    v[1] = padd(e, s);
    v[5] = psub(e, s);
    // X3 = f -+ i d, X7 = f +- i d
    if (INV) {
      v[3] = {f.x - d.y, f.y + d.x};
      v[7] = {f.x + d.y, f.y - d.x};
    } else {
      v[3] = {f.x + d.y, f.y - d.x};
      v[7] = {f.x - d.y, f.y + d.x};
    }
  }
};

}  // namespace inqb
