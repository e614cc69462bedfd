// Division of a sum by a small neighbour count, correctly rounded.
//
// DENSE averages neighbour concentrations as sum / count in the working
// precision (determ.hpp:81-89).  The engines must return exactly that
// IEEE round-to-nearest quotient.  For a count c with rc = RN(1/c) this
// computes
//
//   q0 = RN(x * rc),   r0 = x - q0*c (one FMA),   q1 = RN(q0 + r0*rc),
//
// Markstein's refinement of a quotient by one FMA step (P. Markstein, "Computation
// of elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990), and then proves q1 = RN(x/c) with the exact remainder
// r1 = x - q1*c: q1 is the correctly rounded quotient exactly when x/c lies
// strictly inside q1's rounding interval, i.e. |r1| < c * (half the gap to
// q1's neighbour on r1's side).  The remainder of a quotient within a few
// ulps of x/c is a small multiple of ulp(q1) and so exactly representable,
// and c times a power of two is exact.  Whenever the proof does not go
// through (a tie, an operand outside the normal range, zero, inf, NaN) the
// plain division x / c is returned instead, so the result always equals
// x / c.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define DENSE_HD __host__ __device__
#else
#define DENSE_HD
#endif

namespace dense_b200 {

template <typename T>
struct CountDivTraits;

template <>
struct CountDivTraits<double> {
  using Bits = uint64_t;
  static constexpr int kMant = 52;
  static constexpr double kLo = 0x1p-900, kHi = 0x1p+900;
  static DENSE_HD inline Bits bits(double x) {
#if defined(__CUDA_ARCH__)
    return static_cast<Bits>(__double_as_longlong(x));
#else
    Bits b;
    std::memcpy(&b, &x, sizeof b);
    return b;
#endif
  }
  static DENSE_HD inline double from(Bits b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double(static_cast<long long>(b));
#else
    double x;
    std::memcpy(&x, &b, sizeof x);
    return x;
#endif
  }
};

template <>
struct CountDivTraits<float> {
  using Bits = uint32_t;
  static constexpr int kMant = 23;
  static constexpr float kLo = 0x1p-100f, kHi = 0x1p+100f;
  static DENSE_HD inline Bits bits(float x) {
#if defined(__CUDA_ARCH__)
    return static_cast<Bits>(__float_as_uint(x));
#else
    Bits b;
    std::memcpy(&b, &x, sizeof b);
    return b;
#endif
  }
  static DENSE_HD inline float from(Bits b) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(b);
#else
    float x;
    std::memcpy(&x, &b, sizeof x);
    return x;
#endif
  }
};

template <typename T>
DENSE_HD inline T cd_fma(T a, T b, T c) {
#if defined(__CUDA_ARCH__)
  return fma(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}

template <typename T>
DENSE_HD inline T cd_abs(T a) {
#if defined(__CUDA_ARCH__)
  return fabs(a);
#else
  return std::fabs(a);
#endif
}

// x / c for an integer-valued c >= 1, with rc = RN(1/c); see above.
template <typename T>
DENSE_HD inline T div_by_count(T x, T c, T rc) {
  using Tr = CountDivTraits<T>;
  using Bits = typename Tr::Bits;
  const T ax = cd_abs(x);
  if (ax >= Tr::kLo && ax <= Tr::kHi) {
    const T q0 = x * rc;
    const T r0 = cd_fma(-q0, c, x);
    const T q1 = cd_fma(r0, rc, q0);
    const T r1 = cd_fma(-q1, c, x);  // exact
    const Bits b = Tr::bits(q1);
    const Bits expo = (b >> Tr::kMant) & ((Bits(1) << (sizeof(T) * 8 - 1 - Tr::kMant)) - 1);
    const bool pow2 = (b & ((Bits(1) << Tr::kMant) - 1)) == 0;
    // half the gap to the neighbour away from zero: 2^(e - kMant - 1), as a
    // biased exponent expo - kMant - 1; towards zero it halves again when
    // |q1| is a power of two
    const T up = Tr::from((expo - Tr::kMant - 1) << Tr::kMant);
    const T down = pow2 ? up * T(0.5) : up;
    const bool away = (r1 > T(0)) == (q1 > T(0));
    if (cd_abs(r1) < (away ? up : down) * c) return q1;
  }
  return x / c;
}

}  // namespace dense_b200
