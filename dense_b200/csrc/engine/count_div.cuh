// Correctly rounded division by a divisor known ahead of its uses.
//
// DENSE divides in the working precision: neighbour sums by their count
// (determ.hpp:81-89) and concentrations by critical values that are constant
// for a parameter set (her_model_2014's rates, model_impl.hpp:193-224).  The
// engines must return exactly the IEEE round-to-nearest quotient RN(x/c).
// For a divisor c > 0 with rc = RN(1/c) precomputed this computes
//
//   q0 = RN(x * rc),   r0 = x - q0*c (one FMA),   q1 = RN(q0 + r0*rc),
//
// Markstein's refinement of a quotient by one FMA step (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000
// processor", IBM J. Res. Dev. 34(1), 1990), and then proves q1 = RN(x/c)
// with the remainder r1 = RN(x - q1*c) (one FMA): q1 is the correctly
// rounded quotient when x/c lies strictly inside q1's rounding interval,
// i.e. |x - q1*c| < h*c with h half the gap between q1 and its neighbours.
// For a q1 that is not a power of two, h = p * 2^-(m+1) where p = 2^e is
// q1's leading power of two (its exponent bits alone) and m the mantissa
// width, so h*c = p * cg with cg = c * 2^-(m+1), an exact product while it
// stays in the normal range.  The test |r1| < p * cg is sound even when r1
// is rounded: rounding is monotone and p * cg is representable, so |r1| <
// p * cg implies |x - q1*c| < p * cg.  Whenever the proof does not go
// through (q1 a power of two, zero, subnormal, inf or NaN; p * cg not
// normal; a tie; a refinement that missed) the plain division x / c is
// returned instead, so the result always equals x / c.  A divisor outside
// [2^-900, 2^900] (2^-100, 2^100 in FP32), or not positive, gets rc = cg =
// 0, which makes the proof fail and every quotient take the division.
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

template <typename T>
struct DivConst;

template <>
struct DivConst<double> {
  static constexpr double kGap = 0x1p-53;       // 2^-(m+1)
  static constexpr double kLo = 0x1p-900, kHi = 0x1p+900;
  static constexpr double kMinNormal = 0x1p-1022;
  static constexpr uint64_t kExp = 0x7FF0000000000000ull, kMant = 0x000FFFFFFFFFFFFFull;
};

template <>
struct DivConst<float> {
  static constexpr float kGap = 0x1p-24f;
  static constexpr float kLo = 0x1p-100f, kHi = 0x1p+100f;
  static constexpr float kMinNormal = 0x1p-126f;
  static constexpr uint32_t kExp = 0x7F800000u, kMant = 0x007FFFFFu;
};

// q = x / c proven correctly rounded without the division; false when the
// proof does not go through (q is then undefined).  rc = RN(1/c), cg = c *
// 2^-(m+1); see above.
template <typename T>
DENSE_HD inline bool div_proved_try(T x, T c, T rc, T cg, T& q) {
  using Tr = CountDivTraits<T>;
  using K = DivConst<T>;
  const T q0 = x * rc;
  const T r0 = cd_fma(-q0, c, x);
  const T q1 = cd_fma(r0, rc, q0);
  const T r1 = cd_fma(-q1, c, x);
  const typename Tr::Bits b = Tr::bits(q1);
  const T lim = Tr::from(b & K::kExp) * cg;  // h * c
  q = q1;
  return (b & K::kMant) != 0 && cd_abs(r1) < lim && lim > K::kMinNormal;
}

// x / c for c > 0 with rc = RN(1/c) and cg = c * 2^-(m+1) (both 0 when c is
// outside the quick range); always equal to x / c.
template <typename T>
DENSE_HD inline T div_proved(T x, T c, T rc, T cg) {
  T q;
  if (div_proved_try(x, c, rc, cg, q)) return q;
  return x / c;
}

// rc and cg of a divisor, or zeros when c is outside the quick range.
template <typename T>
DENSE_HD inline void quick_divisor(T c, T& rc, T& cg) {
  using K = DivConst<T>;
  if (c >= K::kLo && c <= K::kHi) {
    rc = T(1) / c;
    cg = c * K::kGap;
  } else {
    rc = T(0);
    cg = T(0);
  }
}

// x / c for an integer-valued count c >= 1, with rc = RN(1/c).
template <typename T>
DENSE_HD inline T div_by_count(T x, T c, T rc) {
  return div_proved(x, c, rc, c * DivConst<T>::kGap);
}

}  // namespace dense_b200
