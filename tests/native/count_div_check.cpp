// Checks the engines' correctly rounded divisions against the plain IEEE
// division on the host: div_by_count (neighbour sums by their count) and
// div_proved (quotients by a divisor with a precomputed reciprocal, such as
// a parameter set's critical values), on random operands of every
// magnitude, concentration-like values, exact multiples, near-ties and the
// edge cases.  Prints "<name> <cases> <quick-path fraction>" per check;
// exit 1 on any mismatch.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>

#include "count_div.cuh"

using dense_b200::CountDivTraits;
using dense_b200::div_by_count;
using dense_b200::div_proved;
using dense_b200::div_proved_try;
using dense_b200::quick_divisor;

template <typename T>
static bool same(T a, T b) {
  if (std::isnan(a) && std::isnan(b)) return true;
  return std::memcmp(&a, &b, sizeof a) == 0;
}

template <typename T>
static T random_bits(std::mt19937_64& g) {
  typename CountDivTraits<T>::Bits b;
  uint64_t r = g();
  std::memcpy(&b, &r, sizeof b);
  return CountDivTraits<T>::from(b);
}

struct Tally {
  long cases = 0, quick = 0, bad = 0;
};

// one quotient: the result must equal x / c bit for bit
template <typename T>
static void check(const char* name, T x, T c, T rc, T cg, Tally& t) {
  const T got = div_proved(x, c, rc, cg), want = x / c;
  T q;
  ++t.cases;
  t.quick += div_proved_try(x, c, rc, cg, q);
  if (!same(got, want) && ++t.bad < 10)
    std::printf("mismatch %s x=%a c=%a got=%a want=%a\n", name, (double)x, (double)c, (double)got, (double)want);
}

template <typename T>
static int run_counts(const char* name, uint64_t seed, int n) {
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  Tally t;
  auto one = [&](T x, int ci) {
    const T c = static_cast<T>(ci), rc = T(1) / c;
    const T got = div_by_count(x, c, rc), want = x / c;
    ++t.cases;
    if (!same(got, want) && ++t.bad < 10)
      std::printf("mismatch %s x=%a c=%d got=%a want=%a\n", name, (double)x, ci, (double)got, (double)want);
  };
  const T specials[] = {T(0), -T(0), std::numeric_limits<T>::infinity(), -std::numeric_limits<T>::infinity(),
                        std::numeric_limits<T>::quiet_NaN(), std::numeric_limits<T>::denorm_min(),
                        std::numeric_limits<T>::min(), std::numeric_limits<T>::max(), T(1), T(3), T(5), T(6)};
  for (T x : specials)
    for (int c = 0; c <= 8; ++c) one(x, c);
  for (int i = 0; i < n; ++i) {
    const int c = 1 + static_cast<int>(g() % 8);
    one(random_bits<T>(g), c);
    // sums of c concentration-like values
    T s = T(0);
    for (int k = 0; k < c; ++k) s += static_cast<T>(std::ldexp(u(g), static_cast<int>(g() % 40) - 20));
    one(s, c);
    // exact multiples and their neighbours
    const T m = static_cast<T>(std::ldexp(std::floor(u(g) * 1e6), static_cast<int>(g() % 20) - 10));
    one(m * static_cast<T>(c), c);
    one(std::nextafter(m * static_cast<T>(c), T(0)), c);
  }
  // how often the refined quotient is accepted without the division
  // (counts 3..6, concentration-like operands)
  long quick = 0;
  for (int i = 0; i < 200000; ++i) {
    const T c = static_cast<T>(3 + static_cast<int>(g() % 4)), rc = T(1) / c;
    T q;
    quick += div_proved_try(static_cast<T>(u(g) * 10.0 + 0.001), c, rc, c * dense_b200::DivConst<T>::kGap, q);
  }
  std::printf("%s %ld %.4f\n", name, t.cases, quick / 200000.0);
  return t.bad == 0 ? 0 : 1;
}

template <typename T>
static int run_divisors(const char* name, uint64_t seed, int n) {
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  using K = dense_b200::DivConst<T>;
  const int span = std::is_same<T, double>::value ? 1000 : 120;  // exponents beyond the quick range too
  Tally t;
  auto with = [&](T x, T c) {
    T rc, cg;
    quick_divisor(c, rc, cg);
    check(name, x, c, rc, cg, t);
  };
  const T specials[] = {T(0), -T(0), std::numeric_limits<T>::infinity(), -std::numeric_limits<T>::infinity(),
                        std::numeric_limits<T>::quiet_NaN(), std::numeric_limits<T>::denorm_min(),
                        std::numeric_limits<T>::min(), std::numeric_limits<T>::max(), T(1), T(3), T(0.1)};
  const T divisors[] = {T(0.1), T(3), T(0.3), T(7.5), K::kLo, K::kHi, T(1), T(2), T(0.7) * K::kLo,
                        std::numeric_limits<T>::min(), std::numeric_limits<T>::max(), T(0), -T(2),
                        std::numeric_limits<T>::infinity(), std::numeric_limits<T>::quiet_NaN()};
  for (T x : specials)
    for (T c : divisors) with(x, c);
  for (int i = 0; i < n; ++i) {
    // divisors log-uniform over (and past) the quick range, and critical-value-like ones
    const T c_wide = static_cast<T>(std::ldexp(1.0 + u(g), static_cast<int>(g() % (2 * span)) - span));
    const T c_crit = static_cast<T>(std::exp(std::log(0.01) + u(g) * std::log(1e4)));
    for (T c : {c_wide, c_crit}) {
      with(random_bits<T>(g), c);
      with(static_cast<T>(std::ldexp(u(g), static_cast<int>(g() % 60) - 30)), c);
      // exact multiples of c and their neighbours (ties and near-ties of x / c)
      const T m = static_cast<T>(std::ldexp(std::floor(u(g) * 1e6) + 0.5, static_cast<int>(g() % 20) - 30));
      const T x = m * c;
      with(x, c);
      with(std::nextafter(x, T(0)), c);
      with(std::nextafter(x, std::numeric_limits<T>::infinity()), c);
    }
  }
  // how often the quick path is taken for critical-value-like divisors and
  // concentration-like operands
  long quick = 0;
  for (int i = 0; i < 200000; ++i) {
    const T c = static_cast<T>(std::exp(std::log(0.01) + u(g) * std::log(1e4)));
    T rc, cg, q;
    quick_divisor(c, rc, cg);
    quick += div_proved_try(static_cast<T>(std::ldexp(u(g) + 0.001, static_cast<int>(g() % 20) - 10)), c, rc, cg, q);
  }
  std::printf("%s %ld %.4f\n", name, t.cases, quick / 200000.0);
  return t.bad == 0 ? 0 : 1;
}

int main() {
  int rc = run_counts<double>("count_double", 1, 2000000);
  rc |= run_counts<float>("count_float", 2, 2000000);
  rc |= run_divisors<double>("divisor_double", 3, 1000000);
  rc |= run_divisors<float>("divisor_float", 4, 1000000);
  return rc;
}
