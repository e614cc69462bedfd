// Checks div_by_count against the plain IEEE division on the host: random
// operands of many magnitudes, neighbour-like sums, and the edge cases.
// Prints "<type> <cases> <fast-path fraction>" per type; exit 1 on any
// mismatch.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>

#include "count_div.cuh"

using dense_b200::div_by_count;

template <typename T>
static bool same(T a, T b) {
  if (std::isnan(a) && std::isnan(b)) return true;
  return std::memcmp(&a, &b, sizeof a) == 0;
}

template <typename T>
static int run(const char* name, uint64_t seed, int n) {
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  long cases = 0, fast = 0, bad = 0;
  auto check = [&](T x, int ci) {
    const T c = static_cast<T>(ci), rc = T(1) / c;
    const T got = div_by_count(x, c, rc), want = x / c;
    ++cases;
    const T q0 = x * rc;
    (void)q0;
    if (!same(got, want)) {
      if (++bad < 10) std::printf("mismatch %s x=%a c=%d got=%a want=%a\n", name, (double)x, ci, (double)got, (double)want);
    }
  };
  const T specials[] = {T(0), -T(0), std::numeric_limits<T>::infinity(), -std::numeric_limits<T>::infinity(),
                        std::numeric_limits<T>::quiet_NaN(), std::numeric_limits<T>::denorm_min(),
                        std::numeric_limits<T>::min(), std::numeric_limits<T>::max(), T(1), T(3), T(5), T(6)};
  for (T x : specials)
    for (int c = 0; c <= 8; ++c) check(x, c);
  for (int i = 0; i < n; ++i) {
    const int c = 1 + static_cast<int>(g() % 8);
    // random bit patterns (all magnitudes, both signs)
    typename dense_b200::CountDivTraits<T>::Bits b;
    uint64_t r = g();
    std::memcpy(&b, &r, sizeof b);
    T x = dense_b200::CountDivTraits<T>::from(b);
    check(x, c);
    // sums of c concentration-like values
    T s = T(0);
    for (int k = 0; k < c; ++k) s += static_cast<T>(std::ldexp(u(g), static_cast<int>(g() % 40) - 20));
    check(s, c);
    // exact multiples and near-ties
    const T m = static_cast<T>(std::ldexp(std::floor(u(g) * 1e6), static_cast<int>(g() % 20) - 10));
    check(m * static_cast<T>(c), c);
    check(std::nextafter(m * static_cast<T>(c), T(0)), c);
  }
  // how often the refined quotient is accepted without the division
  // (counts 3..6, concentration-like operands)
  for (int i = 0; i < 200000; ++i) {
    const int ci = 3 + static_cast<int>(g() % 4);
    const T c = static_cast<T>(ci), rc = T(1) / c;
    const T x = static_cast<T>(u(g) * 10.0 + 0.001);
    const T q0 = x * rc, r0 = std::fma(-q0, c, x), q1 = std::fma(r0, rc, q0), r1 = std::fma(-q1, c, x);
    // the acceptance test of div_by_count (q1 proven correctly rounded)
    int e;
    const T m = std::frexp(q1, &e);
    const T up = std::ldexp(T(1), e - std::numeric_limits<T>::digits - 1);
    const T down = (std::fabs(m) == T(0.5)) ? up * T(0.5) : up;
    const bool away = (r1 > T(0)) == (q1 > T(0));
    fast += std::fabs(r1) < (away ? up : down) * c;
  }
  std::printf("%s %ld %.4f\n", name, cases, fast / 200000.0);
  return bad == 0 ? 0 : 1;
}

int main() {
  int rc = run<double>("double", 1, 2000000);
  rc |= run<float>("float", 2, 2000000);
  return rc;
}
