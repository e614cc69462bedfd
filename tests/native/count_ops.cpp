// Operation and history-read count of one cell-step of a DENSE model, by
// evaluating the model's own active_rate specialisations with a counting
// arithmetic type (the model API's DENSE_B200_REAL hook) and a context that
// records every read.  Compiled per model with -I <model dir>.
//
// Usage: count_ops <avg neighbours> <S_0> ... <S_{NS-1}> <p_0> ... <p_{NP-1}>
// (ring sizes S per species and the parameter set, which sets the delays).
// Prints: rate_adds rate_muls rate_divs rate_cmps neighbour_averages
//         delta_terms species distinct_history_rows
// where neighbour averages are counted as calls (each is one add per
// neighbour and one division, DENSE's calculate_neighbor_average,
// sim/determ/determ.hpp:81-89) and a history row is a (species, lag) the
// rates read other than the cell's own lag-0 state.
#include <cstdio>
#include <cstdlib>
#include <set>
#include <utility>

namespace count {
long long add = 0, mul = 0, dvd = 0, cmp = 0;
}

struct CountReal {
  double v;
  CountReal() : v(0.0) {}
  CountReal(double x) : v(x) {}  // constants and RATETYPE(1.0) in model code
  explicit operator double() const { return v; }
};
inline CountReal operator+(CountReal a, CountReal b) { ++count::add; return a.v + b.v; }
inline CountReal operator-(CountReal a, CountReal b) { ++count::add; return a.v - b.v; }
inline CountReal operator*(CountReal a, CountReal b) { ++count::mul; return a.v * b.v; }
inline CountReal operator/(CountReal a, CountReal b) { ++count::dvd; return a.v / b.v; }
inline CountReal operator-(CountReal a) { return -a.v; }  // a sign flip, not an operation
inline CountReal& operator+=(CountReal& a, CountReal b) { a = a + b; return a; }
inline CountReal& operator-=(CountReal& a, CountReal b) { a = a - b; return a; }
inline CountReal& operator*=(CountReal& a, CountReal b) { a = a * b; return a; }
inline CountReal& operator/=(CountReal& a, CountReal b) { a = a / b; return a; }
inline bool operator<(CountReal a, CountReal b) { ++count::cmp; return a.v < b.v; }
inline bool operator>(CountReal a, CountReal b) { ++count::cmp; return a.v > b.v; }
inline bool operator<=(CountReal a, CountReal b) { ++count::cmp; return a.v <= b.v; }
inline bool operator>=(CountReal a, CountReal b) { ++count::cmp; return a.v >= b.v; }
inline bool operator==(CountReal a, CountReal b) { ++count::cmp; return a.v == b.v; }
inline bool operator!=(CountReal a, CountReal b) { ++count::cmp; return a.v != b.v; }

#define DENSE_B200_REAL CountReal
#include "dense_model_api.hpp"
#include "reaction_deltas.hpp"
#include "model_impl.hpp"

namespace {

int S[NUM_SPECIES];
double P[NUM_PARAMS];
std::set<std::pair<int, int>> rows;  // (species, lag) read from history
long long neighbour_averages = 0;

// DENSE's reads (sim/base.hpp:64-80, sim/determ/determ.hpp:73-89): an own
// read with delay k reads lag (k - 1) mod S, a neighbour average lag k mod S;
// an own read at lag 0 is the cell's state.
struct Counter {
  CountReal getCon(specie_id sp) const { return getCon(sp, 1.0); }
  CountReal getCon(specie_id sp, double delay) const {
    const int k = static_cast<int>(delay);
    const int lag = ((k - 1) % S[sp] + S[sp]) % S[sp];
    if (lag != 0) rows.insert({static_cast<int>(sp), lag});
    return 1.0;
  }
  CountReal calculateNeighborAvg(specie_id sp) const { return calculateNeighborAvg(sp, 0.0); }
  CountReal calculateNeighborAvg(specie_id sp, double delay) const {
    const int k = static_cast<int>(delay);
    rows.insert({static_cast<int>(sp), ((k % S[sp]) + S[sp]) % S[sp]});
    ++neighbour_averages;
    return 1.0;
  }
  CountReal getRate(reaction_id r) const { return P[r]; }
  double getDelay(delay_reaction_id d) const { return P[NUM_REACTIONS + d]; }
  CountReal getCritVal(critspecie_id c) const { return P[NUM_REACTIONS + NUM_DELAY_REACTIONS + c]; }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc != 2 + NUM_SPECIES + NUM_PARAMS) {
    std::fprintf(stderr, "need avg_neighbours, %d ring sizes and %d parameters\n", NUM_SPECIES, NUM_PARAMS);
    return 2;
  }
  for (int i = 0; i < NUM_SPECIES; ++i) S[i] = std::atoi(argv[2 + i]);
  for (int i = 0; i < NUM_PARAMS; ++i) P[i] = std::atof(argv[2 + NUM_SPECIES + i]);
  Counter c;
  long long delta_terms = 0;
#define REACTION(name)                        \
  reaction<name>::active_rate(c);             \
  delta_terms += num_deltas_##name;
#include "reactions_list.hpp"
#undef REACTION
  // a neighbour row is sometimes also the own row of the same lag; rows
  // holding the lag-0 state are not history
  std::set<std::pair<int, int>> hist;
  for (const auto& r : rows)
    if (r.second != 0) hist.insert(r);
  std::printf("%lld %lld %lld %lld %lld %lld %d %zu\n", count::add, count::mul, count::dvd, count::cmp,
              neighbour_averages, delta_terms, NUM_SPECIES, hist.size());
  return 0;
}
