// Host-side tracing of a set's history reads, shared by every entry point
// that plans a batch (dense_engine_create / dense_engine_plan and
// dense_simulate_noalloc), so they size the same rings.
//
//   * ring_sizes: DENSE's ring size per species, S_sp = (int)(max_delays_sp
//     / dt + 2) (baby_cl.cpp:10), max_delays_sp being the largest delay
//     (times 1 + the -b perturbation factor) of the delay reactions whose
//     rate reads sp (Simulation::calc_max_delays, sim/base.cpp:55-140; the
//     gradient loop there never runs, circumference_ is 0 at that point, so
//     the gradient factor is 1).  The readers are found by evaluating the
//     model's own active_rate with a recording context, like DENSE's
//     DummyContext (sim/base.cpp:62-95).
//   * trace_lags: the lag of every history read the model's rates make,
//     with the lag arithmetic of the device contexts (own reads (k-1) mod S,
//     neighbour reads k mod S; determ.hpp:73-89, baby_cl.hpp:28-42).  The
//     rates are evaluated per traced cell four times with different
//     stand-in concentrations and neighbour averages, so reads behind
//     concentration-dependent branches are seen too.  A read missed here is
//     still caught on the device (DENSE_SET_UNSTAGED_LAG).
//
// The includer includes dense_model_api.hpp and the model's
// reaction_deltas.hpp and model_impl.hpp first.
#pragma once

#include <algorithm>
#include <limits>

#include "dense_b200.h"

namespace dense_b200 {

// DummyContext of sim/base.cpp:62-95: records which species a rate reads.
struct DepContext {
  bool* deps;
  double getCon(specie_id sp, int = 0) const { deps[sp] = true; return 0.0; }
  double calculateNeighborAvg(specie_id sp, int = 0) const { deps[sp] = true; return 0.0; }
  double getRate(reaction_id) const { return 0.0; }
  double getDelay(delay_reaction_id) const { return 0.0; }
  double getCritVal(critspecie_id) const { return 0.0; }
};

// What the traced reads of one set need from the history.
struct LagTrace {
  int own_max[NUM_SPECIES];    // deepest own lag (0: lag 0 only)
  int nbr_max[NUM_SPECIES];    // deepest neighbour lag, -1 none
  bool ordered = false;        // some neighbour read is at lag S-1 (the row written this step)
  bool bad = false;            // a delay DENSE would turn into an out-of-bounds read
  bool ord_sp[NUM_SPECIES];    // species read by neighbours at lag S-1
  int plain_min[NUM_SPECIES];  // shallowest other neighbour lag (INT_MAX none)
  int plain_max[NUM_SPECIES];  // deepest other neighbour lag (-1 none)
  LagTrace() {
    for (int sp = 0; sp < NUM_SPECIES; ++sp) {
      own_max[sp] = 0;
      nbr_max[sp] = -1;
      ord_sp[sp] = false;
      plain_min[sp] = std::numeric_limits<int>::max();
      plain_max[sp] = -1;
    }
  }
};

// Records, for one cell, the lag of every history read its reactions make.
struct LagTracer {
  const double* prm;  // the cell's parameters [NUM_PARAMS]
  const double* conc;
  double nbr_value;
  const int* S;
  LagTrace* t;
  double getCon(specie_id sp) const { return conc[sp]; }
  double getCon(specie_id sp, int k) const {
    const int s = S[sp];
    if (k < 0 || k > s + 1) t->bad = true;
    const int lag = (((k - 1) % s) + s) % s;
    t->own_max[sp] = std::max(t->own_max[sp], lag);
    return conc[sp];
  }
  double calculateNeighborAvg(specie_id sp, int k = 0) const {
    const int s = S[sp];
    if (k < 0 || k > s) t->bad = true;
    const int lag = ((k % s) + s) % s;
    if (lag == s - 1 && s > 1) {
      t->ordered = t->ord_sp[sp] = true;
    } else {
      t->plain_min[sp] = std::min(t->plain_min[sp], lag);
      t->plain_max[sp] = std::max(t->plain_max[sp], lag);
    }
    t->nbr_max[sp] = std::max(t->nbr_max[sp], lag);
    return nbr_value;
  }
  double getRate(reaction_id r) const { return prm[r]; }
  double getDelay(delay_reaction_id d) const { return prm[NUM_REACTIONS + d]; }
  double getCritVal(critspecie_id c) const { return prm[NUM_REACTIONS + NUM_DELAY_REACTIONS + c]; }
};

// DENSE's ring sizes of one set; false when one is not a positive int.
inline bool ring_sizes(const dense_set_desc& in, double dt, int* S) {
  bool deps[NUM_REACTIONS][NUM_SPECIES] = {};
#define REACTION(name) { DepContext c{deps[name]}; reaction<name>::active_rate(c); }
#include "reactions_list.hpp"
#undef REACTION
  double max_delays[NUM_SPECIES] = {};
  for (int dr = 0; dr < NUM_DELAY_REACTIONS; ++dr) {
    const int r = dense_delay_reaction_of[dr];
    const double pert = in.perturb ? in.perturb[r] : 0.0;
    for (int sp = 0; sp < NUM_SPECIES; ++sp) {
      if (!deps[r][sp]) continue;
      const double v = in.set_params[NUM_REACTIONS + dr] * 1.0 * (1.0 + pert);
      max_delays[sp] = (v < max_delays[sp]) ? max_delays[sp] : v;
    }
  }
  for (int sp = 0; sp < NUM_SPECIES; ++sp) {
    const double v = max_delays[sp] / dt + 2;  // baby_cl.cpp:10
    if (!(v >= 1.0 && v < 2147483647.0)) return false;
    S[sp] = static_cast<int>(v);
  }
  return true;
}

// Traces cells [0, cells): cell c's parameter i is p[c * cell_stride +
// i * param_stride].
inline void trace_lags(const double* p, int cells, long cell_stride, long param_stride, const int* S,
                       LagTrace& out) {
  double prm[NUM_PARAMS];
  double conc[NUM_SPECIES];
  const double nbr_values[4] = {0.0, 2.0, 0.5, 7.25};
  for (int c = 0; c < cells; ++c) {
    for (int i = 0; i < NUM_PARAMS; ++i) prm[i] = p[c * cell_stride + i * param_stride];
    for (int pass = 0; pass < 4; ++pass) {
      for (int sp = 0; sp < NUM_SPECIES; ++sp) conc[sp] = pass == 0 ? 0.0 : (pass == 1 ? 1.0 : 0.37 * (sp + pass));
      LagTracer t{prm, conc, nbr_values[pass], S, &out};
#define REACTION(name) reaction<name>::active_rate(t);
#include "reactions_list.hpp"
#undef REACTION
    }
  }
}

}  // namespace dense_b200
