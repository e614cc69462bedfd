// ORACLE PIN -- test infrastructure only.
//
// Drives DENSE's own deterministic simulator and analyses (compiled from the
// DENSE sources where they lie, by oracle/build.py, into oracle/_ref/)
// through the same C interface as dense_oracle.cpp, so the tests can check
// the restatement against the reference itself on identical inputs.
//
// Nothing here re-implements DENSE arithmetic: the simulation object is a
// dense::Deterministic_Simulation, the analyses are DENSE's BasicAnalysis
// and OscillationAnalysis, and the time loop calls them in the order of
// run_simulation (run_simulation.hpp:127-163).  Per-cell parameters are
// injected into the public cell_parameters_ matrix (sim/base.hpp:305)
// after construction, which is how a caller supplies an explicit
// per-cell parameter matrix.  DENSE's analyses keep their results in
// private members; this translation unit reads them by compiling DENSE's
// headers with `private`/`protected` mapped to `public`.
//
// ConcentrationCheck (measurement/conccheck.hpp) does not compile against
// the current DENSE headers (it derives from the old non-template Analysis
// and calls a constructor that no longer exists), so the harness carries
// its bound test (conccheck.hpp:25-51) on the current Analysis<Sim>
// interface, applied to the state of DENSE's own Deterministic_Simulation,
// and oracle_run drops a set the way run_simulation does
// (run_simulation.hpp:131-150).

// Standard headers first, so only DENSE's own classes see the access remap.
#include <algorithm>
#include <array>
#include <bitset>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <numeric>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <system_error>
#include <type_traits>
#include <utility>
#include <vector>

#define private public
#define protected public
#include "sim/determ/determ.hpp"
#include "measurement/oscillation.hpp"
#include "measurement/basic.hpp"
#include "measurement/bad_simulation_error.hpp"
#include "model_impl.hpp"
#undef private
#undef protected

using dense::Deterministic_Simulation;
using Sim = Deterministic_Simulation;

namespace {

// ConcentrationCheck::update and check (conccheck.hpp:25-51) as they are
// worded there: every cell of [min, max), the target species or (target -1)
// every species; a concentration below the lower or above the upper bound
// throws Bad_Simulation_Error for the simulation.
class HarnessConcCheck : public Analysis<Sim> {
 public:
  HarnessConcCheck(std::vector<Species> const& sp, dense::Natural cmin, dense::Natural cmax, Real lo, Real hi,
                   Real t0, Real t1, int target)
      : Analysis<Sim>(sp, {cmin, cmax}, {t0, t1}), lower_bound(lo), upper_bound(hi), target_specie(target) {}

  void update(Sim& simulation, std::ostream&) override {
    for (unsigned c = min; c < max; ++c) {
      if (target_specie > -1) {
        check(simulation, c, static_cast<Species>(target_specie));
      } else {
        for (dense::Natural s = 0; s < NUM_SPECIES; ++s) check(simulation, c, static_cast<Species>(s));
      }
    }
  }
  void finalize() override {}
  HarnessConcCheck* clone() const override { return new HarnessConcCheck(*this); }
  dense::Details get_details() override { return dense::Details(); }

 private:
  void check(Sim& simulation, dense::Natural cell, Species species) const {
    Real concentration = simulation.get_concentration(cell, species);
    if (concentration < lower_bound || concentration > upper_bound)
      throw dense::Bad_Simulation_Error<Sim>("Concentration out of bounds", simulation);
  }

  Real lower_bound, upper_bound;
  int target_specie;
};

struct Entry {
  int kind;  // 0 basic, 1 oscillation, 2 concentration check
  std::unique_ptr<Analysis<Sim>> a;
};

struct Harness {
  std::unique_ptr<Sim> sim;
  std::vector<Entry> analyses;
  int cells = 0;
  int status = 0;
  std::ostringstream sink;
};

// DENSE prints "steps per second" on every age_by (determ.cpp:18-19);
// the harness sends std::cout to a string sink while it runs.
struct Quiet {
  std::streambuf* old;
  explicit Quiet(std::ostream& to) : old(std::cout.rdbuf(to.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

}  // namespace

extern "C" {

struct oracle_model_info { int num_species, num_reactions, num_delay_reactions, num_critical_species, num_params; };

int oracle_model_info_get(oracle_model_info* out) {
  out->num_species = NUM_SPECIES;
  out->num_reactions = NUM_REACTIONS;
  out->num_delay_reactions = NUM_DELAY_REACTIONS;
  out->num_critical_species = NUM_CRITICAL_SPECIES;
  out->num_params = NUM_PARAMS;
  return 0;
}

const char* oracle_specie_name(int i) { return (i >= 0 && i < NUM_SPECIES) ? specie_str[i].c_str() : nullptr; }
const char* oracle_reaction_name(int i) { return (i >= 0 && i < NUM_REACTIONS) ? reaction_str[i].c_str() : nullptr; }

// DENSE's create_default_graph lives in Sim_Initializer.hpp, whose include
// chain needs the stochastic simulators; the tests build the default graph
// through the oracle restatement and hand the same CSR to both sides.
int oracle_default_graph(int, int, int*, int*) { return -1; }

void* oracle_create(int cells, const int* nbr_off, const int* nbr_idx,
                    const double* cell_params, const double* set_params,
                    const double* init_conc, double dt, const double* pert) {
  NGraph::Graph g;
  for (int c = 0; c < cells; ++c) g.insert_vertex(c);
  for (int c = 0; c < cells; ++c)
    for (int e = nbr_off[c]; e < nbr_off[c + 1]; ++e) g.insert_edge(c, nbr_idx[e]);
  Parameter_Set ps;
  std::copy(set_params, set_params + NUM_PARAMS, ps.begin());
  // initialize_params reads NUM_PARAMS perturbation factors (base.cpp:13-15)
  // from an array sized NUM_REACTIONS by parse_perturbations; pass a full
  // NUM_PARAMS array with zeros past NUM_REACTIONS.
  std::vector<Real> pert_buf;
  Real* pert_ptr = nullptr;
  if (pert) {
    pert_buf.assign(NUM_PARAMS, 0.0);
    std::copy(pert, pert + NUM_REACTIONS, pert_buf.begin());
    pert_ptr = pert_buf.data();
  }
  std::vector<Real> conc;
  if (init_conc) conc.assign(init_conc, init_conc + NUM_SPECIES);
  Harness* h = new Harness();
  h->cells = cells;
  {
    Quiet q(h->sink);
    h->sim.reset(new Sim(ps, pert_ptr, nullptr, Minutes{dt}, conc, std::move(g), 0));
  }
  for (int c = 0; c < cells; ++c)
    for (int i = 0; i < NUM_PARAMS; ++i)
      h->sim->cell_parameters_[c][i] = cell_params[static_cast<size_t>(c) * NUM_PARAMS + i];
  return h;
}

void oracle_destroy(void* p) { delete static_cast<Harness*>(p); }

void oracle_ring_sizes(void* p, int* S, double* max_delays) {
  Harness* h = static_cast<Harness*>(p);
  for (int i = 0; i < NUM_SPECIES; ++i) {
    S[i] = h->sim->_baby_cl.get_species_size(i);
    if (max_delays) max_delays[i] = h->sim->max_delays[i];
  }
}

int oracle_add_basic(void* p, int n, const int* species, int cmin, int cmax, double t0, double t1) {
  Harness* h = static_cast<Harness*>(p);
  std::vector<Species> sp;
  for (int i = 0; i < n; ++i) sp.push_back(static_cast<Species>(species[i]));
  h->analyses.push_back(Entry{0, std::unique_ptr<Analysis<Sim>>(
      new BasicAnalysis<Sim>(sp, {cmin, cmax}, {t0, t1}))});
  return static_cast<int>(h->analyses.size() - 1);
}

int oracle_add_oscillation(void* p, int n, const int* species, int cmin, int cmax, double t0, double t1,
                           double win_range, double anlys_intvl) {
  Harness* h = static_cast<Harness*>(p);
  std::vector<Species> sp;
  for (int i = 0; i < n; ++i) sp.push_back(static_cast<Species>(species[i]));
  h->analyses.push_back(Entry{1, std::unique_ptr<Analysis<Sim>>(
      new OscillationAnalysis<Sim>(anlys_intvl, win_range, sp, {cmin, cmax}, {t0, t1}))});
  return static_cast<int>(h->analyses.size() - 1);
}

int oracle_add_conccheck(void* p, int target, int cmin, int cmax, double lo, double hi, double t0, double t1) {
  Harness* h = static_cast<Harness*>(p);
  std::vector<Species> sp;
  if (target >= 0) sp.push_back(static_cast<Species>(target));
  h->analyses.push_back(Entry{2, std::unique_ptr<Analysis<Sim>>(
      new HarnessConcCheck(sp, cmin, cmax, lo, hi, t0, t1, target))});
  return static_cast<int>(h->analyses.size() - 1);
}

void oracle_steps(void* p, long n) {
  Harness* h = static_cast<Harness*>(p);
  for (long i = 0; i < n; ++i) h->sim->step();
}

// run_simulation's loop for one simulation (run_simulation.hpp:127-163):
// every analysis is called back in each chunk, each inside its own try; a
// Bad_Simulation_Error from any of them removes the simulation after the
// chunk's callbacks (it is not aged again, and its analyses are neither
// finalized nor shown), status 1.  Returns the chunks begun.
long oracle_run(void* p, double duration, double interval) {
  Harness* h = static_cast<Harness*>(p);
  using D = std::chrono::duration<Real, std::chrono::minutes::period>;
  D dur(duration), intvl(interval);
  Quiet q(h->sink);
  Real analysis_chunks = dur / intvl;
  long a = 0;
  for (a = 0; a < analysis_chunks; a++) {
    bool bad = false;
    for (auto& e : h->analyses) {
      try {
        e.a->when_updated_by(*h->sim, h->sink);
      } catch (dense::Bad_Simulation_Error<Sim>&) {
        bad = true;
      }
    }
    if (bad) {
      h->status |= 1;
      return a;
    }
    h->sim->age_by(intvl);
    h->sink.str("");
  }
  for (auto& e : h->analyses) if (e.kind == 1) e.a->finalize();
  return a;
}

// DENSE's analyses over imported samples [k][NS][cells] (what its
// --data-import means to do, main.cpp:160-175; its CSV_Streamed_Simulation
// never worked, io/csvr_sim.cpp:87-96 calls itself): sample a is written
// into DENSE's current rows (what get_concentration reads), the analyses
// are called back as in oracle_run, and the age advances by the interval
// through Simulation::age_by without stepping.  Returns the samples
// analysed.
long oracle_replay(void* p, const double* samples, long k, double t0, double interval) {
  Harness* h = static_cast<Harness*>(p);
  using D = std::chrono::duration<Real, std::chrono::minutes::period>;
  Quiet q(h->sink);
  h->sim->dense::Simulation::age_by(D(t0));
  long a = 0;
  for (a = 0; a < k; a++) {
    for (int sp = 0; sp < NUM_SPECIES; ++sp) {
      Real* row = h->sim->_baby_cl.row_at(sp, 0);
      for (int c = 0; c < h->cells; ++c) row[c] = samples[(static_cast<size_t>(a) * NUM_SPECIES + sp) * h->cells + c];
    }
    bool bad = false;
    for (auto& e : h->analyses) {
      try {
        e.a->when_updated_by(*h->sim, h->sink);
      } catch (dense::Bad_Simulation_Error<Sim>&) {
        bad = true;
      }
    }
    if (bad) {
      h->status |= 1;
      return a;
    }
    h->sim->dense::Simulation::age_by(D(interval));
    h->sink.str("");
  }
  for (auto& e : h->analyses) if (e.kind == 1) e.a->finalize();
  return a;
}

int oracle_status(void* p) { return static_cast<Harness*>(p)->status; }
double oracle_age(void* p) { return static_cast<Harness*>(p)->sim->age().count(); }

void oracle_get_state(void* p, double* out) {
  Harness* h = static_cast<Harness*>(p);
  for (int sp = 0; sp < NUM_SPECIES; ++sp)
    for (int c = 0; c < h->cells; ++c)
      out[static_cast<size_t>(sp) * h->cells + c] = h->sim->get_concentration(c, static_cast<Species>(sp));
}

void oracle_get_history(void* p, int sp, double* out) {
  Harness* h = static_cast<Harness*>(p);
  int S = h->sim->_baby_cl.get_species_size(sp);
  for (int lag = 0; lag < S; ++lag) {
    const Real* row = static_cast<const dense::baby_cl&>(h->sim->_baby_cl).row_at(sp, -lag);
    for (int c = 0; c < h->cells; ++c) out[static_cast<size_t>(lag) * h->cells + c] = row[c];
  }
}

void oracle_get_basic(void* p, int idx, double* mins, double* sums, double* maxs,
                      double* cmins, double* csums, double* cmaxs, int* samples, double* time) {
  Harness* h = static_cast<Harness*>(p);
  auto* b = static_cast<BasicAnalysis<Sim>*>(h->analyses[idx].a.get());
  size_t n = b->mins.size();
  for (size_t i = 0; i < n; ++i) { mins[i] = b->mins[i]; sums[i] = b->means[i]; maxs[i] = b->maxs[i]; }
  // Per-cell rows are only meaningful for cell_start == 0 in DENSE (they
  // are indexed by absolute cell number, basic.ipp:30-32).
  size_t rows = b->mins_by_context.size();
  for (size_t r = 0; r < rows; ++r)
    for (size_t i = 0; i < n; ++i) {
      if (cmins) cmins[r * n + i] = b->mins_by_context[r][i];
      if (csums) csums[r * n + i] = b->means_by_context[r][i];
      if (cmaxs) cmaxs[r * n + i] = b->maxs_by_context[r][i];
    }
  *samples = b->samples;
  *time = b->time;
}

void oracle_get_oscillation(void* p, int idx, double* amps, double* pers, double* avg_peak,
                            int* ncrit, int* samples, double* time) {
  Harness* h = static_cast<Harness*>(p);
  auto* o = static_cast<OscillationAnalysis<Sim>*>(h->analyses[idx].a.get());
  size_t ns = o->observed_species_.size();
  size_t nc = static_cast<size_t>(o->max - o->min);
  for (size_t s = 0; s < ns; ++s)
    for (size_t c = 0; c < nc; ++c) {
      size_t k = s * nc + c;
      amps[k] = o->amplitudes[s][c];
      pers[k] = o->periods[s][c];
      auto& x = o->peaksAndTroughs[s][c];
      int peaks = 0;
      double total = std::accumulate(x.begin(), x.end(), 0.0, [&](Real t, decltype(x[0]) cp) {
        if (cp.is_peak) { ++peaks; return t + cp.conc; }
        return t;
      });
      if (peaks != 0) total /= Real(peaks);
      avg_peak[k] = total;
      ncrit[k] = static_cast<int>(x.size());
    }
  *samples = o->samples;
  *time = o->time;
}

int oracle_get_crits(void* p, int idx, int s, int c, double* t, double* conc, int* is_peak, int cap) {
  Harness* h = static_cast<Harness*>(p);
  auto* o = static_cast<OscillationAnalysis<Sim>*>(h->analyses[idx].a.get());
  auto& list = o->peaksAndTroughs[s][c];
  int n = static_cast<int>(list.size());
  for (int i = 0; i < n && i < cap; ++i) { t[i] = list[i].time; conc[i] = list[i].conc; is_peak[i] = list[i].is_peak; }
  return n;
}

}  // extern "C"
