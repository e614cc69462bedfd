// ORACLE -- test infrastructure only.
//
// A CPU restatement, in plain sequential C++, of DENSE's deterministic
// delay-differential simulation path.  It exists to check the CUDA engine:
// only the tests, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// load it, and never as the thing measured or shipped.
//
// Parity is pinned two ways (tests/test_oracle_*.py):
//   * against the golden files of DENSE's own CTest suite
//     (test/her_model_2014/anlys_basic_a.csv, anlys_oscil.csv; the fixtures
//     under tests/golden/ hold the values), and
//   * against DENSE itself, compiled from its sources by oracle/build.py into
//     oracle/_ref/ and driven through the same C interface (ref_harness.cpp),
//     bit for bit on trajectories and analysis outputs.
//
// It compiles against the model headers of one DENSE model directory
// (-I<model_dir>) through the engine's model-API headers
// (dense_b200/csrc/model_api), exactly like the engine does.
//
// Every function cites the DENSE source lines (paths inside the DENSE tree)
// whose behaviour it restates.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "dense_model_api.hpp"
#include "reaction_deltas.hpp"
#include "model_impl.hpp"

namespace {

constexpr int NS = NUM_SPECIES;
constexpr int NR = NUM_REACTIONS;
constexpr int NP = NUM_PARAMS;

enum : int {
  ST_OK = 0,
  ST_DROPPED = 1,      // a concentration check rejected the set
  ST_NAN_PARAM = 2,    // getRate / getDelay saw NaN (DENSE throws)
  ST_BAD_INDEX = 4,    // a ring offset DENSE would read out of bounds
};

// ------------------------------------------------------------ the history
// baby_cl (sim/determ/baby_cl.hpp:13-55, baby_cl.cpp:5-15): one circular
// buffer of S_sp rows per species, each row one value per cell.
struct History {
  int cells = 0;
  int S[NS] = {};
  int j[NS] = {};
  std::vector<double> rows[NS];

  // baby_cl::wrap (baby_cl.hpp:26-30): C++ remainder, may be negative.
  static int wrap(int x, int y) { return (x + y) % y; }

  // baby_cl::row_at (baby_cl.hpp:39-47).  Returns -1 where DENSE would
  // index before the start of its array.
  int row(int sp, int off) const {
    int r = (off == 0) ? j[sp] : wrap(j[sp] + off, S[sp]);
    return r;
  }
  // baby_cl::advance (baby_cl.hpp:49-54).
  void advance() {
    for (int i = 0; i < NS; ++i) j[i] = wrap(j[i] + 1, S[i]);
  }
};

struct Sim;

// Context (sim/base.hpp:51-88, 393-427) over one cell of one simulation.
struct Ctx {
  Sim* s;
  int cell;
  double getCon(specie_id sp) const;
  double getCon(specie_id sp, int delay) const;
  double calculateNeighborAvg(specie_id sp, int delay = 0) const;
  double getRate(reaction_id r) const;
  double getDelay(delay_reaction_id d) const;
  double getCritVal(critspecie_id c) const;
};

// Dependency tracer of calc_max_delays (sim/base.cpp:62-95): records which
// species each reaction reads; every getter returns 0.
struct DepCtx {
  bool* deps;
  double getCon(specie_id sp, int = 0) const { deps[sp] = true; return 0.0; }
  double calculateNeighborAvg(specie_id sp, int = 0) const { deps[sp] = true; return 0.0; }
  double getRate(reaction_id) const { return 0.0; }
  double getDelay(delay_reaction_id) const { return 0.0; }
  double getCritVal(critspecie_id) const { return 0.0; }
};

// ------------------------------------------------------------- analyses
struct Basic {  // measurement/basic.ipp:5-75
  std::vector<int> species;
  int cmin = 0, cmax = 0;
  double t0 = 0, t1 = std::numeric_limits<double>::infinity();
  double time = 0;
  int samples = 0;
  std::vector<double> mins, maxs, sums;            // [species]
  std::vector<double> cmins, cmaxs, csums;         // [cell][species]
};

struct Crit { double time, conc; bool is_peak; };

// core/queue.hpp:29-88, with its index arithmetic kept as is.
struct Queue {
  std::vector<double> contents;
  long start = 0, end = -1, current = -1, size = 0;
  explicit Queue(long length) : contents(length + 1), size(length + 1) {}
  long getSize() const { return (size + end - start) % size + 1; }
  void enqueue(double v) {
    end = (end == size - 1) ? 0 : end + 1;
    contents[end] = v;
    if (2 * getSize() >= size) { ++current; if (current == size) current = 0; }
  }
  double dequeue() {
    double popped = contents[start];
    start = (start == size - 1) ? 0 : start + 1;
    if (2 * getSize() <= size) { ++current; if (current == size) current = 0; }
    return popped;
  }
};

struct Oscil {  // measurement/oscillation.hpp:17-117, oscillation.ipp
  std::vector<int> species;
  int cmin = 0, cmax = 0;
  double t0 = 0, t1 = std::numeric_limits<double>::infinity();
  double time = 0;
  int samples = 0;
  int range_steps = 0;
  double interval = 0;
  std::vector<Queue> win;                 // [s][c]
  std::vector<std::vector<double>> live;  // the multiset mirror: live values
  std::vector<std::vector<Crit>> crits;   // [s][c]
  std::vector<double> amps, pers;         // [s][c]
};

struct Check {  // measurement/conccheck.hpp:7-53
  int target = -1;  // -1: every species
  int cmin = 0, cmax = 0;
  double lo = 0, hi = 0;
  double t0 = 0, t1 = std::numeric_limits<double>::infinity();
  double time = 0;
};

struct Sim {
  int cells = 0;
  std::vector<std::vector<int>> nbrs;  // ascending ids (std::set order)
  std::vector<double> params;          // [cell][NP]
  double set_params[NP] = {};
  double max_delays[NS] = {};
  double dt = 0;
  double age = 0;
  History h;
  int status = ST_OK;
  std::vector<Basic> basics;
  std::vector<Oscil> oscils;
  std::vector<Check> checks;
  std::vector<int> order;  // analysis callback order: (kind, index)

  double* row_ptr(int sp, int off) {
    int r = h.row(sp, off);
    if (r < 0 || r >= h.S[sp]) { status |= ST_BAD_INDEX; r = ((r % h.S[sp]) + h.S[sp]) % h.S[sp]; }
    return h.rows[sp].data() + static_cast<size_t>(r) * cells;
  }
  // Deterministic_Simulation::get_concentration (determ.hpp:73-79).
  double conc(int cell, int sp, int delay) { return row_ptr(sp, 1 - delay)[cell]; }
  double conc(int cell, int sp) { return conc(cell, sp, 1); }
  // Deterministic_Simulation::calculate_neighbor_average (determ.hpp:81-89).
  double nbr_avg(int cell, int sp, int delay) {
    double sum = 0.0;
    const double* row = row_ptr(sp, -delay);
    for (int n : nbrs[cell]) sum += row[n];
    double avg = sum / static_cast<int>(nbrs[cell].size());
    return std::isnan(avg) ? 0 : avg;
  }
};

double Ctx::getCon(specie_id sp) const { return s->conc(cell, sp); }
double Ctx::getCon(specie_id sp, int delay) const { return s->conc(cell, sp, delay); }
double Ctx::calculateNeighborAvg(specie_id sp, int delay) const { return s->nbr_avg(cell, sp, delay); }
double Ctx::getRate(reaction_id r) const {  // base.hpp:398-404
  double v = s->params[static_cast<size_t>(cell) * NP + r];
  if (std::isnan(v)) s->status |= ST_NAN_PARAM;
  return v;
}
double Ctx::getDelay(delay_reaction_id d) const {  // base.hpp:406-412
  double v = s->params[static_cast<size_t>(cell) * NP + NR + d];
  if (std::isnan(v)) s->status |= ST_NAN_PARAM;
  return v;
}
double Ctx::getCritVal(critspecie_id c) const {  // base.hpp:393-396
  return s->params[static_cast<size_t>(cell) * NP + NR + NUM_DELAY_REACTIONS + c];
}

// Simulation::calc_max_delays (sim/base.cpp:55-140).  The gradient factor
// loop there runs over circumference_, which is still 0 when the
// constructor calls it (base.cpp:36, 46-47), so max_gradient stays 1.
void calc_max_delays(Sim& s, const double* pert) {
  for (int i = 0; i < NS; ++i) s.max_delays[i] = 0.0;
  bool deps[NR][NS] = {};
#define REACTION(name) { DepCtx c{deps[name]}; reaction<name>::active_rate(c); }
#include "reactions_list.hpp"
#undef REACTION
  for (int d = 0; d < NUM_DELAY_REACTIONS; ++d) {
    int r = dense_delay_reaction_of[d];
    double max_gradient = 1.0;
    double p = pert ? pert[r] : 0.0;
    for (int sp = 0; sp < NS; ++sp) {
      if (!deps[r][sp]) continue;
      double v = s.set_params[NR + d] * max_gradient * (1.0 + p);
      s.max_delays[sp] = (v < s.max_delays[sp]) ? s.max_delays[sp] : v;  // std::max(v, cur)
    }
  }
}

// baby_cl::baby_cl (baby_cl.cpp:5-15) and the history fill of the
// Deterministic_Simulation constructor (determ.cpp:31-52).
void init_history(Sim& s, const double* init_conc) {
  for (int sp = 0; sp < NS; ++sp) {
    s.h.S[sp] = static_cast<int>(s.max_delays[sp] / s.dt + 2);
    s.h.j[sp] = 0;
    s.h.rows[sp].assign(static_cast<size_t>(s.h.S[sp]) * s.cells, 0.0);
    if (init_conc)
      std::fill(s.h.rows[sp].begin(), s.h.rows[sp].end(), init_conc[sp]);
  }
  s.h.cells = s.cells;
}

// calculate_concentrations + update_concentrations + step
// (determ.cpp:23-29, 54-88): cells in index order, every rate first, then
// the deltas reaction by reaction, then x(+1) = x(0) + dt * delta.
void step(Sim& s) {
  for (int c = 0; c < s.cells; ++c) {
    Ctx ctx{&s, c};
    double rates[NR];
#define REACTION(name) rates[name] = reaction<name>::active_rate(ctx);
#include "reactions_list.hpp"
#undef REACTION
    double d[NS] = {};
#define REACTION(name) \
    for (int j = 0; j < num_deltas_##name; j++) d[delta_ids_##name[j]] += rates[name] * deltas_##name[j];
#include "reactions_list.hpp"
#undef REACTION
    for (int i = 0; i < NS; ++i) {
      double* nxt = s.row_ptr(i, 1);
      double* cur = s.row_ptr(i, 0);
      nxt[c] = cur[c] + s.dt * d[i];
    }
  }
  s.h.advance();
}

// BasicAnalysis::update (basic.ipp:22-36).  std::min(a, b) is
// (b < a) ? b : a and std::max(a, b) is (a < b) ? b : a; the NaN behaviour
// of those expressions is kept.  Per-cell rows are indexed from cell_start.
void basic_update(Sim& s, Basic& b) {
  for (int c = b.cmin; c < b.cmax; ++c) {
    for (size_t i = 0; i < b.species.size(); ++i) {
      double x = s.conc(c, b.species[i]);
      b.mins[i] = (b.mins[i] < x) ? b.mins[i] : x;
      b.maxs[i] = (x < b.maxs[i]) ? b.maxs[i] : x;
      b.sums[i] += x;
      size_t k = static_cast<size_t>(c - b.cmin) * b.species.size() + i;
      b.cmins[k] = (b.cmins[k] < x) ? b.cmins[k] : x;
      b.cmaxs[k] = (x < b.cmaxs[k]) ? b.cmaxs[k] : x;
      b.csums[k] += x;
    }
  }
  ++b.samples;
}

double window_max(const std::vector<double>& v) {  // *multiset.rbegin()
  double m = v[0];
  for (double x : v) if (m < x) m = x;
  return m;
}
double window_min(const std::vector<double>& v) {  // *multiset.begin()
  double m = v[0];
  for (double x : v) if (x < m) m = x;
  return m;
}
void erase_one(std::vector<double>& v, double x) {  // multiset.erase(find(x))
  for (size_t i = 0; i < v.size(); ++i)
    if (v[i] == x) { v.erase(v.begin() + i); return; }
}

// OscillationAnalysis::addCritPoint (oscillation.ipp:129-144).
void add_crit(std::vector<Crit>& list, Crit c) {
  if (!list.empty()) {
    Crit prev = list.back();
    if (prev.is_peak == c.is_peak) {
      if (c.is_peak ? (c.conc >= prev.conc) : (c.conc <= prev.conc)) list.back() = c;
    } else {
      list.push_back(c);
    }
  } else {
    list.push_back(c);
  }
}

// OscillationAnalysis::checkCritPoint (oscillation.ipp:110-119).  Where
// the queue's middle index is still -1 (one sample per window, as it first
// reaches range_steps/2 values) DENSE reads contents[-1]; here that sample
// yields no critical point.  An empty multiset yields none either.
void check_crit(Oscil& o, int s, int c) {
  size_t k = static_cast<size_t>(s) * (o.cmax - o.cmin) + c;
  Queue& q = o.win[k];
  if (q.current < 0 || o.live[k].empty()) return;
  double mid = q.contents[q.current];
  double hi = window_max(o.live[k]), lo = window_min(o.live[k]);
  double t = (o.samples - o.range_steps / 2) * o.interval + o.t0;
  t = (0.0 < t) ? t : 0.0;  // std::max<Real>(0.0, t)
  if (mid == hi && mid != lo) add_crit(o.crits[k], Crit{t, mid, true});
  else if (mid == lo) add_crit(o.crits[k], Crit{t, mid, false});
}

// OscillationAnalysis::update / get_peaks_and_troughs (oscillation.ipp:
// 154-160, 86-103), including the early return that skips the remaining
// species of a cell while the current species' window is short.
void oscil_update(Sim& s, Oscil& o) {
  for (int c = o.cmin; c < o.cmax; ++c) {
    int cc = c - o.cmin;
    for (size_t i = 0; i < o.species.size(); ++i) {
      size_t k = i * (o.cmax - o.cmin) + cc;
      double added = s.conc(c, o.species[i]);
      o.win[k].enqueue(added);
      o.live[k].push_back(added);
      if (o.win[k].getSize() == o.range_steps + 1) {
        double removed = o.win[k].dequeue();
        erase_one(o.live[k], removed);
      }
      if (o.win[k].getSize() < o.range_steps / 2) break;
      check_crit(o, static_cast<int>(i), cc);
    }
  }
  ++o.samples;
}

// OscillationAnalysis::calcAmpsAndPers (oscillation.ipp:167-185).
void amps_pers(Oscil& o, size_t k) {
  const std::vector<Crit>& cr = o.crits[k];
  double peakSum = 0.0, troughSum = 0.0, cycleSum = 0.0;
  int numPeaks = 0, numTroughs = 0, cycles = 0;
  for (size_t i = 0; i < cr.size(); ++i) {
    if (cr[i].is_peak) { peakSum += cr[i].conc; ++numPeaks; }
    else { troughSum += cr[i].conc; ++numTroughs; }
    if (i < 2) continue;
    ++cycles;
    cycleSum += (cr[i].time - cr[i - 2].time);
  }
  o.amps[k] = ((peakSum / numPeaks) - (troughSum / numTroughs)) / 2;
  o.pers[k] = cycleSum / cycles;
}

// OscillationAnalysis::finalize (oscillation.ipp:6-26).
void oscil_finalize(Oscil& o) {
  int timeTemp = o.samples;
  int ncell = o.cmax - o.cmin;
  for (size_t s = 0; s < o.species.size(); ++s) {
    for (int c = 0; c < ncell; ++c) {
      size_t k = s * ncell + c;
      o.samples = timeTemp;
      while (o.win[k].getSize() >= (o.range_steps / 2) && !o.live[k].empty()) {
        double removed = o.win[k].dequeue();
        erase_one(o.live[k], removed);
        check_crit(o, static_cast<int>(s), c);
        ++o.samples;
      }
      amps_pers(o, k);
    }
  }
}

// ConcentrationCheck::update / check (conccheck.hpp:25-51).
bool check_update(Sim& s, Check& ck) {
  for (int c = ck.cmin; c < ck.cmax; ++c) {
    for (int sp = 0; sp < NS; ++sp) {
      if (ck.target >= 0 && sp != ck.target) continue;
      double x = s.conc(c, sp);
      if (x < ck.lo || x > ck.hi) return false;
    }
  }
  return true;
}

}  // namespace

// ------------------------------------------------------------- C interface
extern "C" {

struct oracle_model_info { int num_species, num_reactions, num_delay_reactions, num_critical_species, num_params; };

int oracle_model_info_get(oracle_model_info* out) {
  out->num_species = NS;
  out->num_reactions = NR;
  out->num_delay_reactions = NUM_DELAY_REACTIONS;
  out->num_critical_species = NUM_CRITICAL_SPECIES;
  out->num_params = NP;
  return 0;
}

const char* oracle_specie_name(int i) { return (i >= 0 && i < NS) ? dense_specie_names[i] : nullptr; }
const char* oracle_reaction_name(int i) { return (i >= 0 && i < NR) ? dense_reaction_names[i] : nullptr; }

// create_default_graph (Sim_Initializer.hpp:103-136): hexagonal stencil
// with periodic wrap; each cell's out-neighbour set is ascending (std::set).
// Writes CSR arrays; nbr_idx must hold 6 * cells entries.  Returns the edge
// count.
int oracle_default_graph(int cell_total, int width, int* nbr_off, int* nbr_idx) {
  std::vector<std::vector<int>> out(cell_total);
  auto ins = [&](int a, int b) {
    b = std::abs(b);
    auto& v = out[a];
    if (std::find(v.begin(), v.end(), b) == v.end()) v.push_back(b);
  };
  for (int i = 0; i < cell_total; ++i) {
    bool former = i % width == 0;
    bool latter = (i + 1) % width == 0;
    bool even = i % 2 == 0;
    int la = (former || !even) ? width - 1 : -1;
    int ra = !(latter || even) ? width + 1 : 1;
    int top = (i - width + cell_total) % cell_total;
    int bottom = (i + width) % cell_total;
    int bottom_right = (i + ra) % cell_total;
    int top_left = (i + la) % cell_total;
    int top_right = (i - width + ra + cell_total) % cell_total;
    int bottom_left = (i - width + la + cell_total) % cell_total;
    if (former) { ins(i, top); ins(i, top_left); ins(i, top_right); ins(i, bottom_left); }
    else if (latter) { ins(i, top); ins(i, top_right); ins(i, bottom_right); ins(i, bottom); }
    else { ins(i, top_right); ins(i, bottom_right); ins(i, bottom); ins(i, top_left); ins(i, bottom_left); }
  }
  int e = 0;
  for (int i = 0; i < cell_total; ++i) {
    std::sort(out[i].begin(), out[i].end());
    nbr_off[i] = e;
    for (int n : out[i]) nbr_idx[e++] = n;
  }
  nbr_off[cell_total] = e;
  return e;
}

// Build one simulation.  cell_params ([cells][NP]) are the per-cell
// parameters the step reads (DENSE's cell_parameters_, base.hpp:305);
// set_params ([NP]) is the parameter set the ring sizes are derived from
// (calc_max_delays reads parameter_set_, base.cpp:135).  pert ([NR] or
// NULL) only enters the ring sizing, as in DENSE.  init_conc ([NS] or NULL
// for all-zero rows).
void* oracle_create(int cells, const int* nbr_off, const int* nbr_idx,
                    const double* cell_params, const double* set_params,
                    const double* init_conc, double dt, const double* pert) {
  Sim* s = new Sim();
  s->cells = cells;
  s->nbrs.resize(cells);
  for (int c = 0; c < cells; ++c)
    for (int e = nbr_off[c]; e < nbr_off[c + 1]; ++e) s->nbrs[c].push_back(nbr_idx[e]);
  s->params.assign(cell_params, cell_params + static_cast<size_t>(cells) * NP);
  std::memcpy(s->set_params, set_params, sizeof(double) * NP);
  s->dt = dt;
  calc_max_delays(*s, pert);
  init_history(*s, init_conc);
  return s;
}

void oracle_destroy(void* h) { delete static_cast<Sim*>(h); }

void oracle_ring_sizes(void* h, int* S, double* max_delays) {
  Sim* s = static_cast<Sim*>(h);
  for (int i = 0; i < NS; ++i) { S[i] = s->h.S[i]; if (max_delays) max_delays[i] = s->max_delays[i]; }
}

int oracle_add_basic(void* h, int n, const int* species, int cmin, int cmax, double t0, double t1) {
  Sim* s = static_cast<Sim*>(h);
  Basic b;
  b.species.assign(species, species + n);
  b.cmin = cmin; b.cmax = cmax; b.t0 = t0; b.t1 = t1;
  b.mins.assign(n, std::numeric_limits<double>::infinity());
  b.maxs.assign(n, 0.0);
  b.sums.assign(n, 0.0);
  b.cmins.assign(static_cast<size_t>(cmax - cmin) * n, std::numeric_limits<double>::infinity());
  b.cmaxs.assign(static_cast<size_t>(cmax - cmin) * n, 0.0);
  b.csums.assign(static_cast<size_t>(cmax - cmin) * n, 0.0);
  s->basics.push_back(b);
  s->order.push_back(0 * 65536 + static_cast<int>(s->basics.size() - 1));
  return static_cast<int>(s->order.size() - 1);
}

int oracle_add_oscillation(void* h, int n, const int* species, int cmin, int cmax, double t0, double t1,
                           double win_range, double anlys_intvl) {
  Sim* s = static_cast<Sim*>(h);
  Oscil o;
  o.species.assign(species, species + n);
  o.cmin = cmin; o.cmax = cmax; o.t0 = t0; o.t1 = t1;
  o.range_steps = static_cast<int>(win_range / anlys_intvl);  // oscillation.hpp:64
  o.interval = anlys_intvl;
  size_t cells = static_cast<size_t>(cmax - cmin);
  for (size_t i = 0; i < n * cells; ++i) o.win.emplace_back(o.range_steps);
  o.live.resize(n * cells);
  o.crits.resize(n * cells);
  o.amps.assign(n * cells, 0.0);
  o.pers.assign(n * cells, 0.0);
  s->oscils.push_back(std::move(o));
  s->order.push_back(1 * 65536 + static_cast<int>(s->oscils.size() - 1));
  return static_cast<int>(s->order.size() - 1);
}

int oracle_add_conccheck(void* h, int target, int cmin, int cmax, double lo, double hi, double t0, double t1) {
  Sim* s = static_cast<Sim*>(h);
  Check ck;
  ck.target = target; ck.cmin = cmin; ck.cmax = cmax; ck.lo = lo; ck.hi = hi; ck.t0 = t0; ck.t1 = t1;
  s->checks.push_back(ck);
  s->order.push_back(2 * 65536 + static_cast<int>(s->checks.size() - 1));
  return static_cast<int>(s->order.size() - 1);
}

// Raw Euler steps, no analyses (Deterministic_Simulation::step,
// sim/determ/determ.cpp:77-88).
void oracle_steps(void* h, long n) {
  Sim* s = static_cast<Sim*>(h);
  for (long i = 0; i < n; ++i) step(*s);
}

// The time loop of run_simulation (run_simulation.hpp:127-163) with
// Analysis::when_updated_by (measurement/base.ipp:4-9) and
// Deterministic_Simulation::age_by (determ.cpp:8-21):
//   chunks a = 0, 1, ... while a < duration / interval;
//   each chunk: every analysis samples the current state if
//   time-start <= age < time-end, a failed concentration check drops the
//   simulation, then (int)(interval / dt) steps and age += interval;
//   at the end every oscillation analysis is finalized.
// Returns the number of chunks run before the set was dropped (or all).
// One round of analysis callbacks at the current age (run_simulation.hpp:
// 131-136): each analysis samples the state if time-start <= age <
// time-end; false when a concentration check failed.
static bool callbacks(Sim* s) {
  bool bad = false;
  for (int key : s->order) {
    int kind = key / 65536, idx = key % 65536;
    if (kind == 0) {
      Basic& b = s->basics[idx];
      b.time = s->age;
      if (b.time < b.t0 || b.time >= b.t1) continue;
      basic_update(*s, b);
    } else if (kind == 1) {
      Oscil& o = s->oscils[idx];
      o.time = s->age;
      if (o.time < o.t0 || o.time >= o.t1) continue;
      oscil_update(*s, o);
    } else {
      Check& ck = s->checks[idx];
      ck.time = s->age;
      if (ck.time < ck.t0 || ck.time >= ck.t1) continue;
      if (!check_update(*s, ck)) bad = true;
    }
  }
  return !bad;
}

long oracle_run(void* h, double duration, double interval) {
  Sim* s = static_cast<Sim*>(h);
  double chunks = duration / interval;
  long a = 0;
  for (a = 0; a < chunks; a++) {
    if (!callbacks(s)) { s->status |= ST_DROPPED; return a; }
    int steps = static_cast<int>(interval / s->dt);
    for (int i = 0; i < steps; ++i) step(*s);
    s->age += interval;
  }
  for (auto& o : s->oscils) oscil_finalize(o);
  return a;
}

// The analyses over imported samples [k][NS][cells] instead of simulated
// states (what DENSE's --data-import means to do, main.cpp:160-175): sample
// a is written into the current rows, the analyses are called back at age
// t0 + a intervals (accumulated), a failed check stops the run; the
// oscillations are finalized at the end.  Returns the samples analysed.
long oracle_replay(void* h, const double* samples, long k, double t0, double interval) {
  Sim* s = static_cast<Sim*>(h);
  s->age += t0;
  long a = 0;
  for (a = 0; a < k; a++) {
    for (int sp = 0; sp < NS; ++sp) {
      double* row = s->row_ptr(sp, 0);
      for (int c = 0; c < s->cells; ++c) row[c] = samples[(static_cast<size_t>(a) * NS + sp) * s->cells + c];
    }
    if (!callbacks(s)) { s->status |= ST_DROPPED; return a; }
    s->age += interval;
  }
  for (auto& o : s->oscils) oscil_finalize(o);
  return a;
}

int oracle_status(void* h) { return static_cast<Sim*>(h)->status; }
double oracle_age(void* h) { return static_cast<Sim*>(h)->age; }

// Lag-0 state, [species][cell] (what get_concentration(cell, sp) returns).
void oracle_get_state(void* h, double* out) {
  Sim* s = static_cast<Sim*>(h);
  for (int sp = 0; sp < NS; ++sp)
    for (int c = 0; c < s->cells; ++c) out[static_cast<size_t>(sp) * s->cells + c] = s->conc(c, sp);
}

// Whole ring of one species in logical order: row r = lag r (0 = current).
void oracle_get_history(void* h, int sp, double* out) {
  Sim* s = static_cast<Sim*>(h);
  for (int lag = 0; lag < s->h.S[sp]; ++lag) {
    const double* row = s->row_ptr(sp, -lag);
    for (int c = 0; c < s->cells; ++c) out[static_cast<size_t>(lag) * s->cells + c] = row[c];
  }
}

// Analyses are numbered in the order they were added, across kinds.
// Basic results: mins/sums/maxs [n]; per-cell [cells][n]; samples; time.
void oracle_get_basic(void* h, int idx, double* mins, double* sums, double* maxs,
                      double* cmins, double* csums, double* cmaxs, int* samples, double* time) {
  Sim* s = static_cast<Sim*>(h);
  Basic& b = s->basics[s->order[idx] % 65536];
  std::copy(b.mins.begin(), b.mins.end(), mins);
  std::copy(b.sums.begin(), b.sums.end(), sums);
  std::copy(b.maxs.begin(), b.maxs.end(), maxs);
  if (cmins) std::copy(b.cmins.begin(), b.cmins.end(), cmins);
  if (csums) std::copy(b.csums.begin(), b.csums.end(), csums);
  if (cmaxs) std::copy(b.cmaxs.begin(), b.cmaxs.end(), cmaxs);
  *samples = b.samples;
  *time = b.time;
}

// Oscillation results per [species][cell]: amplitude, period, mean peak
// (OscillationAnalysis::show's "avg peak", oscillation.ipp:34-48), number
// of critical points; plus samples and time.
void oracle_get_oscillation(void* h, int idx, double* amps, double* pers, double* avg_peak,
                            int* ncrit, int* samples, double* time) {
  Sim* s = static_cast<Sim*>(h);
  Oscil& o = s->oscils[s->order[idx] % 65536];
  for (size_t k = 0; k < o.amps.size(); ++k) {
    amps[k] = o.amps[k];
    pers[k] = o.pers[k];
    double total = 0.0;
    int peaks = 0;
    for (const Crit& c : o.crits[k]) if (c.is_peak) { ++peaks; total += c.conc; }
    if (peaks != 0) total /= static_cast<double>(peaks);
    avg_peak[k] = total;
    ncrit[k] = static_cast<int>(o.crits[k].size());
  }
  *samples = o.samples;
  *time = o.time;
}

// Critical points of one (species, cell): time, conc, is_peak.
int oracle_get_crits(void* h, int idx, int s, int c, double* t, double* conc, int* is_peak, int cap) {
  Sim* sim = static_cast<Sim*>(h);
  Oscil& o = sim->oscils[sim->order[idx] % 65536];
  const auto& list = o.crits[static_cast<size_t>(s) * (o.cmax - o.cmin) + c];
  int n = static_cast<int>(list.size());
  for (int i = 0; i < n && i < cap; ++i) { t[i] = list[i].time; conc[i] = list[i].conc; is_peak[i] = list[i].is_peak; }
  return n;
}

}  // extern "C"
