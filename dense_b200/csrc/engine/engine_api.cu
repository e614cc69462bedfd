// Host side of the engine: batch set-up and the C ABI of include/dense_b200.h.
//
// Set-up restates, per parameter set, what DENSE's constructors compute:
//   * max_delays per species from the delay reactions that read it
//     (Simulation::calc_max_delays, sim/base.cpp:55-140), traced through the
//     model's own active_rate specialisations;
//   * DENSE's ring size S_sp = (int)(max_delays_sp / dt + 2)
//     (baby_cl.cpp:5-15);
//   * the lags each cell actually reads (the model's active_rate evaluated
//     per cell with a recording context), from which the staged history
//     depth D_sp follows;
//   * the chunk count of run_simulation (chunks a = 0, 1, ... while
//     a < duration / interval) and the steps per chunk (int)(interval / dt)
//     (run_simulation.hpp:127-130, determ.cpp:11).

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <limits>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "dense_model_api.hpp"
#include "reaction_deltas.hpp"
#include "model_impl.hpp"

#include "dense_b200.h"
#include "engine_launch.hpp"
#include "engine_types.hpp"
#include "lag_trace.hpp"

using namespace dense_b200;

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

#define CUDA_TRY(expr)                                                              \
  do {                                                                              \
    cudaError_t e_ = (expr);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return fail(DENSE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Named NVTX ranges on the host timeline (batch set-up, runs, graph capture,
// batched reads); header-only and inert unless a profiler injects a handler.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

struct SetPlan {
  SetDesc d;
  int status = 0;
  bool use_mem = false;         // run by the memory-state kernel (or the wave kernel)
  bool wave = false;            // an ordered set run by the wave kernel
  int mem_block = 256;          // its CTA size
  std::vector<int> lvl_off;     // memory kernel: level offsets into lvl_cells
  std::vector<int> lvl_cells;   // memory kernel: cells in level order
};

// Cell-dependency levels of DENSE's in-order cell loop for reads of the
// row written in the same step: level(c) = 1 + the highest level of c's
// lower-numbered neighbours (0 without any), cells of a level in id order.
void plan_levels(const dense_set_desc& in, bool ordered, SetPlan& plan) {
  const int n = in.num_cells;
  std::vector<int> level(n, 0);
  int n_levels = 1;
  if (ordered) {
    for (int c = 0; c < n; ++c) {
      int l = 0;
      for (int k = in.nbr_offsets[c]; k < in.nbr_offsets[c + 1]; ++k) {
        const int v = in.nbr_ids[k];
        if (v < c) l = std::max(l, level[v] + 1);
      }
      level[c] = l;
      n_levels = std::max(n_levels, l + 1);
    }
  }
  plan.lvl_off.assign(n_levels + 1, 0);
  for (int c = 0; c < n; ++c) plan.lvl_off[level[c] + 1]++;
  for (int l = 0; l < n_levels; ++l) plan.lvl_off[l + 1] += plan.lvl_off[l];
  plan.lvl_cells.assign(n, 0);
  std::vector<int> fill(plan.lvl_off.begin(), plan.lvl_off.end() - 1);
  for (int c = 0; c < n; ++c) plan.lvl_cells[fill[level[c]]++] = c;
  plan.d.n_levels = n_levels;
}

struct DeviceBuffer {
  void* p = nullptr;
  size_t bytes = 0;
  ~DeviceBuffer() {
    if (p) cudaFree(p);
  }
  int alloc(size_t n) {
    bytes = n;
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      p = nullptr;
      return fail(DENSE_ERR_MEMORY, std::string("cudaMalloc(") + std::to_string(n) + "): " + cudaGetErrorString(e));
    }
    return DENSE_OK;
  }
};

}  // namespace

struct dense_engine {
  int device = 0;
  int precision = DENSE_FP64;
  int num_sets = 0;
  cudaStream_t stream = nullptr;
  StepArgs args{};
  size_t smem = 0;
  int64_t total_cell_steps = 0;
  int64_t device_bytes = 0;
  int64_t anl_block = 0;  // doubles of analysis state per set
  std::vector<SetDesc> sets;
  std::vector<AnalysisDesc> analyses;
  std::vector<int> init_status;
  DeviceBuffer d_sets, d_prog, d_params, d_nbr_off, d_nbr_idx, d_state, d_ring, d_anl, d_init_conc,
      d_init_status, d_lists, d_lvl_off, d_lvl_cells, d_wave_rec;
  int n_reg = 0, n_mem = 0;  // sets run by the register / memory kernels (d_lists: reg then mem)
  // memory- and wave-kernel sets in launch groups of one kernel, CTA size
  // and dynamic shared memory: (kernel: 0 memory, 1 wave, 2 wave with
  // everything shared; threads; shared bytes; first index in the mem list;
  // count)
  std::vector<std::array<int, 5>> mem_groups;
  std::map<int, cudaGraphExec_t> graphs;
  // the kernel launches of one run (register kernel, one per memory- or
  // wave-kernel group) fork onto side streams of their own so that they run
  // concurrently; launch k goes to side[k], whose priority ranks the
  // group's longest set (the block scheduler starts the CTAs of
  // higher-priority streams first)
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev_join;
  cudaEvent_t ev_fork = nullptr;
  ~dense_engine() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    for (auto& x : side) cudaStreamDestroy(x);
    for (auto& x : ev_join) cudaEventDestroy(x);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// ring sizes and traced depths for one set
int next_pow2(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Input checks of one set (CSR tissue, sizes, hints).
int check_set(const dense_set_desc& in, const std::string& where) {
  if (in.num_cells <= 0 || in.num_cells > kMaxCells)
    return fail(DENSE_ERR_UNSUPPORTED, where + "1.." + std::to_string(kMaxCells) + " cells per set are supported");
  if (!in.nbr_offsets || !in.nbr_ids || !in.set_params) return fail(DENSE_ERR_INVALID, where + "null input");
  if (!(in.duration >= 0.0)) return fail(DENSE_ERR_INVALID, where + "negative duration");
  const int n = in.num_cells;
  if (in.nbr_offsets[0] != 0) return fail(DENSE_ERR_INVALID, where + "CSR offsets must start at 0");
  for (int c = 0; c < n; ++c) {
    if (in.nbr_offsets[c + 1] < in.nbr_offsets[c]) return fail(DENSE_ERR_INVALID, where + "CSR offsets decrease");
    for (int k = in.nbr_offsets[c]; k < in.nbr_offsets[c + 1]; ++k) {
      const int v = in.nbr_ids[k];
      if (v < 0 || v >= n) return fail(DENSE_ERR_INVALID, where + "neighbour id outside the tissue");
      if (k > in.nbr_offsets[c] && in.nbr_ids[k - 1] >= v)
        return fail(DENSE_ERR_INVALID, where + "neighbour ids must ascend (DENSE keeps them in a std::set)");
    }
  }
  if (in.schedule < DENSE_SCHEDULE_AUTO || in.schedule > DENSE_SCHEDULE_REGISTER)
    return fail(DENSE_ERR_INVALID, where + "unknown schedule hint");
  if (in.mem_block != 0 && (in.mem_block < 32 || in.mem_block > 256 || in.mem_block % 32))
    return fail(DENSE_ERR_INVALID, where + "mem_block must be 32..256, a multiple of 32");
  return DENSE_OK;
}

// The analyses of a run (analyses.xml entries) and the doubles of analysis
// state each set of the batch holds.
int build_analyses(const dense_run_desc* run, int num_sets, const dense_set_desc* in_sets,
                   std::vector<AnalysisDesc>& out, int64_t& anl_block_out) {
  const double interval = run->analysis_interval;
  int min_cells = kMaxCells + 1;
  for (int s = 0; s < num_sets; ++s) min_cells = std::min(min_cells, in_sets[s].num_cells);
  int64_t anl_block = 0;
  for (int ai = 0; ai < run->num_analyses; ++ai) {
    const dense_analysis_desc& in = run->analyses[ai];
    AnalysisDesc A{};
    A.kind = in.kind;
    A.cmin = in.cell_start;
    A.cmax = in.cell_end;
    A.t0 = in.time_start;
    A.t1 = in.time_end;
    if (A.cmin < 0 || A.cmax < A.cmin || A.cmax > min_cells)
      return fail(DENSE_ERR_INVALID, "analysis " + std::to_string(ai) + ": cell range outside the tissue");
    if (in.kind == DENSE_ANALYSIS_CONCCHECK && in.num_species == 0) {
      A.nsp = NUM_SPECIES;
      for (int i = 0; i < NUM_SPECIES; ++i) A.sp[i] = i;
    } else {
      if (in.num_species <= 0 || in.num_species > NUM_SPECIES || !in.species)
        return fail(DENSE_ERR_INVALID, "analysis " + std::to_string(ai) + ": bad species list");
      A.nsp = in.num_species;
      for (int i = 0; i < in.num_species; ++i) {
        if (in.species[i] < 0 || in.species[i] >= NUM_SPECIES)
          return fail(DENSE_ERR_INVALID, "analysis " + std::to_string(ai) + ": bad species id");
        A.sp[i] = in.species[i];
      }
    }
    const int64_t m = A.cmax - A.cmin;
    A.off = anl_block;
    if (in.kind == DENSE_ANALYSIS_BASIC) {
      anl_block += 3 * A.nsp + 2 + 3 * m * A.nsp;
    } else if (in.kind == DENSE_ANALYSIS_OSCILLATION) {
      if (!(in.anlys_intvl > 0.0) || !(in.win_range >= 0.0))
        return fail(DENSE_ERR_INVALID, "oscillation: bad window");
      const double rs = in.win_range / in.anlys_intvl;  // oscillation.hpp:64
      if (!(rs < 1e6)) return fail(DENSE_ERR_UNSUPPORTED, "oscillation window too long");
      A.range_steps = static_cast<int>(rs);
      A.interval = in.anlys_intvl;
      anl_block += 2 + m * A.nsp * kOscFields + static_cast<int64_t>(A.nsp) * (A.range_steps + 1) * m;
    } else if (in.kind == DENSE_ANALYSIS_CONCCHECK) {
      A.lo = in.lower;
      A.hi = in.upper;
      anl_block += 1;
    } else if (in.kind == DENSE_ANALYSIS_TRAJECTORY) {
      // room for every sample inside [time_start, time_end) of the longest
      // horizon in the batch
      // (sets with a negative or NaN duration are rejected by check_set)
      int cap = 0;
      for (int s = 0; s < num_sets; ++s) {
        const double dur = in_sets[s].duration;
        if (!(dur >= 0.0)) continue;
        const double t1 = std::min(in.time_end, dur), t0 = std::max(in.time_start, 0.0);
        const double all = std::ceil(dur / interval);
        const double in_window = t1 > t0 ? std::ceil((t1 - t0) / interval) + 2.0 : 0.0;
        const double c = std::min(all, in_window);
        if (!(c < 1e9)) return fail(DENSE_ERR_UNSUPPORTED, "trajectory: too many samples");
        cap = std::max(cap, static_cast<int>(c));
      }
      A.range_steps = cap;
      anl_block += 2 + cap + static_cast<int64_t>(cap) * A.nsp * m;
    } else {
      return fail(DENSE_ERR_INVALID, "unknown analysis kind");
    }
    anl_block = (anl_block + 1) & ~int64_t(1);
    out.push_back(A);
  }

  anl_block_out = anl_block;
  return DENSE_OK;
}

int plan_set(const dense_set_desc& in, double dt, int elem_bytes, SetPlan& plan, std::vector<double>& cell_params) {
  const bool force_mem = in.schedule != DENSE_SCHEDULE_AUTO && in.schedule != DENSE_SCHEDULE_REGISTER;
  const int n = in.num_cells;
  SetDesc& d = plan.d;
  d.n_cells = n;
  // DENSE's ring sizes (base.cpp:55-140, baby_cl.cpp:10)
  if (!ring_sizes(in, dt, d.S)) return fail(DENSE_ERR_INVALID, "a ring size is not a positive int");
  // parameters for the device: one row [NP] when every cell uses the set's
  // parameters, else [NP][n]; NaN rates/delays reject the set, as DENSE's
  // getRate/getDelay throw (sim/base.hpp:398-412)
  const int pcols = in.cell_params ? n : 1;
  d.param_stride = in.cell_params ? n : 0;
  cell_params.resize(static_cast<size_t>(NUM_PARAMS) * pcols);
  for (int c = 0; c < pcols; ++c) {
    const double* p = in.cell_params ? in.cell_params + static_cast<size_t>(c) * NUM_PARAMS : in.set_params;
    for (int i = 0; i < NUM_PARAMS; ++i) {
      cell_params[static_cast<size_t>(i) * pcols + c] = p[i];
      if (i < NUM_REACTIONS + NUM_DELAY_REACTIONS && std::isnan(p[i])) plan.status |= kSetNanParam;
    }
  }
  // traced lags; cells sharing the set's parameters all read the same
  // lags, so one is traced
  LagTrace tr;
  trace_lags(cell_params.data(), in.cell_params ? n : 1, 1, pcols, d.S, tr);
  const int* own_max = tr.own_max;
  const int* nbr_max = tr.nbr_max;
  const bool* ord_sp = tr.ord_sp;
  const int* plain_min = tr.plain_min;
  const int* plain_max = tr.plain_max;
  const bool ordered = tr.ordered, bad = tr.bad;
  if (bad) plan.status |= kSetBadDelay;
  // sets whose neighbour reads see the row written in the same step, and
  // sets larger than a CTA, run in the memory-state kernel, which keeps
  // every species in its ring (at least two rows)
  d.ordered = ordered ? 1 : 0;
  plan.use_mem = ordered || n > kStepThreads || force_mem;
  plan_levels(in, ordered, plan);
  // the wave kernel takes ordered sets whose cells have at most
  // kWaveMaxNbrs neighbours and whose ids and level offsets fit 16 bits
  // (and, on request, sets without such reads: the wave kernel's rows in
  // shared memory as far as they fit, one level per step)
  if ((ordered || in.schedule == DENSE_SCHEDULE_SHARED_ROWS) && in.schedule != DENSE_SCHEDULE_GLOBAL && n < 65536 &&
      2 * static_cast<int64_t>(plan.lvl_off.size()) + 16 <= kWaveSmemBudget) {
    plan.wave = true;
    for (int c = 0; c < n; ++c)
      if (in.nbr_offsets[c + 1] - in.nbr_offsets[c] > kWaveMaxNbrs) plan.wave = false;
  }
  // memory-kernel CTA size: the hint, else the widest level in warps (32..256)
  int widest = 0;
  for (size_t l = 0; l + 1 < plan.lvl_off.size(); ++l) widest = std::max(widest, plan.lvl_off[l + 1] - plan.lvl_off[l]);
  plan.mem_block = in.mem_block > 0 ? in.mem_block : std::min(256, std::max(32, (widest + 31) / 32 * 32));
  int64_t off = 0;
  for (int sp = 0; sp < NUM_SPECIES; ++sp) {
    int depth = 0;
    if (own_max[sp] >= 1) depth = own_max[sp] + 1;
    if (nbr_max[sp] >= 0) depth = std::max(depth, nbr_max[sp] + 2);
    if (plan.use_mem) depth = std::max(depth, 2);
    // a power of two, so a row is (step - lag) & (D - 1); the wave kernel
    // indexes rows modulo D and keeps exactly the rows it reads
    d.D[sp] = depth > 0 ? (plan.wave ? depth : next_pow2(depth)) : 0;
    depth = d.D[sp];
    d.ring_off[sp] = off;
    off += static_cast<int64_t>(depth) * n;
  }
  // wave kernel shared memory, filled in priority order while it fits:
  // the rows of the species read at lag S-1, the FP32 Kahan terms (every
  // cell reads and writes them each step), the cell records, the rows of
  // other neighbour-read species, then (unless the hint keeps them global)
  // the rest; the 16-bit level offsets always, at the end
  d.wave = plan.wave ? 1 : 0;
  d.topo_off = -1;
  d.comp_smem_off = -1;
  d.lvl_smem_off = 0;
  d.smem_bytes = 0;
  for (int sp = 0; sp < NUM_SPECIES; ++sp) d.smem_off[sp] = -1;
  if (plan.wave) {
    const int64_t lvl_bytes = (2 * static_cast<int64_t>(plan.lvl_off.size()) + 15) / 16 * 16;
    int64_t used = 0;
    auto take = [&](int64_t bytes) -> int64_t {
      bytes = (bytes + 15) / 16 * 16;
      if (used + bytes + lvl_bytes > kWaveSmemBudget) return -1;
      const int64_t at = used;
      used += bytes;
      return at;
    };
    const bool global_rows = in.schedule == DENSE_SCHEDULE_WAVE_GLOBAL;
    for (int sp = 0; sp < NUM_SPECIES && !global_rows; ++sp)
      if (ord_sp[sp]) d.smem_off[sp] = static_cast<int>(take(static_cast<int64_t>(d.D[sp]) * n * elem_bytes));
    if (elem_bytes == 4 && !global_rows && in.schedule != DENSE_SCHEDULE_SHARED_NEIGHBOUR)
      d.comp_smem_off = static_cast<int>(take(static_cast<int64_t>(NUM_SPECIES) * n * elem_bytes));
    d.topo_off = global_rows ? -1 : static_cast<int>(take(16 * static_cast<int64_t>(n)));
    for (int pass = 0; pass < 2 && !global_rows; ++pass) {
      if (pass == 1 && in.schedule == DENSE_SCHEDULE_SHARED_NEIGHBOUR) break;
      for (int sp = 0; sp < NUM_SPECIES; ++sp)
        if (d.smem_off[sp] < 0 && (pass == 1 || nbr_max[sp] >= 0))
          d.smem_off[sp] = static_cast<int>(take(static_cast<int64_t>(d.D[sp]) * n * elem_bytes));
    }
    d.lvl_smem_off = static_cast<int>(used);
    d.smem_bytes = static_cast<int>(used + lvl_bytes);
  }
  // Time pipelining of the wave kernel.  Step k's level l runs in interval
  // T(k, l) = k * delta + l, intervals separated by barriers.  A read of a
  // neighbour v's row must come after the interval that wrote it and
  // before the one that overwrites its slot (rows are kept modulo D):
  //   lag-(S-1) read of v > c: row k+1-S, written in step k-S and rewritten
  //     in step k-S+D:   l_v - l_c < S delta,   l_c - l_v < (D - S) delta;
  //   read at another lag m:  l_v - l_c < (m + 1) delta,
  //                           l_c - l_v < (D - m - 1) delta;
  //   lag-(S-1) read of v < c reads this step's row (lower levels) only.
  // delta is the least integer meeting every such bound; the steps in flight
  // are ceil(L / delta), at most kWaveMaxFronts.
  d.wave_delta = 0;
  d.wave_fronts = 1;
  if (plan.wave) {
    const int L = static_cast<int>(plan.lvl_off.size()) - 1;
    std::vector<int> level(n, 0);
    for (int l = 0; l < L; ++l)
      for (int i = plan.lvl_off[l]; i < plan.lvl_off[l + 1]; ++i) level[plan.lvl_cells[i]] = l;
    int64_t delta = 1;
    bool pipe = true;
    // delta > num / den
    auto need = [&](int64_t num, int64_t den) {
      if (den <= 0) {
        if (num >= 0) pipe = false;
        return;
      }
      if (num >= 0) delta = std::max(delta, num / den + 1);
    };
    for (int c = 0; c < n && pipe; ++c)
      for (int k = in.nbr_offsets[c]; k < in.nbr_offsets[c + 1]; ++k) {
        const int v = in.nbr_ids[k];
        const int64_t dl = level[v] - level[c];
        for (int sp = 0; sp < NUM_SPECIES; ++sp) {
          if (ord_sp[sp] && v > c) {
            need(dl, d.S[sp]);
            need(-dl, d.D[sp] - d.S[sp]);
          }
          if (plain_max[sp] >= 0) {
            need(dl, plain_min[sp] + 1);
            need(-dl, d.D[sp] - plain_max[sp] - 1);
          }
        }
      }
    int fronts = pipe ? static_cast<int>((L + delta - 1) / delta) : 1;
    fronts = std::max(1, std::min(fronts, kWaveMaxFronts));
    // a CTA-size hint caps the fronts at one warp each
    if (in.mem_block > 0) fronts = std::max(1, std::min(fronts, in.mem_block / 32));
    // fewer fronts than the bound allows: space the steps further apart
    delta = std::max<int64_t>(delta, (L + fronts - 1) / fronts);
    d.wave_delta = static_cast<int>(std::max<int64_t>(delta, 1));
    d.wave_fronts = fronts;
    // a thread group per front: the widest level in warps, or the hint's
    // share; the whole CTA at most 256 threads
    int widest = 0;
    for (int l = 0; l < L; ++l) widest = std::max(widest, plan.lvl_off[l + 1] - plan.lvl_off[l]);
    int group = in.mem_block > 0 ? in.mem_block / fronts : (widest + 31) / 32 * 32;
    group = std::max(32, std::min(group, 256 / fronts) / 32 * 32);
    plan.mem_block = group * fronts;
  }
  // chunk count: a = 0, 1, ... while a < duration / interval
  return DENSE_OK;
}

// Dynamic shared memory of a wave-kernel launch group holding a set that
// needs `bytes`: a few fixed sizes, so sets of similar size share a launch.
int wave_smem_bucket(int bytes) {
  static const int kb[] = {1, 2, 4, 8, 16, 24, 32, 48, 64, 80, 96, 112, 128, 160, 192};
  for (int k : kb)
    if (bytes <= k * 1024) return k * 1024;
  return kWaveSmemBudget;
}

int64_t ring_elems(const SetDesc& d) {
  int64_t t = 0;
  for (int sp = 0; sp < NUM_SPECIES; ++sp) t += static_cast<int64_t>(d.D[sp]) * d.n_cells;
  return t;
}

}  // namespace

extern "C" {

int dense_model_get_info(dense_model_info* out) {
  if (!out) return fail(DENSE_ERR_INVALID, "null out");
  out->num_species = NUM_SPECIES;
  out->num_reactions = NUM_REACTIONS;
  out->num_delay_reactions = NUM_DELAY_REACTIONS;
  out->num_critical_species = NUM_CRITICAL_SPECIES;
  out->num_params = NUM_PARAMS;
  return DENSE_OK;
}

const char* dense_model_specie_name(int i) { return (i >= 0 && i < NUM_SPECIES) ? dense_specie_names[i] : nullptr; }
const char* dense_model_reaction_name(int i) { return (i >= 0 && i < NUM_REACTIONS) ? dense_reaction_names[i] : nullptr; }
const char* dense_model_delay_reaction_name(int d) {
  return (d >= 0 && d < NUM_DELAY_REACTIONS) ? dense_reaction_names[dense_delay_reaction_of[d]] : nullptr;
}
const char* dense_model_critical_specie_name(int c) {
  return (c >= 0 && c < NUM_CRITICAL_SPECIES) ? dense_specie_names[dense_critical_species_of[c]] : nullptr;
}
const char* dense_last_error(void) { return g_error.c_str(); }

int dense_engine_create(const dense_run_desc* run, int num_sets, const dense_set_desc* in_sets,
                        dense_engine** out) {
  NvtxRange range_("dense_engine_create");
  if (!run || !out || num_sets <= 0 || !in_sets) return fail(DENSE_ERR_INVALID, "null argument or no sets");
  *out = nullptr;
  if (!(run->step_size > 0.0) || !(run->analysis_interval > 0.0))
    return fail(DENSE_ERR_INVALID, "step size and analysis interval must be positive");
  if (run->precision != DENSE_FP64 && run->precision != DENSE_FP32_KAHAN)
    return fail(DENSE_ERR_INVALID, "unknown precision");
  if (run->num_analyses < 0 || run->num_analyses > kMaxAnalyses)
    return fail(DENSE_ERR_UNSUPPORTED, "at most " + std::to_string(kMaxAnalyses) + " analyses per batch");
  const double dt = run->step_size, interval = run->analysis_interval;
  const double steps_d = interval / dt;  // determ.cpp:11
  if (!(steps_d < 2147483647.0)) return fail(DENSE_ERR_INVALID, "interval / step size too large");
  const int steps_per_chunk = static_cast<int>(steps_d);

  std::unique_ptr<dense_engine> e(new dense_engine());
  e->device = run->device;
  e->precision = run->precision;
  e->num_sets = num_sets;
  CUDA_TRY(cudaSetDevice(run->device));

  // ---- analyses
  int64_t anl_block = 0;
  {
    const int rc = build_analyses(run, num_sets, in_sets, e->analyses, anl_block);
    if (rc != DENSE_OK) return rc;
  }

  // ---- sets
  std::vector<double> params_all, conc_all(static_cast<size_t>(num_sets) * NUM_SPECIES, 0.0);
  std::vector<int> off_all, idx_all;
  int64_t cells_total = 0, ring_total = 0;
  int max_cells = 0, max_edges = 0;
  std::vector<int> reg_list, mem_list, mem_block_of, mem_smem_of, mem_kind_of, lvl_off_all, lvl_cells_all;
  std::vector<uint16_t> rec_all;  // wave-kernel cell records, 8 x 16 bits each
  e->sets.resize(num_sets);
  e->init_status.resize(num_sets);
  std::vector<double> cp;
  for (int s = 0; s < num_sets; ++s) {
    const dense_set_desc& in = in_sets[s];
    const std::string where = "set " + std::to_string(s) + ": ";
    {
      const int rc = check_set(in, where);
      if (rc != DENSE_OK) return rc;
    }
    const int n = in.num_cells;
    SetPlan plan;
    int rc = plan_set(in, dt, run->precision == DENSE_FP64 ? 8 : 4, plan, cp);
    if (rc != DENSE_OK) return fail(rc, where + g_error);
    SetDesc& d = plan.d;
    const double chunks = in.duration / interval;  // run_simulation.hpp:127
    if (!(chunks < 2147483647.0)) return fail(DENSE_ERR_INVALID, where + "too many chunks");
    d.n_chunks = static_cast<int>(std::ceil(chunks));
    d.steps_per_chunk = steps_per_chunk;
    d.param_base = static_cast<int64_t>(params_all.size());
    d.cell_base = cells_total;
    d.nbr_base = static_cast<int64_t>(off_all.size());
    d.ring_base = ring_total;
    d.anl_base = anl_block * s;
    e->anl_block = anl_block;
    const int e0 = static_cast<int>(idx_all.size());
    for (int c = 0; c <= n; ++c) off_all.push_back(e0 + in.nbr_offsets[c]);
    idx_all.insert(idx_all.end(), in.nbr_ids, in.nbr_ids + in.nbr_offsets[n]);
    params_all.insert(params_all.end(), cp.begin(), cp.end());
    if (in.init_conc)
      for (int sp = 0; sp < NUM_SPECIES; ++sp) conc_all[static_cast<size_t>(s) * NUM_SPECIES + sp] = in.init_conc[sp];
    // a set whose reads alias rows written in the same step (Gauss-Seidel
    // order, e.g. neighbour averages with delay 1 and no delay reactions)
    // is not run by this schedule
    e->init_status[s] = plan.status;
    cells_total += n;
    ring_total += ring_elems(d);
    ring_total = (ring_total + 31) & ~int64_t(31);
    if (plan.use_mem) {
      mem_list.push_back(s);
      mem_block_of.push_back(plan.mem_block);
      mem_smem_of.push_back(plan.wave ? wave_smem_bucket(d.smem_bytes) : -1);
      bool all_shared = plan.wave && d.topo_off >= 0;
      for (int sp = 0; sp < NUM_SPECIES; ++sp) all_shared = all_shared && d.smem_off[sp] >= 0;
      mem_kind_of.push_back(plan.wave ? (all_shared ? 2 : 1) : 0);
      d.lvl_base = static_cast<int64_t>(lvl_off_all.size());
      lvl_off_all.insert(lvl_off_all.end(), plan.lvl_off.begin(), plan.lvl_off.end());
    } else {
      reg_list.push_back(s);
      max_cells = std::max(max_cells, n);
      max_edges = std::max(max_edges, in.nbr_offsets[n]);
    }
    lvl_cells_all.insert(lvl_cells_all.end(), plan.lvl_cells.begin(), plan.lvl_cells.end());
    if (plan.wave) {
      // cell records in level order: {cell, neighbour count, ids (ascending), 0...}
      d.rec_base = static_cast<int64_t>(rec_all.size() / 8);
      for (int i = 0; i < n; ++i) {
        const int c = plan.lvl_cells[i];
        const int k0 = in.nbr_offsets[c], cnt = in.nbr_offsets[c + 1] - k0;
        uint16_t r[8] = {static_cast<uint16_t>(c), static_cast<uint16_t>(cnt), 0, 0, 0, 0, 0, 0};
        for (int e = 0; e < cnt; ++e) r[2 + e] = static_cast<uint16_t>(in.nbr_ids[k0 + e]);
        rec_all.insert(rec_all.end(), r, r + 8);
      }
    }
    e->total_cell_steps += static_cast<int64_t>(n) * d.n_chunks * steps_per_chunk;
    e->sets[s] = d;
  }

  // ---- device buffers
  CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  const size_t tsz = run->precision == DENSE_FP64 ? sizeof(double) : sizeof(float);
  int rc;
  if ((rc = e->d_sets.alloc(sizeof(SetDesc) * num_sets))) return rc;
  if ((rc = e->d_prog.alloc(sizeof(SetProgress) * num_sets))) return rc;
  if ((rc = e->d_params.alloc(tsz * params_all.size()))) return rc;
  if ((rc = e->d_nbr_off.alloc(sizeof(int) * off_all.size()))) return rc;
  if ((rc = e->d_nbr_idx.alloc(sizeof(int) * idx_all.size()))) return rc;
  if ((rc = e->d_state.alloc(tsz * 2 * NUM_SPECIES * cells_total))) return rc;
  if ((rc = e->d_ring.alloc(tsz * ring_total))) return rc;
  if ((rc = e->d_anl.alloc(sizeof(double) * anl_block * num_sets))) return rc;
  if ((rc = e->d_init_conc.alloc(sizeof(double) * conc_all.size()))) return rc;
  if ((rc = e->d_init_status.alloc(sizeof(int) * num_sets))) return rc;
  if ((rc = e->d_lists.alloc(sizeof(int) * num_sets))) return rc;
  if ((rc = e->d_lvl_off.alloc(sizeof(int) * std::max<size_t>(1, lvl_off_all.size())))) return rc;
  if ((rc = e->d_lvl_cells.alloc(sizeof(int) * lvl_cells_all.size()))) return rc;
  if ((rc = e->d_wave_rec.alloc(sizeof(uint16_t) * rec_all.size()))) return rc;
  e->n_reg = static_cast<int>(reg_list.size());
  e->n_mem = static_cast<int>(mem_list.size());
  {
    // longest sets first (cells x Euler steps): CTAs start in list order, so
    // uneven horizons finish close together (longest-processing-time order)
    auto cost = [&](int i) {
      return static_cast<int64_t>(e->sets[i].n_cells) * e->sets[i].n_chunks * e->sets[i].steps_per_chunk;
    };
    auto by_cost = [&](int x, int y) { return cost(x) != cost(y) ? cost(x) > cost(y) : x < y; };
    std::stable_sort(reg_list.begin(), reg_list.end(), by_cost);
    // memory- and wave-kernel sets: grouped by kernel, CTA size and shared
    // memory bucket (-1: memory kernel), longest first in a group
    // key: (kernel: 0 memory, 1 wave, 2 wave with everything shared; shared
    // memory bucket; CTA size)
    std::vector<std::array<int, 3>> key_of(num_sets, {0, 0, 0});
    for (size_t k = 0; k < mem_list.size(); ++k)
      key_of[mem_list[k]] = {mem_kind_of[k], std::max(0, mem_smem_of[k]), mem_block_of[k]};
    std::stable_sort(mem_list.begin(), mem_list.end(), [&](int x, int y) {
      return key_of[x] != key_of[y] ? key_of[x] < key_of[y] : by_cost(x, y);
    });
    for (size_t k = 0; k < mem_list.size(); ++k) {
      const auto key = key_of[mem_list[k]];
      if (e->mem_groups.empty() || e->mem_groups.back()[0] != key[0] || e->mem_groups.back()[1] != key[2] ||
          e->mem_groups.back()[2] != key[1])
        e->mem_groups.push_back({key[0], key[2], key[1], static_cast<int>(k), 0});
      e->mem_groups.back()[4]++;
    }
    std::vector<int> lists(reg_list);
    lists.insert(lists.end(), mem_list.begin(), mem_list.end());
    CUDA_TRY(cudaMemcpyAsync(e->d_lists.p, lists.data(), sizeof(int) * num_sets, cudaMemcpyHostToDevice, e->stream));
    if (!lvl_off_all.empty())
      CUDA_TRY(cudaMemcpyAsync(e->d_lvl_off.p, lvl_off_all.data(), sizeof(int) * lvl_off_all.size(),
                               cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaMemcpyAsync(e->d_lvl_cells.p, lvl_cells_all.data(), sizeof(int) * lvl_cells_all.size(),
                             cudaMemcpyHostToDevice, e->stream));
    if (!rec_all.empty())
      CUDA_TRY(cudaMemcpyAsync(e->d_wave_rec.p, rec_all.data(), sizeof(uint16_t) * rec_all.size(),
                               cudaMemcpyHostToDevice, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
  }
  {
    // one side stream per launch, prioritised by the group's longest set in
    // dependent steps: Euler steps x levels (x cells per thread for the
    // memory kernel); register-kernel sets count one level per step
    std::vector<std::pair<double, int>> est;  // (latency estimate, launch index)
    int k = 0;
    if (e->n_reg > 0) {
      double m = 0;
      for (int i : reg_list) m = std::max(m, static_cast<double>(e->sets[i].n_chunks) * e->sets[i].steps_per_chunk);
      est.push_back({m, k++});
    }

    for (const auto& g : e->mem_groups) {
      double m = 0;
      for (int j = g[3]; j < g[3] + g[4]; ++j) {
        const SetDesc& d = e->sets[mem_list[j]];
        const double per_step = g[0] ? d.wave_delta : d.n_levels * std::ceil(static_cast<double>(d.n_cells) /
                                                                            (d.n_levels * g[1]));
        m = std::max(m, static_cast<double>(d.n_chunks) * d.steps_per_chunk * per_step);
      }
      est.push_back({m, k++});
    }
    std::stable_sort(est.begin(), est.end(), [](const std::pair<double, int>& x, const std::pair<double, int>& y) {
      return x.first > y.first;
    });
    int least = 0, greatest = 0;
    CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    std::vector<int> prio(est.size(), least);
    for (size_t r = 0; r < est.size(); ++r) prio[est[r].second] = std::min(least, greatest + static_cast<int>(r));
    CUDA_TRY(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
    for (size_t i = 0; i < est.size(); ++i) {
      cudaStream_t x;
      cudaEvent_t ev;
      CUDA_TRY(cudaStreamCreateWithPriority(&x, cudaStreamNonBlocking, prio[i]));
      e->side.push_back(x);
      CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      e->ev_join.push_back(ev);
    }
  }
  CUDA_TRY(cudaMemcpyAsync(e->d_sets.p, e->sets.data(), sizeof(SetDesc) * num_sets, cudaMemcpyHostToDevice, e->stream));
  std::vector<float> params_f;
  if (run->precision == DENSE_FP64) {
    CUDA_TRY(cudaMemcpyAsync(e->d_params.p, params_all.data(), sizeof(double) * params_all.size(),
                             cudaMemcpyHostToDevice, e->stream));
  } else {
    params_f.assign(params_all.begin(), params_all.end());
    CUDA_TRY(cudaMemcpyAsync(e->d_params.p, params_f.data(), sizeof(float) * params_f.size(),
                             cudaMemcpyHostToDevice, e->stream));
  }
  CUDA_TRY(cudaMemcpyAsync(e->d_nbr_off.p, off_all.data(), sizeof(int) * off_all.size(), cudaMemcpyHostToDevice, e->stream));
  if (!idx_all.empty())
    CUDA_TRY(cudaMemcpyAsync(e->d_nbr_idx.p, idx_all.data(), sizeof(int) * idx_all.size(), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaMemcpyAsync(e->d_init_conc.p, conc_all.data(), sizeof(double) * conc_all.size(), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaMemcpyAsync(e->d_init_status.p, e->init_status.data(), sizeof(int) * num_sets, cudaMemcpyHostToDevice, e->stream));
  e->device_bytes = static_cast<int64_t>(e->d_sets.bytes + e->d_prog.bytes + e->d_params.bytes + e->d_nbr_off.bytes +
                                         e->d_nbr_idx.bytes + e->d_state.bytes + e->d_ring.bytes + e->d_anl.bytes +
                                         e->d_init_conc.bytes + e->d_init_status.bytes);

  StepArgs& a = e->args;
  a.sets = static_cast<const SetDesc*>(e->d_sets.p);
  a.prog = static_cast<SetProgress*>(e->d_prog.p);
  a.params = e->d_params.p;
  a.nbr_off = static_cast<const int*>(e->d_nbr_off.p);
  a.nbr_idx = static_cast<const int*>(e->d_nbr_idx.p);
  a.state = e->d_state.p;
  a.ring = e->d_ring.p;
  a.anl = static_cast<double*>(e->d_anl.p);
  a.lvl_off = static_cast<const int*>(e->d_lvl_off.p);
  a.lvl_cells = static_cast<const int*>(e->d_lvl_cells.p);
  a.wave_rec = static_cast<const uint4*>(e->d_wave_rec.p);
  for (size_t i = 0; i < e->analyses.size(); ++i) a.analyses[i] = e->analyses[i];
  a.n_analyses = static_cast<int>(e->analyses.size());
  a.num_sets = num_sets;
  a.dt = dt;
  a.interval = interval;
  a.chunk_count = -1;
  a.block_threads = std::max(32, (max_cells + 31) / 32 * 32);
  a.uniform_params = 1;
  for (const SetDesc& d : e->sets)
    if (d.param_stride != 0) a.uniform_params = 0;
  // shared memory: sampled state (with analyses), truncated delays, and
  // each set's neighbour ids when the largest list fits
  // rows of the sampled-state buffer: the species some analysis observes
  a.n_vals = 0;
  for (int sp = 0; sp < NUM_SPECIES; ++sp) a.val_slot[sp] = -1;
  for (auto& A : e->analyses)
    for (int i = 0; i < A.nsp; ++i)
      if (a.val_slot[A.sp[i]] < 0) a.val_slot[A.sp[i]] = a.n_vals++;
  for (int i = 0; i < a.n_analyses; ++i)
    for (int k = 0; k < a.analyses[i].nsp; ++k) a.analyses[i].slot[k] = a.val_slot[a.analyses[i].sp[k]];
  e->analyses.assign(a.analyses, a.analyses + a.n_analyses);
  size_t smem = (a.n_analyses > 0 ? sizeof(double) * a.n_vals * a.block_threads : 0) +
                sizeof(int) * NUM_DELAY_REACTIONS * a.block_threads;
  const size_t csr_bytes = sizeof(int) * max_edges;
  const size_t smem_cap = a.block_threads <= 224 ? 100000 : 200000;
  a.csr_in_smem = smem + csr_bytes <= smem_cap ? 1 : 0;
  if (a.csr_in_smem) smem += csr_bytes;
  if (smem > smem_cap) return fail(DENSE_ERR_UNSUPPORTED, "shared memory need of the batch too large");
  e->smem = smem;

  rc = dense_engine_reset(e.get(), nullptr);
  if (rc != DENSE_OK) return rc;
  *out = e.release();
  return DENSE_OK;
}

int dense_engine_reset(dense_engine* e, void* stream) {
  NvtxRange range_("dense_engine_reset");
  if (!e) return fail(DENSE_ERR_INVALID, "null engine");
  CUDA_TRY(cudaSetDevice(e->device));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : e->stream;
  const double* ic = static_cast<const double*>(e->d_init_conc.p);
  const int* is = static_cast<const int*>(e->d_init_status.p);
  CUDA_TRY(e->precision == DENSE_FP64 ? launch_init_fp64(e->args, ic, is, s) : launch_init_fp32(e->args, ic, is, s));
  return DENSE_OK;
}

// One run: the register kernel over its sets, the memory or wave kernel
// once per group.  Every launch goes to its own side stream forked from `s`
// and joined back into it, so the kernels share the GPU instead of running
// one after the other (in a captured graph they become parallel branches
// that keep their priorities).
static cudaError_t launch_all(dense_engine* e, const StepArgs& a, cudaStream_t s) {
  const int* reg = static_cast<const int*>(e->d_lists.p);
  const int* mem = reg + e->n_reg;
  cudaError_t r;
  if ((r = cudaEventRecord(e->ev_fork, s)) != cudaSuccess) return r;
  int k = 0;  // launches issued so far
  auto stream_for = [&](cudaStream_t& st) -> cudaError_t {
    st = e->side[k];
    return cudaStreamWaitEvent(st, e->ev_fork, 0);
  };
  auto join = [&](cudaStream_t st) -> cudaError_t {
    cudaError_t rj = cudaEventRecord(e->ev_join[k], st);
    if (rj == cudaSuccess) rj = cudaStreamWaitEvent(s, e->ev_join[k], 0);
    ++k;
    return rj;
  };
  cudaStream_t st;
  if (e->n_reg > 0) {
    if ((r = stream_for(st)) != cudaSuccess) return r;
    r = e->precision == DENSE_FP64 ? launch_step_fp64(a, reg, e->n_reg, e->smem, st)
                                   : launch_step_fp32(a, reg, e->n_reg, e->smem, st);
    if (r != cudaSuccess) return r;
    if ((r = join(st)) != cudaSuccess) return r;
  }
  for (const auto& g : e->mem_groups) {
    if ((r = stream_for(st)) != cudaSuccess) return r;
    if (g[0])
      r = e->precision == DENSE_FP64 ? launch_step_wave_fp64(a, mem + g[3], g[4], g[1], g[2], g[0] == 2, st)
                                     : launch_step_wave_fp32(a, mem + g[3], g[4], g[1], g[2], g[0] == 2, st);
    else
      r = e->precision == DENSE_FP64 ? launch_step_mem_fp64(a, mem + g[3], g[4], g[1], st)
                                     : launch_step_mem_fp32(a, mem + g[3], g[4], g[1], st);
    if (r != cudaSuccess) return r;
    if ((r = join(st)) != cudaSuccess) return r;
  }
  return cudaSuccess;
}

int dense_engine_run(dense_engine* e, int num_chunks, void* stream) {
  NvtxRange range_("dense_engine_run");
  if (!e) return fail(DENSE_ERR_INVALID, "null engine");
  CUDA_TRY(cudaSetDevice(e->device));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : e->stream;
  StepArgs a = e->args;
  a.chunk_count = num_chunks < 0 ? -1 : num_chunks;
  CUDA_TRY(launch_all(e, a, s));
  return DENSE_OK;
}

int dense_engine_run_graph(dense_engine* e, int num_chunks, void* stream) {
  NvtxRange range_("dense_engine_run_graph");
  if (!e) return fail(DENSE_ERR_INVALID, "null engine");
  CUDA_TRY(cudaSetDevice(e->device));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : e->stream;
  auto it = e->graphs.find(num_chunks);
  if (it == e->graphs.end()) {
    // first use: make sure the kernel attributes are set outside capture
    StepArgs a0 = e->args;
    a0.chunk_count = 0;
    CUDA_TRY(launch_all(e, a0, s));
    cudaStream_t cap;
    CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaGraph_t g;
    CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    StepArgs a = e->args;
    a.chunk_count = num_chunks < 0 ? -1 : num_chunks;
    cudaError_t le = launch_all(e, a, cap);
    cudaError_t ce = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    CUDA_TRY(le);
    CUDA_TRY(ce);
    cudaGraphExec_t ge;
    cudaError_t ie = cudaGraphInstantiateWithFlags(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    CUDA_TRY(ie);
    it = e->graphs.emplace(num_chunks, ge).first;
  }
  CUDA_TRY(cudaGraphLaunch(it->second, s));
  return DENSE_OK;
}

int dense_engine_sync(dense_engine* e) {
  if (!e) return fail(DENSE_ERR_INVALID, "null engine");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  CUDA_TRY(cudaDeviceSynchronize());
  return DENSE_OK;
}

static int read_progress(dense_engine* e, std::vector<SetProgress>& p) {
  p.resize(e->num_sets);
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(p.data(), e->d_prog.p, sizeof(SetProgress) * e->num_sets, cudaMemcpyDeviceToHost));
  return DENSE_OK;
}

int dense_engine_status(dense_engine* e, int32_t* out) {
  if (!e || !out) return fail(DENSE_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(e->device));
  std::vector<SetProgress> p;
  int rc = read_progress(e, p);
  if (rc) return rc;
  for (int s = 0; s < e->num_sets; ++s) out[s] = p[s].status;
  return DENSE_OK;
}

int dense_engine_progress(dense_engine* e, int32_t* chunks, double* age) {
  if (!e) return fail(DENSE_ERR_INVALID, "null engine");
  CUDA_TRY(cudaSetDevice(e->device));
  std::vector<SetProgress> p;
  int rc = read_progress(e, p);
  if (rc) return rc;
  for (int s = 0; s < e->num_sets; ++s) {
    if (chunks) chunks[s] = p[s].chunk;
    if (age) age[s] = p[s].age;
  }
  return DENSE_OK;
}

int dense_engine_read_state(dense_engine* e, int set, double* out) {
  if (!e || !out || set < 0 || set >= e->num_sets) return fail(DENSE_ERR_INVALID, "bad argument");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaDeviceSynchronize());
  const SetDesc& d = e->sets[set];
  const size_t cnt = static_cast<size_t>(NUM_SPECIES) * d.n_cells;
  if (e->precision == DENSE_FP64) {
    CUDA_TRY(cudaMemcpy(out, static_cast<double*>(e->d_state.p) + d.cell_base * 2 * NUM_SPECIES,
                        sizeof(double) * cnt, cudaMemcpyDeviceToHost));
  } else {
    // FP32: the Kahan-compensated value, state minus its compensation term
    // (the term follows the state in the set's block), in double
    std::vector<float> tmp(2 * cnt);
    CUDA_TRY(cudaMemcpy(tmp.data(), static_cast<float*>(e->d_state.p) + d.cell_base * 2 * NUM_SPECIES,
                        sizeof(float) * 2 * cnt, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < cnt; ++i) out[i] = static_cast<double>(tmp[i]) - static_cast<double>(tmp[cnt + i]);
  }
  return DENSE_OK;
}

static int read_analysis_block(dense_engine* e, int analysis, int set, int kind, std::vector<double>& blk,
                               const AnalysisDesc** A) {
  if (!e || set < 0 || set >= e->num_sets || analysis < 0 || analysis >= static_cast<int>(e->analyses.size()))
    return fail(DENSE_ERR_INVALID, "bad analysis or set index");
  *A = &e->analyses[analysis];
  if ((*A)->kind != kind) return fail(DENSE_ERR_INVALID, "analysis kind mismatch");
  const SetDesc& d = e->sets[set];
  int64_t len;
  const int64_t m = (*A)->cmax - (*A)->cmin, nsp = (*A)->nsp;
  if (kind == kBasic) len = 3 * nsp + 2 + 3 * m * nsp;
  else len = 2 + m * nsp * kOscFields;
  blk.resize(len);
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(blk.data(), static_cast<double*>(e->d_anl.p) + d.anl_base + (*A)->off, sizeof(double) * len,
                      cudaMemcpyDeviceToHost));
  return DENSE_OK;
}

int dense_engine_read_basic(dense_engine* e, int analysis, int set, double* mins, double* sums, double* maxs,
                            double* cell_mins, double* cell_sums, double* cell_maxs, int* samples, double* time) {
  std::vector<double> b;
  const AnalysisDesc* A;
  int rc = read_analysis_block(e, analysis, set, kBasic, b, &A);
  if (rc) return rc;
  const int n = A->nsp;
  const size_t mn = static_cast<size_t>(A->cmax - A->cmin) * n;
  for (int i = 0; i < n; ++i) {
    if (mins) mins[i] = b[i];
    if (maxs) maxs[i] = b[n + i];
    if (sums) sums[i] = b[2 * n + i];
  }
  if (samples) *samples = static_cast<int>(b[3 * n]);
  if (time) *time = b[3 * n + 1];
  const double* cb = b.data() + 3 * n + 2;  // [n][m] on the device, [m][n] for the caller
  const int m = A->cmax - A->cmin;
  for (int c = 0; c < m; ++c)
    for (int i = 0; i < n; ++i) {
      const size_t dev = static_cast<size_t>(i) * m + c, out = static_cast<size_t>(c) * n + i;
      if (cell_mins) cell_mins[out] = cb[dev];
      if (cell_maxs) cell_maxs[out] = cb[mn + dev];
      if (cell_sums) cell_sums[out] = cb[2 * mn + dev];
    }
  return DENSE_OK;
}

int dense_engine_read_oscillation(dense_engine* e, int analysis, int set, double* amps, double* periods,
                                  double* avg_peaks, int* num_crit, int* samples, double* time) {
  std::vector<double> b;
  const AnalysisDesc* A;
  int rc = read_analysis_block(e, analysis, set, kOscillation, b, &A);
  if (rc) return rc;
  const size_t k = static_cast<size_t>(A->cmax - A->cmin) * A->nsp;
  const double* f = b.data() + 2;  // [field][species][cell]
  for (size_t i = 0; i < k; ++i) {
    if (amps) amps[i] = f[kOscAmp * k + i];
    if (periods) periods[i] = f[kOscPer * k + i];
    if (avg_peaks) avg_peaks[i] = f[kOscAvgPeak * k + i];
    if (num_crit) num_crit[i] = static_cast<int>(f[kOscNcrit * k + i]);
  }
  if (samples) *samples = static_cast<int>(b[0]);
  if (time) *time = b[1];
  return DENSE_OK;
}

int dense_engine_read_trajectory(dense_engine* e, int analysis, int set, double* times, double* values,
                                 int capacity, int* samples) {
  if (!e || set < 0 || set >= e->num_sets || analysis < 0 || analysis >= static_cast<int>(e->analyses.size()))
    return fail(DENSE_ERR_INVALID, "bad analysis or set index");
  const AnalysisDesc& A = e->analyses[analysis];
  if (A.kind != kTrajectory) return fail(DENSE_ERR_INVALID, "analysis kind mismatch");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaDeviceSynchronize());
  const double* st = static_cast<const double*>(e->d_anl.p) + e->sets[set].anl_base + A.off;
  double cnt = 0;
  CUDA_TRY(cudaMemcpy(&cnt, st, sizeof(double), cudaMemcpyDeviceToHost));
  const int k = std::min(static_cast<int>(cnt), A.range_steps);
  if (samples) *samples = k;
  const int n = std::min(k, capacity);
  const size_t per = static_cast<size_t>(A.nsp) * (A.cmax - A.cmin);
  if (n > 0 && times) CUDA_TRY(cudaMemcpy(times, st + 2, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (n > 0 && values)
    CUDA_TRY(cudaMemcpy(values, st + 2 + A.range_steps, sizeof(double) * per * n, cudaMemcpyDeviceToHost));
  return DENSE_OK;
}

// Every set's Oscillation results at once, [sets][species][cells]: one
// strided copy per field.
int dense_engine_read_oscillation_all(dense_engine* e, int analysis, double* amps, double* periods) {
  NvtxRange range_("dense_engine_read_oscillation_all");
  if (!e || analysis < 0 || analysis >= static_cast<int>(e->analyses.size()))
    return fail(DENSE_ERR_INVALID, "bad analysis index");
  const AnalysisDesc& A = e->analyses[analysis];
  if (A.kind != kOscillation) return fail(DENSE_ERR_INVALID, "analysis kind mismatch");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaDeviceSynchronize());
  const size_t k = static_cast<size_t>(A.cmax - A.cmin) * A.nsp;
  const double* base = static_cast<const double*>(e->d_anl.p) + A.off + 2;
  const int fields[2] = {kOscAmp, kOscPer};
  double* outs[2] = {amps, periods};
  for (int f = 0; f < 2; ++f) {
    if (!outs[f] || k == 0) continue;
    CUDA_TRY(cudaMemcpy2D(outs[f], k * sizeof(double), base + fields[f] * k, e->anl_block * sizeof(double),
                          k * sizeof(double), e->num_sets, cudaMemcpyDeviceToHost));
  }
  return DENSE_OK;
}

// Every set's recorded Trajectory values, [sets][capacity][species][cells]
// (capacity from dense_engine_trajectory_capacity), into dst -- device
// memory when on_device, else host -- and each set's sample count.
int dense_engine_copy_trajectory(dense_engine* e, int analysis, void* dst, int on_device, int* samples,
                                 void* stream) {
  NvtxRange range_("dense_engine_copy_trajectory");
  if (!e || analysis < 0 || analysis >= static_cast<int>(e->analyses.size()))
    return fail(DENSE_ERR_INVALID, "bad analysis index");
  const AnalysisDesc& A = e->analyses[analysis];
  if (A.kind != kTrajectory) return fail(DENSE_ERR_INVALID, "analysis kind mismatch");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaDeviceSynchronize());
  const double* st = static_cast<const double*>(e->d_anl.p) + A.off;
  const size_t width = sizeof(double) * static_cast<size_t>(A.range_steps) * A.nsp * (A.cmax - A.cmin);
  const size_t pitch = sizeof(double) * e->anl_block;
  if (dst && width > 0)
    CUDA_TRY(cudaMemcpy2DAsync(dst, width, st + 2 + A.range_steps, pitch, width, e->num_sets,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               static_cast<cudaStream_t>(stream)));
  if (samples) {
    std::vector<double> cnt(e->num_sets);
    CUDA_TRY(cudaMemcpy2D(cnt.data(), sizeof(double), st, pitch, sizeof(double), e->num_sets,
                          cudaMemcpyDeviceToHost));
    for (int i = 0; i < e->num_sets; ++i) samples[i] = std::min(static_cast<int>(cnt[i]), A.range_steps);
  }
  CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  return DENSE_OK;
}

int dense_engine_trajectory_capacity(dense_engine* e, int analysis, int* capacity) {
  if (!e || !capacity || analysis < 0 || analysis >= static_cast<int>(e->analyses.size()))
    return fail(DENSE_ERR_INVALID, "bad analysis index");
  const AnalysisDesc& A = e->analyses[analysis];
  if (A.kind != kTrajectory) return fail(DENSE_ERR_INVALID, "analysis kind mismatch");
  *capacity = A.range_steps;
  return DENSE_OK;
}

int dense_engine_info(dense_engine* e, int64_t* total_cell_steps, int64_t* device_bytes, int* max_block_threads) {
  if (!e) return fail(DENSE_ERR_INVALID, "null engine");
  if (total_cell_steps) *total_cell_steps = e->total_cell_steps;
  if (device_bytes) *device_bytes = e->device_bytes;
  if (max_block_threads) *max_block_threads = e->args.block_threads;
  return DENSE_OK;
}

int dense_engine_ring_info(dense_engine* e, int set, int* S, int* D) {
  if (!e || set < 0 || set >= e->num_sets) return fail(DENSE_ERR_INVALID, "bad argument");
  for (int sp = 0; sp < NUM_SPECIES; ++sp) {
    if (S) S[sp] = e->sets[set].S[sp];
    if (D) D[sp] = e->sets[set].D[sp];
  }
  return DENSE_OK;
}

// Per-set device bytes and kernel of a batch, from the same planning as
// dense_engine_create, without touching the GPU.
int dense_engine_plan(const dense_run_desc* run, int num_sets, const dense_set_desc* in_sets, int64_t* set_bytes,
                      int* set_kernel, int* set_levels) {
  if (!run || num_sets <= 0 || !in_sets) return fail(DENSE_ERR_INVALID, "null argument or no sets");
  if (!(run->step_size > 0.0) || !(run->analysis_interval > 0.0))
    return fail(DENSE_ERR_INVALID, "step size and analysis interval must be positive");
  if (run->precision != DENSE_FP64 && run->precision != DENSE_FP32_KAHAN)
    return fail(DENSE_ERR_INVALID, "unknown precision");
  if (run->num_analyses < 0 || run->num_analyses > kMaxAnalyses)
    return fail(DENSE_ERR_UNSUPPORTED, "at most " + std::to_string(kMaxAnalyses) + " analyses per batch");
  std::vector<AnalysisDesc> analyses;
  int64_t anl_block = 0;
  int rc = build_analyses(run, num_sets, in_sets, analyses, anl_block);
  if (rc != DENSE_OK) return rc;
  const int64_t tsz = run->precision == DENSE_FP64 ? 8 : 4;
  std::vector<double> cp;
  for (int s = 0; s < num_sets; ++s) {
    const dense_set_desc& in = in_sets[s];
    const std::string where = "set " + std::to_string(s) + ": ";
    if ((rc = check_set(in, where)) != DENSE_OK) return rc;
    SetPlan plan;
    if ((rc = plan_set(in, run->step_size, run->precision == DENSE_FP64 ? 8 : 4, plan, cp)) != DENSE_OK)
      return fail(rc, where + g_error);
    const int64_t n = in.num_cells;
    if (set_bytes)
      set_bytes[s] = tsz * (((ring_elems(plan.d) + 31) & ~int64_t(31)) + 2 * NUM_SPECIES * n +
                            static_cast<int64_t>(cp.size())) +
                     4 * (n + 1 + in.nbr_offsets[n] + static_cast<int64_t>(plan.lvl_off.size()) + n + 2) +
                     8 * (anl_block + NUM_SPECIES) + static_cast<int64_t>(sizeof(SetDesc) + sizeof(SetProgress)) +
                     (plan.wave ? 16 * n : 0);
    if (set_kernel) set_kernel[s] = plan.use_mem ? plan.mem_block : 0;
    if (set_levels) set_levels[s] = plan.d.ordered ? static_cast<int>(plan.lvl_off.size()) - 1 : 1;
  }
  return DENSE_OK;
}

// One CUDA graph over several engines (of any models' libraries): each
// engine's dense_engine_run, passed as a function pointer, is captured on a
// stream of its own forked from the capture stream, and the graph keeps
// every kernel node's stream priority.
int dense_graph_capture(int num_engines, void* const* run_fns, dense_engine* const* engines, int num_chunks,
                        int device, void** graph_exec) {
  NvtxRange range_("dense_graph_capture");
  if (num_engines <= 0 || !run_fns || !engines || !graph_exec) return fail(DENSE_ERR_INVALID, "null argument");
  *graph_exec = nullptr;
  CUDA_TRY(cudaSetDevice(device));
  typedef int (*run_fn)(dense_engine*, int, void*);
  cudaStream_t cap;
  CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
  std::vector<cudaStream_t> st(num_engines, nullptr);
  std::vector<cudaEvent_t> ev(num_engines + 1, nullptr);
  cudaError_t ce = cudaSuccess;
  int failed = -1;  // the engine whose run failed (its message is in its own library's dense_last_error)
  for (int i = 0; i < num_engines && ce == cudaSuccess; ++i) ce = cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking);
  for (int i = 0; i <= num_engines && ce == cudaSuccess; ++i) ce = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
  int rc = DENSE_OK;
  cudaGraph_t g = nullptr;
  if (ce == cudaSuccess) ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) {
    cudaError_t le = cudaEventRecord(ev[num_engines], cap);
    for (int i = 0; i < num_engines && le == cudaSuccess && rc == DENSE_OK; ++i) {
      le = cudaStreamWaitEvent(st[i], ev[num_engines], 0);
      if (le == cudaSuccess) rc = reinterpret_cast<run_fn>(run_fns[i])(engines[i], num_chunks, st[i]);
      if (rc != DENSE_OK) failed = i;
      if (le == cudaSuccess && rc == DENSE_OK) le = cudaEventRecord(ev[i], st[i]);
      if (le == cudaSuccess && rc == DENSE_OK) le = cudaStreamWaitEvent(cap, ev[i], 0);
    }
    ce = cudaStreamEndCapture(cap, &g);
    if (le != cudaSuccess) ce = le;
  }
  cudaGraphExec_t ge = nullptr;
  if (ce == cudaSuccess && rc == DENSE_OK) ce = cudaGraphInstantiateWithFlags(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
  if (g) cudaGraphDestroy(g);
  for (auto x : st)
    if (x) cudaStreamDestroy(x);
  for (auto x : ev)
    if (x) cudaEventDestroy(x);
  cudaStreamDestroy(cap);
  if (rc != DENSE_OK)
    return fail(rc, "capture: the run of engine " + std::to_string(failed) + " failed with code " +
                        std::to_string(rc) + " (its model library's dense_last_error has the reason)");
  if (ce != cudaSuccess) return fail(DENSE_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(ce));
  *graph_exec = ge;
  return DENSE_OK;
}

int dense_graph_launch(void* graph_exec, void* stream) {
  if (!graph_exec) return fail(DENSE_ERR_INVALID, "null graph");
  CUDA_TRY(cudaGraphLaunch(static_cast<cudaGraphExec_t>(graph_exec), static_cast<cudaStream_t>(stream)));
  return DENSE_OK;
}

int dense_graph_destroy(void* graph_exec) {
  if (graph_exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(graph_exec));
  return DENSE_OK;
}

// Analyses of imported samples (simulation -i): the set's analyses run over
// the given sampled states instead of simulated ones.
int dense_engine_analyze_samples(dense_engine* e, int set, const double* samples, int num_samples,
                                 double time_start) {
  NvtxRange range_("dense_engine_analyze_samples");
  if (!e || set < 0 || set >= e->num_sets || num_samples < 0 || (num_samples > 0 && !samples))
    return fail(DENSE_ERR_INVALID, "bad argument");
  const StepArgs& a = e->args;
  const int n = e->sets[set].n_cells;
  // the samples in the rows of the kernels' sampled-state buffer: the
  // species some analysis observes
  const size_t per = static_cast<size_t>(std::max(1, a.n_vals)) * n;
  std::vector<double> rows(per * std::max(1, num_samples), 0.0);
  for (int k = 0; k < num_samples; ++k)
    for (int sp = 0; sp < NUM_SPECIES; ++sp)
      if (a.val_slot[sp] >= 0)
        std::memcpy(rows.data() + k * per + static_cast<size_t>(a.val_slot[sp]) * n,
                    samples + (static_cast<size_t>(k) * NUM_SPECIES + sp) * n, sizeof(double) * n);
  CUDA_TRY(cudaSetDevice(e->device));
  DeviceBuffer d_rows;
  int rc = d_rows.alloc(sizeof(double) * rows.size());
  if (rc != DENSE_OK) return rc;
  CUDA_TRY(cudaMemcpyAsync(d_rows.p, rows.data(), sizeof(double) * rows.size(), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(e->precision == DENSE_FP64
               ? launch_import_fp64(a, set, static_cast<const double*>(d_rows.p), num_samples, time_start, e->stream)
               : launch_import_fp32(a, set, static_cast<const double*>(d_rows.p), num_samples, time_start, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return DENSE_OK;
}

// ---- checkpoint / resume
//
// Snapshot layout: a CheckpointHeader, then the device blocks in the order
// progress, state, history rings, analysis state.  The header carries the
// block sizes and a hash of the batch's set descriptors and analyses, so a
// snapshot is only accepted by an engine with the same layout.

namespace {

struct CheckpointHeader {
  char magic[8];  // "DENSECK1"
  int32_t precision, num_sets;
  int64_t layout_hash;
  int64_t bytes[4];
};

uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

CheckpointHeader checkpoint_header(const dense_engine* e) {
  CheckpointHeader h{};
  std::memcpy(h.magic, "DENSECK1", 8);
  h.precision = e->precision;
  h.num_sets = e->num_sets;
  // the fields that place a set's run state in the four blocks (field by
  // field: the structs' padding bytes are not initialised)
  uint64_t x = 1469598103934665603ull;
  auto mix = [&x](const void* p, size_t n) { x = fnv1a(x, p, n); };
  for (const SetDesc& d : e->sets) {
    mix(&d.n_cells, sizeof d.n_cells);
    mix(&d.n_chunks, sizeof d.n_chunks);
    mix(&d.steps_per_chunk, sizeof d.steps_per_chunk);
    mix(&d.cell_base, sizeof d.cell_base);
    mix(&d.ring_base, sizeof d.ring_base);
    mix(&d.anl_base, sizeof d.anl_base);
    mix(d.S, sizeof d.S);
    mix(d.D, sizeof d.D);
    mix(d.ring_off, sizeof d.ring_off);
  }
  for (const AnalysisDesc& A : e->analyses) {
    mix(&A.kind, sizeof A.kind);
    mix(&A.nsp, sizeof A.nsp);
    mix(A.sp, sizeof(int) * A.nsp);
    mix(&A.cmin, sizeof A.cmin);
    mix(&A.cmax, sizeof A.cmax);
    mix(&A.range_steps, sizeof A.range_steps);
    mix(&A.off, sizeof A.off);
  }
  h.layout_hash = static_cast<int64_t>(x);
  const DeviceBuffer* blocks[4] = {&e->d_prog, &e->d_state, &e->d_ring, &e->d_anl};
  for (int i = 0; i < 4; ++i) h.bytes[i] = static_cast<int64_t>(blocks[i]->bytes);
  return h;
}

}  // namespace

int dense_engine_checkpoint_size(dense_engine* e, int64_t* bytes) {
  if (!e || !bytes) return fail(DENSE_ERR_INVALID, "null argument");
  const CheckpointHeader h = checkpoint_header(e);
  *bytes = static_cast<int64_t>(sizeof h) + h.bytes[0] + h.bytes[1] + h.bytes[2] + h.bytes[3];
  return DENSE_OK;
}

int dense_engine_checkpoint(dense_engine* e, void* buf, int64_t bytes) {
  NvtxRange range_("dense_engine_checkpoint");
  int64_t need = 0;
  if (!e || !buf) return fail(DENSE_ERR_INVALID, "null argument");
  dense_engine_checkpoint_size(e, &need);
  if (bytes < need) return fail(DENSE_ERR_INVALID, "checkpoint buffer smaller than dense_engine_checkpoint_size");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaDeviceSynchronize());
  const CheckpointHeader h = checkpoint_header(e);
  unsigned char* out = static_cast<unsigned char*>(buf);
  std::memcpy(out, &h, sizeof h);
  size_t off = sizeof h;
  const DeviceBuffer* blocks[4] = {&e->d_prog, &e->d_state, &e->d_ring, &e->d_anl};
  for (int i = 0; i < 4; ++i) {
    if (h.bytes[i] > 0) CUDA_TRY(cudaMemcpy(out + off, blocks[i]->p, h.bytes[i], cudaMemcpyDeviceToHost));
    off += h.bytes[i];
  }
  return DENSE_OK;
}

int dense_engine_restore(dense_engine* e, const void* buf, int64_t bytes) {
  NvtxRange range_("dense_engine_restore");
  if (!e || !buf) return fail(DENSE_ERR_INVALID, "null argument");
  CheckpointHeader got;
  if (bytes < static_cast<int64_t>(sizeof got)) return fail(DENSE_ERR_INVALID, "checkpoint shorter than its header");
  std::memcpy(&got, buf, sizeof got);
  const CheckpointHeader want = checkpoint_header(e);
  if (std::memcmp(got.magic, want.magic, 8) != 0) return fail(DENSE_ERR_INVALID, "not a dense_b200 checkpoint");
  if (got.precision != want.precision || got.num_sets != want.num_sets || got.layout_hash != want.layout_hash ||
      std::memcmp(got.bytes, want.bytes, sizeof got.bytes) != 0)
    return fail(DENSE_ERR_INVALID, "checkpoint of a batch with another layout (sets, analyses or precision)");
  int64_t need = 0;
  dense_engine_checkpoint_size(e, &need);
  if (bytes < need) return fail(DENSE_ERR_INVALID, "checkpoint truncated");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaDeviceSynchronize());
  const unsigned char* in = static_cast<const unsigned char*>(buf) + sizeof got;
  DeviceBuffer* blocks[4] = {&e->d_prog, &e->d_state, &e->d_ring, &e->d_anl};
  for (int i = 0; i < 4; ++i) {
    if (want.bytes[i] > 0) CUDA_TRY(cudaMemcpy(blocks[i]->p, in, want.bytes[i], cudaMemcpyHostToDevice));
    in += want.bytes[i];
  }
  return DENSE_OK;
}

int dense_engine_destroy(dense_engine* e) {
  if (!e) return DENSE_OK;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  delete e;
  return DENSE_OK;
}

}  // extern "C"
