// The batched deterministic step kernel for one DENSE model, templated on
// the arithmetic type T (double: the exact FP64 engine; float: the FP32
// engine with Kahan-compensated state updates).
//
// Mapping: one CTA per parameter set, one thread per tissue cell.  A launch
// runs the chunked time loop of DENSE's run_simulation
// (run_simulation.hpp:127-157) for every set from its current chunk up to
// StepArgs::chunk_count more chunks: at each chunk boundary the fused analyses sample the
// state, then (int)(interval/dt) Euler steps follow.  One __syncthreads per
// step separates the writes of step n from the neighbour reads of step n+1.
//
// State: each thread keeps its cell's lag-0 concentrations in registers.
// Only species whose history is read (found by tracing the model's
// active_rate on the host) get a ring in global memory, D_sp rows deep,
// where D_sp is one more than the deepest lag read (two more for
// neighbour-read species, so the row being written is never one a
// neighbour still reads).  Lags follow DENSE exactly (baby_cl row_at with
// the offsets of determ.hpp:73-89): an own read with integer delay k reads
// lag (k-1) mod S_sp, a neighbour average reads lag k mod S_sp, S_sp being
// DENSE's ring size.
//
// The includer defines DENSE_B200_REAL and includes dense_model_api.hpp,
// the model's reaction_deltas.hpp and model_impl.hpp first.
#pragma once

#include <cuda_runtime.h>

#include "engine_types.hpp"

namespace dense_b200 {

template <typename T>
struct DeviceContext {
  const T* cur;            // this cell's lag-0 state [NS]
  const T* prm;            // this cell's parameters [NP]
  T* const* ring;          // per species ring base for this set (nullptr: unstaged)
  const int* head;         // per species slot holding lag 0
  const int* S;            // DENSE ring sizes (shared memory)
  const int* D;            // staged depths (shared memory)
  const int* nbr;          // neighbour ids of this cell (global)
  int nnbr;
  int n_cells;
  int cell;
  int* err;

  // Context::getCon(sp) -> get_concentration(cell, sp, 1) -> row_at(sp, 0).
  __device__ __forceinline__ T getCon(specie_id sp) const { return cur[sp]; }

  // Context::getCon(sp, delay) -> row_at(sp, 1 - delay)[cell]
  // (sim/base.hpp:419-422, determ.hpp:77-79).
  __device__ __forceinline__ T getCon(specie_id sp, int k) const {
    const int s = S[sp];
    int lag = k - 1;
    if (lag < 0) lag += s;
    else if (lag >= s) lag -= s;
    if (k < 0 || k > s + 1) {
      *err |= kSetBadDelay;
      lag = ((k - 1) % s + s) % s;
    }
    if (lag == 0) return cur[sp];
    const int d = D[sp];
    if (lag >= d) {
      *err |= kSetUnstagedLag;
      return T(0);
    }
    int slot = head[sp] - lag;
    if (slot < 0) slot += d;
    return ring[sp][static_cast<size_t>(slot) * n_cells + cell];
  }

  // Context::calculateNeighborAvg -> calculate_neighbor_average
  // (determ.hpp:81-89): ascending neighbour order, sum / count, NaN -> 0.
  __device__ __forceinline__ T calculateNeighborAvg(specie_id sp, int k = 0) const {
    const int s = S[sp];
    int lag = k;
    if (lag >= s) lag -= s;
    if (k < 0 || k > s) {
      *err |= kSetBadDelay;
      lag = (k % s + s) % s;
    }
    const int d = D[sp];
    if (lag + 1 >= d) {
      *err |= (lag == s - 1) ? kSetOrderedReads : kSetUnstagedLag;
      return T(0);
    }
    int slot = head[sp] - lag;
    if (slot < 0) slot += d;
    const T* row = ring[sp] + static_cast<size_t>(slot) * n_cells;
    T sum = T(0);
    for (int e = 0; e < nnbr; ++e) sum += row[nbr[e]];
    T avg = sum / static_cast<T>(nnbr);
    return isnan(avg) ? T(0) : avg;
  }

  // Context::getRate / getDelay / getCritVal (sim/base.hpp:393-412).  NaN
  // rates and delays are rejected when the batch is created.
  __device__ __forceinline__ T getRate(reaction_id r) const { return prm[r]; }
  __device__ __forceinline__ T getDelay(delay_reaction_id d) const { return prm[kNR + d]; }
  __device__ __forceinline__ T getCritVal(critspecie_id c) const { return prm[kNR + kND + c]; }
};

// ------------------------------------------------------------ analyses
// BasicAnalysis::update (basic.ipp:22-36), per-cell part: thread c updates
// its own row.  std::min(x, m) = (m < x) ? m : x, std::max(x, M) =
// (x < M) ? M : x, NaN behaviour kept.
__device__ __forceinline__ void basic_cell_update(double* st, const AnalysisDesc& A,
                                                  const double* s_vals, int blk, int c) {
  const int n = A.nsp;
  const int m = A.cmax - A.cmin;
  if (c < A.cmin || c >= A.cmax) return;
  double* cmins = st + 3 * n + 2;
  double* cmaxs = cmins + static_cast<size_t>(m) * n;
  double* csums = cmaxs + static_cast<size_t>(m) * n;
  const int cc = c - A.cmin;
  for (int i = 0; i < n; ++i) {
    const double x = s_vals[A.sp[i] * blk + c];
    const size_t k = static_cast<size_t>(cc) * n + i;
    const double mn = cmins[k], mx = cmaxs[k];
    cmins[k] = (mn < x) ? mn : x;
    cmaxs[k] = (x < mx) ? mx : x;
    csums[k] = csums[k] + x;
  }
}

// The whole-range part: lane i of warp 0 folds species i over the cells in
// cell order, as DENSE's loop does (cells outer, species inner; each
// species' accumulator only sees its own values, so per-species folds in
// cell order give the same results bit for bit).
__device__ __forceinline__ void basic_range_fold(double* st, const AnalysisDesc& A,
                                                 const double* s_vals, int blk, int lane) {
  const int n = A.nsp;
  for (int i = lane; i < n; i += 32) {
    double mn = st[i], mx = st[n + i], sm = st[2 * n + i];
    const double* v = s_vals + A.sp[i] * blk;
    for (int c = A.cmin; c < A.cmax; ++c) {
      const double x = v[c];
      mn = (mn < x) ? mn : x;
      mx = (x < mx) ? mx : x;
      sm = sm + x;
    }
    st[i] = mn;
    st[n + i] = mx;
    st[2 * n + i] = sm;
  }
}

// Queue (core/queue.hpp:29-88) over a window slice of `w` rows.
struct DevQueue {
  long start, end, current, size;
  __device__ __forceinline__ long get_size() const { return (size + end - start) % size + 1; }
};

// OscillationAnalysis::addCritPoint (oscillation.ipp:129-144), keeping the
// sums calcAmpsAndPers (oscillation.ipp:167-185) needs in index order:
// every point but the last is final, so it is folded in when the next one
// is appended.
__device__ __forceinline__ void osc_fold_last(OscCell& o) {
  if (o.ncrit < 1) return;
  if (o.last_peak != 0.0) {
    o.peak_sum = o.peak_sum + o.last_conc;
    o.num_peaks += 1.0;
  } else {
    o.trough_sum = o.trough_sum + o.last_conc;
    o.num_troughs += 1.0;
  }
  if (o.ncrit - 1 >= 2) {
    o.cycles += 1.0;
    o.cycle_sum = o.cycle_sum + (o.last_time - o.t_m2);
  }
}

__device__ __forceinline__ void osc_add_crit(OscCell& o, double t, double conc, bool peak) {
  if (o.ncrit > 0) {
    const bool prev_peak = o.last_peak != 0.0;
    if (prev_peak == peak) {
      if (peak ? (conc >= o.last_conc) : (conc <= o.last_conc)) {
        o.last_time = t;
        o.last_conc = conc;
      }
      return;
    }
    osc_fold_last(o);
    o.t_m2 = o.t_m1;
    o.t_m1 = o.last_time;
  }
  o.last_time = t;
  o.last_conc = conc;
  o.last_peak = peak ? 1.0 : 0.0;
  o.ncrit += 1.0;
}

// OscillationAnalysis::checkCritPoint (oscillation.ipp:110-119).  The
// window max/min are those of the live values (DENSE keeps them in a
// multiset).  A middle index of -1 (DENSE reads contents[-1]) or an empty
// window gives no critical point.
__device__ __forceinline__ void osc_check(OscCell& o, const double* win, int m, int w,
                                          double samples, const AnalysisDesc& A) {
  const long cur = static_cast<long>(o.current);
  const long live = static_cast<long>(o.live);
  if (cur < 0 || live <= 0) return;
  const double mid = win[static_cast<size_t>(cur) * m];
  long idx = static_cast<long>(o.start);
  double hi = win[static_cast<size_t>(idx) * m], lo = hi;
  for (long q = 1; q < live; ++q) {
    idx = (idx == w - 1) ? 0 : idx + 1;
    const double x = win[static_cast<size_t>(idx) * m];
    hi = (hi < x) ? x : hi;
    lo = (x < lo) ? x : lo;
  }
  double t = (samples - static_cast<double>(A.range_steps / 2)) * A.interval + A.t0;
  t = (0.0 < t) ? t : 0.0;
  if (mid == hi && mid != lo) osc_add_crit(o, t, mid, true);
  else if (mid == lo) osc_add_crit(o, t, mid, false);
}

__device__ __forceinline__ double osc_dequeue(OscCell& o, const double* win, int m, int w) {
  const long size = w;
  long start = static_cast<long>(o.start);
  const double popped = win[static_cast<size_t>(start) * m];
  start = (start == size - 1) ? 0 : start + 1;
  o.start = static_cast<double>(start);
  DevQueue q{start, static_cast<long>(o.end), static_cast<long>(o.current), size};
  if (2 * q.get_size() <= size) {
    long cur = q.current + 1;
    if (cur == size) cur = 0;
    o.current = static_cast<double>(cur);
  }
  o.live -= 1.0;
  return popped;
}

// OscillationAnalysis::update / get_peaks_and_troughs (oscillation.ipp:
// 86-103, 154-160) for thread c's cell, species in observation order,
// stopping at the first species whose window is still short.
__device__ __forceinline__ void osc_cell_update(double* st, const AnalysisDesc& A,
                                                const double* s_vals, int blk, int c,
                                                double samples) {
  if (c < A.cmin || c >= A.cmax) return;
  const int n = A.nsp, m = A.cmax - A.cmin, w = A.range_steps + 1;
  const int cc = c - A.cmin;
  OscCell* cells = reinterpret_cast<OscCell*>(st + 2);
  double* windows = st + 2 + static_cast<size_t>(n) * m * kOscCellDoubles;
  for (int i = 0; i < n; ++i) {
    OscCell o = cells[static_cast<size_t>(i) * m + cc];
    double* win = windows + static_cast<size_t>(i) * w * m + cc;
    const double added = s_vals[A.sp[i] * blk + c];
    // enqueue
    long end = static_cast<long>(o.end);
    end = (end == w - 1) ? 0 : end + 1;
    win[static_cast<size_t>(end) * m] = added;
    o.end = static_cast<double>(end);
    o.live += 1.0;
    DevQueue q{static_cast<long>(o.start), end, static_cast<long>(o.current), w};
    if (2 * q.get_size() >= w) {
      long cur = q.current + 1;
      if (cur == w) cur = 0;
      o.current = static_cast<double>(cur);
    }
    q.current = static_cast<long>(o.current);
    if (q.get_size() == A.range_steps + 1) {
      osc_dequeue(o, win, m, w);
      q.start = static_cast<long>(o.start);
    }
    const bool stop = q.get_size() < A.range_steps / 2;
    if (!stop) osc_check(o, win, m, w, samples, A);
    cells[static_cast<size_t>(i) * m + cc] = o;
    if (stop) break;
  }
}

// OscillationAnalysis::finalize (oscillation.ipp:6-26) and
// calcAmpsAndPers for thread c's cell; also the "avg peak" of show().
// DENSE's sample counter restarts from its pre-finalize value for every
// (species, cell) window and is left at the value of the last one; the
// thread of the last cell writes that value.
__device__ __forceinline__ void osc_cell_finalize(double* st, const AnalysisDesc& A, int c, double samples0) {
  if (c < A.cmin || c >= A.cmax) return;
  const int n = A.nsp, m = A.cmax - A.cmin, w = A.range_steps + 1;
  const int cc = c - A.cmin;
  OscCell* cells = reinterpret_cast<OscCell*>(st + 2);
  double* windows = st + 2 + static_cast<size_t>(n) * m * kOscCellDoubles;
  double samples = samples0;
  for (int i = 0; i < n; ++i) {
    OscCell o = cells[static_cast<size_t>(i) * m + cc];
    double* win = windows + static_cast<size_t>(i) * w * m + cc;
    samples = samples0;
    for (;;) {
      DevQueue q{static_cast<long>(o.start), static_cast<long>(o.end), static_cast<long>(o.current), w};
      if (!(q.get_size() >= (A.range_steps / 2) && o.live > 0.0)) break;
      osc_dequeue(o, win, m, w);
      osc_check(o, win, m, w, samples, A);
      samples += 1.0;
    }
    osc_fold_last(o);
    o.amp = ((o.peak_sum / o.num_peaks) - (o.trough_sum / o.num_troughs)) / 2;
    o.per = o.cycle_sum / o.cycles;
    o.avg_peak = (o.num_peaks != 0.0) ? o.peak_sum / o.num_peaks : o.peak_sum;
    cells[static_cast<size_t>(i) * m + cc] = o;
  }
  if (cc == m - 1) st[0] = samples;
}

// ---------------------------------------------------------------- kernel
template <typename T, bool kKahan>
__global__ void __launch_bounds__(256, 1) dense_step_kernel(const StepArgs a) {
  extern __shared__ double s_vals[];  // [NS][blockDim] sampled state
  __shared__ int s_S[kNS], s_D[kNS];
  __shared__ int s_flags;
  __shared__ double s_samples[kMaxAnalyses];

  const int set = blockIdx.x;
  if (set >= a.num_sets) return;
  const SetDesc& sd = a.sets[set];
  const int n = sd.n_cells;
  const int blk = blockDim.x;
  const int c = threadIdx.x;
  const bool active = c < n;

  SetProgress pg = a.prog[set];
  if ((pg.status & (kSetDropped | kSetNotRunnable)) || pg.finalized) return;

  if (c < kNS) {
    s_S[c] = sd.S[c];
    s_D[c] = sd.D[c];
  }
  if (c == 0) s_flags = 0;
  double* anl = a.anl + sd.anl_base;
  if (c < a.n_analyses) s_samples[c] = anl[a.analyses[c].off];
  __syncthreads();

  T* ring_base = static_cast<T*>(a.ring) + sd.ring_base;
  T* ringp[kNS];
  int head[kNS];
#pragma unroll
  for (int sp = 0; sp < kNS; ++sp) {
    const int d = s_D[sp];
    ringp[sp] = d > 0 ? ring_base + sd.ring_off[sp] : nullptr;
    head[sp] = d > 0 ? static_cast<int>(pg.step % d) : 0;
  }

  T prm[kNP];
  T cur[kNS];
  T comp[kNS];
  T* state = static_cast<T*>(a.state) + sd.cell_base * (2 * kNS);
  const int cell = active ? c : 0;
  {
    const double* P = a.params + sd.cell_base * kNP;
#pragma unroll
    for (int i = 0; i < kNP; ++i) prm[i] = static_cast<T>(P[static_cast<size_t>(i) * n + cell]);
#pragma unroll
    for (int sp = 0; sp < kNS; ++sp) {
      cur[sp] = state[static_cast<size_t>(sp) * n + cell];
      comp[sp] = kKahan ? state[static_cast<size_t>(kNS + sp) * n + cell] : T(0);
    }
  }
  const int* nbr_off = a.nbr_off + sd.nbr_base;
  const int nb0 = nbr_off[cell];
  const int nnbr = nbr_off[cell + 1] - nb0;
  int err = 0;
  DeviceContext<T> ctx{cur, prm, ringp, head, s_S, s_D, a.nbr_idx + nb0, nnbr, n, cell, &err};

  const T dt = static_cast<T>(a.dt);
  int chunk = pg.chunk;
  const int chunk_end = (a.chunk_count < 0 || sd.n_chunks - chunk < a.chunk_count)
                            ? sd.n_chunks
                            : chunk + a.chunk_count;
  double age = pg.age;
  int64_t step = pg.step;
  bool dropped = false;

  for (; chunk < chunk_end; ++chunk) {
    // ---- analyses sample the state at `age` (measurement/base.ipp:4-9)
    if (a.n_analyses > 0) {
#pragma unroll
      for (int sp = 0; sp < kNS; ++sp) s_vals[sp * blk + c] = static_cast<double>(cur[sp]);
      __syncthreads();
      bool bad = false;
      for (int ai = 0; ai < a.n_analyses; ++ai) {
        const AnalysisDesc& A = a.analyses[ai];
        double* st = anl + A.off;
        const bool in_range = !(age < A.t0 || age >= A.t1);
        if (A.kind == kBasic) {
          if (c == 0) st[3 * A.nsp + 1] = age;
          if (!in_range) continue;
          basic_cell_update(st, A, s_vals, blk, c);
          if (c < 32) basic_range_fold(st, A, s_vals, blk, c);
          if (c == 0) st[3 * A.nsp] += 1.0;
        } else if (A.kind == kOscillation) {
          if (c == 0) st[1] = age;
          if (!in_range) continue;
          osc_cell_update(st, A, s_vals, blk, c, s_samples[ai]);
          if (c == 0) st[0] = s_samples[ai] + 1.0;
        } else if (A.kind == kConcCheck) {
          if (c == 0) st[0] = age;
          if (!in_range) continue;
          if (c >= A.cmin && c < A.cmax) {
            for (int i = 0; i < A.nsp; ++i) {
              const double x = s_vals[A.sp[i] * blk + c];
              if (x < A.lo || x > A.hi) bad = true;
            }
          }
        }
      }
      if (bad) atomicOr(&s_flags, 1);
      __syncthreads();
      if (c < a.n_analyses) s_samples[c] = anl[a.analyses[c].off];
      if (s_flags & 1) {
        dropped = true;
        break;
      }
    }

    // ---- (int)(interval/dt) Euler steps (determ.cpp:8-21, 77-88)
    for (int s = 0; s < sd.steps_per_chunk; ++s) {
      T nxt[kNS];
      if (active) {
        T rates[kNR];
#define REACTION(name) rates[name] = reaction<name>::active_rate(ctx);
#include "reactions_list.hpp"
#undef REACTION
        T dsp[kNS];
#pragma unroll
        for (int sp = 0; sp < kNS; ++sp) dsp[sp] = T(0);
#define REACTION(name)                                                      \
  _Pragma("unroll") for (int j = 0; j < num_deltas_##name; j++)             \
      dsp[delta_ids_##name[j]] += rates[name] * static_cast<T>(deltas_##name[j]);
#include "reactions_list.hpp"
#undef REACTION
#pragma unroll
        for (int sp = 0; sp < kNS; ++sp) {
          if (kKahan) {
            const T y = dt * dsp[sp] - comp[sp];
            const T t = cur[sp] + y;
            comp[sp] = (t - cur[sp]) - y;
            nxt[sp] = t;
          } else {
            nxt[sp] = cur[sp] + dt * dsp[sp];
          }
        }
      }
#pragma unroll
      for (int sp = 0; sp < kNS; ++sp) {
        const int d = s_D[sp];
        if (d > 0) {
          int h = head[sp] + 1;
          if (h == d) h = 0;
          head[sp] = h;
          if (active) ringp[sp][static_cast<size_t>(h) * n + c] = nxt[sp];
        }
      }
      __syncthreads();
      if (active) {
#pragma unroll
        for (int sp = 0; sp < kNS; ++sp) cur[sp] = nxt[sp];
      }
    }
    step += sd.steps_per_chunk;
    age += a.interval;
  }

  // ---- save
  if (active) {
#pragma unroll
    for (int sp = 0; sp < kNS; ++sp) {
      state[static_cast<size_t>(sp) * n + c] = cur[sp];
      if (kKahan) state[static_cast<size_t>(kNS + sp) * n + c] = comp[sp];
    }
  }
  if (err) atomicOr(&s_flags, err << 1);
  // pre-finalize sample counters, read before any thread finalizes
  if (c < a.n_analyses) s_samples[c] = anl[a.analyses[c].off];
  __syncthreads();
  const int status = pg.status | (dropped ? kSetDropped : 0) | (s_flags >> 1);
  const bool finish = !dropped && chunk >= sd.n_chunks;
  if (finish) {
    for (int ai = 0; ai < a.n_analyses; ++ai) {
      const AnalysisDesc& A = a.analyses[ai];
      if (A.kind == kOscillation) osc_cell_finalize(anl + A.off, A, c, s_samples[ai]);
    }
  }
  if (c == 0) {
    SetProgress out = pg;
    out.step = step;
    out.chunk = chunk;
    out.age = age;
    out.status = status;
    out.finalized = finish ? 1 : 0;
    a.prog[set] = out;
  }
}

}  // namespace dense_b200

namespace dense_b200 {

// Fills every set's state, history rows and analysis state with their
// initial values: all rows of every ring hold the initial concentrations
// (determ.cpp:42-51, zeros when none are given), Basic minima start at
// +inf and maxima at 0 (basic.ipp:13-15), queues start empty
// (core/queue.hpp:31-37).
template <typename T>
__global__ void dense_init_kernel(const StepArgs a, const double* init_conc, const int* init_status) {
  const int set = blockIdx.x;
  if (set >= a.num_sets) return;
  const SetDesc& sd = a.sets[set];
  const int n = sd.n_cells;
  const double* ic = init_conc + static_cast<size_t>(set) * kNS;
  T* state = static_cast<T*>(a.state) + sd.cell_base * (2 * kNS);
  for (int i = threadIdx.x; i < kNS * n; i += blockDim.x) {
    state[i] = static_cast<T>(ic[i / n]);
    state[kNS * n + i] = T(0);
  }
  T* ring = static_cast<T*>(a.ring) + sd.ring_base;
  for (int sp = 0; sp < kNS; ++sp) {
    const int64_t rows = static_cast<int64_t>(sd.D[sp]) * n;
    const T v = static_cast<T>(ic[sp]);
    for (int64_t i = threadIdx.x; i < rows; i += blockDim.x) ring[sd.ring_off[sp] + i] = v;
  }
  double* anl = a.anl + sd.anl_base;
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  for (int ai = 0; ai < a.n_analyses; ++ai) {
    const AnalysisDesc& A = a.analyses[ai];
    double* st = anl + A.off;
    const int nsp = A.nsp, m = A.cmax - A.cmin;
    if (A.kind == kBasic) {
      const int64_t total = 3 * nsp + 2 + 3 * static_cast<int64_t>(m) * nsp;
      for (int64_t i = threadIdx.x; i < total; i += blockDim.x) {
        double v = 0.0;
        if (i < nsp) v = inf;
        else if (i >= 3 * nsp + 2 && i < 3 * nsp + 2 + static_cast<int64_t>(m) * nsp) v = inf;
        st[i] = v;
      }
    } else if (A.kind == kOscillation) {
      const int64_t cellsz = static_cast<int64_t>(nsp) * m * kOscCellDoubles;
      const int64_t total = 2 + cellsz + static_cast<int64_t>(nsp) * (A.range_steps + 1) * m;
      for (int64_t i = threadIdx.x; i < total; i += blockDim.x) {
        double v = 0.0;
        if (i >= 2 && i < 2 + cellsz) {
          const int f = static_cast<int>((i - 2) % kOscCellDoubles);
          if (f == 1 || f == 2) v = -1.0;  // end = current = -1
        }
        st[i] = v;
      }
    } else {
      if (threadIdx.x == 0) st[0] = 0.0;
    }
  }
  if (threadIdx.x == 0) {
    SetProgress p{};
    p.step = 0;
    p.chunk = 0;
    p.status = init_status[set];
    p.age = 0.0;
    p.finalized = 0;
    a.prog[set] = p;
  }
}

}  // namespace dense_b200

// Launchers, named by the including translation unit's precision suffix.
#define DENSE_B200_DEFINE_LAUNCHERS(SUFFIX, T, KAHAN)                                             \
  namespace dense_b200 {                                                                        \
  cudaError_t launch_init_##SUFFIX(const StepArgs& a, const double* init_conc,                   \
                                   const int* init_status, cudaStream_t s) {                    \
    dense_init_kernel<T><<<a.num_sets, 256, 0, s>>>(a, init_conc, init_status);                  \
    return cudaGetLastError();                                                                  \
  }                                                                                             \
  cudaError_t launch_step_##SUFFIX(const StepArgs& a, size_t smem, cudaStream_t s) {            \
    static bool configured = false;                                                             \
    if (!configured) {                                                                          \
      cudaError_t e = cudaFuncSetAttribute(dense_step_kernel<T, KAHAN>,                          \
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                                           kNS * kMaxCellsPerSet * (int)sizeof(double));         \
      if (e != cudaSuccess) return e;                                                           \
      configured = true;                                                                        \
    }                                                                                           \
    dense_step_kernel<T, KAHAN><<<a.num_sets, a.block_threads, smem, s>>>(a);                    \
    return cudaGetLastError();                                                                  \
  }                                                                                             \
  }
