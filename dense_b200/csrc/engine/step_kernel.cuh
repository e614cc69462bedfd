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

#include "count_div.cuh"
#include "engine_types.hpp"

namespace dense_b200 {

// What getDelay returns: the delay reaction and this cell's delay truncated
// to int (the conversion DENSE applies when the delay is passed on as
// getCon's or calculateNeighborAvg's `int delay`, sim/base.hpp:68-71).
// Used as a number it converts to the delay value itself.
template <typename T>
struct DelayArg {
  const T* prm;
  int pstride;
  int dr;
  int k;
  __device__ __forceinline__ operator T() const { return prm[(kNR + dr) * pstride]; }
};

// Neighbour counts whose reciprocals the memory kernel keeps in a table.
constexpr int kRcTable = 33;

// kUniform: every cell of the set has the set's parameters, so the lag of
// each (delay reaction, species) read is the same for all cells and is
// looked up in per-set tables (olag / nlag, [ND][NS]): a value >= 0 is a
// lag the staging holds (own reads: 0 means the register state), -1 sends
// the read through the checked path, which also records the error.
template <typename T, bool kUniform>
struct DeviceContext {
  const T* cur;            // this cell's lag-0 state [NS] (registers)
  const T* prm;            // parameters: shared row (pstride 1) or this cell's column (pstride n)
  int pstride;
  const int* kd;           // truncated delays, kd[d * kd_stride] (shared)
  int kd_stride;
  const int* S;            // DENSE ring sizes (shared)
  const int* mask;         // staged depth - 1 per species, -1 unstaged (shared)
  const int64_t* roff;     // ring offset per species (shared)
  T* ring;                 // this set's ring block
  int step;                // Euler steps done: lag 0 sits in row step & mask
  const int* nbr;          // this cell's neighbour ids (shared, or global for large lists)
  int nnbr;
  T rc;                    // RN(1 / nnbr)
  const int* olag;         // kUniform: own-read lag table [ND][NS] (shared)
  const int* nlag;         // kUniform: neighbour-read lag table [ND][NS] (shared)
  bool ordered;            // the set runs in cell-dependency levels (memory kernel)
  int n_cells;
  int cell;
  int* err;

  __device__ __forceinline__ T own(specie_id sp, int k) const {
    const int s = S[sp];
    int lag = k - 1;
    if (lag < 0) lag += s;
    if (static_cast<unsigned>(k) > static_cast<unsigned>(s)) {  // k < 0 or k > S: rare
      if (k < 0 || k > s + 1) *err |= kSetBadDelay;
      lag = ((k - 1) % s + s) % s;
    }
    if (lag == 0) return cur[sp];
    const int m = mask[sp];
    if (lag > m) {
      *err |= kSetUnstagedLag;
      return T(0);
    }
    return ring[roff[sp] + static_cast<int64_t>((step - lag) & m) * n_cells + cell];
  }

  __device__ __forceinline__ T own_lag(specie_id sp, int lag) const {
    if (lag == 0) return cur[sp];
    return ring[roff[sp] + static_cast<int64_t>((step - lag) & mask[sp]) * n_cells + cell];
  }

  __device__ __forceinline__ T nbr_lag(specie_id sp, int lag) const {
    const T* row = ring + roff[sp] + static_cast<int64_t>((step - lag) & mask[sp]) * n_cells;
    T sum = T(0);
    for (int e = 0; e < nnbr; ++e) sum += row[nbr[e]];
    const T avg = div_by_count(sum, static_cast<T>(nnbr), rc);
    return isnan(avg) ? T(0) : avg;
  }

  __device__ __forceinline__ T nbr_avg(specie_id sp, int k) const {
    const int s = S[sp];
    int lag = k;
    if (static_cast<unsigned>(k) >= static_cast<unsigned>(s)) {  // k < 0 or k >= S: rare
      if (k < 0 || k > s) *err |= kSetBadDelay;
      lag = (k % s + s) % s;
    }
    const int m = mask[sp];
    // lag S-1 is the row DENSE's cell-ordered loop is writing in this very
    // step: lower-numbered neighbours have their new value there already,
    // the others (and the cell itself) still the old one.  Only a set run
    // in cell-dependency levels, with rings deeper than S, reads it.
    if (lag == s - 1 && s > 1) {
      if (!ordered || m < s) {
        *err |= kSetOrderedReads;
        return T(0);
      }
      const T* fresh = ring + roff[sp] + static_cast<int64_t>((step + 1) & m) * n_cells;
      const T* old = ring + roff[sp] + static_cast<int64_t>((step - lag) & m) * n_cells;
      T sum = T(0);
      for (int e = 0; e < nnbr; ++e) {
        const int v = nbr[e];
        sum += v < cell ? fresh[v] : old[v];
      }
      const T avg = div_by_count(sum, static_cast<T>(nnbr), rc);
      return isnan(avg) ? T(0) : avg;
    }
    if (lag >= m) {
      *err |= kSetUnstagedLag;
      return T(0);
    }
    return nbr_lag(sp, lag);
  }

  // Context::getCon(sp) -> get_concentration(cell, sp, 1) -> row_at(sp, 0).
  __device__ __forceinline__ T getCon(specie_id sp) const { return cur[sp]; }
  // Context::getCon(sp, delay) -> row_at(sp, 1 - delay)[cell]
  // (sim/base.hpp:419-422, determ.hpp:77-79): lag (k - 1) mod S.
  __device__ __forceinline__ T getCon(specie_id sp, int k) const { return own(sp, k); }
  __device__ __forceinline__ T getCon(specie_id sp, DelayArg<T> d) const {
    if (kUniform) {
      const int lag = olag[d.dr * kNS + sp];
      if (lag >= 0) return own_lag(sp, lag);
    }
    return own(sp, d.k);
  }
  // Context::calculateNeighborAvg -> calculate_neighbor_average
  // (determ.hpp:81-89): row_at(sp, -delay), lag k mod S, ascending
  // neighbour order, sum / count, NaN -> 0.
  __device__ __forceinline__ T calculateNeighborAvg(specie_id sp, int k = 0) const { return nbr_avg(sp, k); }
  __device__ __forceinline__ T calculateNeighborAvg(specie_id sp, DelayArg<T> d) const {
    if (kUniform) {
      const int lag = nlag[d.dr * kNS + sp];
      if (lag >= 0) return nbr_lag(sp, lag);
    }
    return nbr_avg(sp, d.k);
  }
  // Context::getRate / getDelay / getCritVal (sim/base.hpp:393-412).  NaN
  // rates and delays are rejected when the batch is created.
  __device__ __forceinline__ T getRate(reaction_id r) const { return prm[r * pstride]; }
  __device__ __forceinline__ DelayArg<T> getDelay(delay_reaction_id d) const {
    return DelayArg<T>{prm, pstride, static_cast<int>(d),
                       kd ? kd[d * kd_stride] : static_cast<int>(prm[(kNR + d) * pstride])};
  }
  __device__ __forceinline__ T getCritVal(critspecie_id c) const { return prm[(kNR + kND + c) * pstride]; }
};

// ------------------------------------------------------------ analyses
// All per-cell analysis state is structure-of-arrays over the analysed
// cells, so the threads of a warp touch consecutive doubles.

// BasicAnalysis::update (basic.ipp:22-36), per-cell part: thread c updates
// its own column.  std::min(x, m) = (m < x) ? m : x, std::max(x, M) =
// (x < M) ? M : x, NaN behaviour kept.
template <typename Vals>
__device__ __forceinline__ void basic_cell_update(double* st, const AnalysisDesc& A, const Vals& vals, int c) {
  const int n = A.nsp;
  const int m = A.cmax - A.cmin;
  if (c < A.cmin || c >= A.cmax) return;
  double* cmins = st + 3 * n + 2;  // [n][m]
  double* cmaxs = cmins + static_cast<size_t>(m) * n;
  double* csums = cmaxs + static_cast<size_t>(m) * n;
  const int cc = c - A.cmin;
  for (int i = 0; i < n; ++i) {
    const double x = vals(A.slot[i], c);
    const size_t k = static_cast<size_t>(i) * m + cc;
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
template <typename Vals>
__device__ __forceinline__ void basic_range_fold(double* st, const AnalysisDesc& A, const Vals& vals, int lane) {
  const int n = A.nsp;
  for (int i = lane; i < n; i += 32) {
    double mn = st[i], mx = st[n + i], sm = st[2 * n + i];
    for (int c = A.cmin; c < A.cmax; ++c) {
      const double x = vals(A.slot[i], c);
      mn = (mn < x) ? mn : x;
      mx = (x < mx) ? mx : x;
      sm = sm + x;
    }
    st[i] = mn;
    st[n + i] = mx;
    st[2 * n + i] = sm;
  }
}

// One (species, cell) of an OscillationAnalysis: field k lives at
// p[k * stride].  The queue indices follow core/queue.hpp:29-88; the
// critical-point fields keep what calcAmpsAndPers (oscillation.ipp:167-185)
// needs: every point but the last is final and already folded into the
// sums, in index order.
struct OscRef {
  double* p;
  size_t stride;
  __device__ __forceinline__ double& f(int k) const { return p[k * stride]; }
};

// Queue::getSize, (size + end - start) % size + 1.  With end in [-1, size)
// and start in [0, size) the dividend lies in [0, 2 * size), so one
// conditional subtraction gives the same remainder.
__device__ __forceinline__ long q_size(long start, long end, long size) {
  const long x = size + end - start;
  return (x < size ? x : x - size) + 1;
}

__device__ __forceinline__ void osc_fold_last(const OscRef& o) {
  const double ncrit = o.f(kOscNcrit);
  if (ncrit < 1) return;
  if (o.f(kOscLastPeak) != 0.0) {
    o.f(kOscPeakSum) = o.f(kOscPeakSum) + o.f(kOscLastConc);
    o.f(kOscNumPeaks) += 1.0;
  } else {
    o.f(kOscTroughSum) = o.f(kOscTroughSum) + o.f(kOscLastConc);
    o.f(kOscNumTroughs) += 1.0;
  }
  if (ncrit - 1 >= 2) {
    o.f(kOscCycles) += 1.0;
    o.f(kOscCycleSum) = o.f(kOscCycleSum) + (o.f(kOscLastTime) - o.f(kOscTm2));
  }
}

// OscillationAnalysis::addCritPoint (oscillation.ipp:129-144).
__device__ __forceinline__ void osc_add_crit(const OscRef& o, double t, double conc, bool peak) {
  if (o.f(kOscNcrit) > 0) {
    const bool prev_peak = o.f(kOscLastPeak) != 0.0;
    if (prev_peak == peak) {
      if (peak ? (conc >= o.f(kOscLastConc)) : (conc <= o.f(kOscLastConc))) {
        o.f(kOscLastTime) = t;
        o.f(kOscLastConc) = conc;
      }
      return;
    }
    osc_fold_last(o);
    o.f(kOscTm2) = o.f(kOscTm1);
    o.f(kOscTm1) = o.f(kOscLastTime);
  }
  o.f(kOscLastTime) = t;
  o.f(kOscLastConc) = conc;
  o.f(kOscLastPeak) = peak ? 1.0 : 0.0;
  o.f(kOscNcrit) += 1.0;
}

// The queue part of one (species, cell), held in registers while a sample
// is processed; loaded and stored as one batch of independent accesses.
struct OscQueue {
  long start, end, current, live;
  long same;  // the newest `same` values are equal (so the window is flat when same >= live)
  __device__ __forceinline__ void load(const OscRef& o) {
    const double s0 = o.f(kOscStart), e0 = o.f(kOscEnd), c0 = o.f(kOscCurrent), l0 = o.f(kOscLive);
    const double m0 = o.f(kOscSame);
    start = static_cast<long>(s0);
    end = static_cast<long>(e0);
    current = static_cast<long>(c0);
    live = static_cast<long>(l0);
    same = static_cast<long>(m0);
  }
  __device__ __forceinline__ void store(const OscRef& o) const {
    o.f(kOscStart) = static_cast<double>(start);
    o.f(kOscEnd) = static_cast<double>(end);
    o.f(kOscCurrent) = static_cast<double>(current);
    o.f(kOscLive) = static_cast<double>(live);
    o.f(kOscSame) = static_cast<double>(same);
  }
  // Queue::dequeue (the value leaves DENSE's multiset too)
  __device__ __forceinline__ void dequeue(int w) {
    start = (start == w - 1) ? 0 : start + 1;
    if (2 * q_size(start, end, w) <= w) {
      current = current + 1;
      if (current == w) current = 0;
    }
    live -= 1;
  }
};

// OscillationAnalysis::checkCritPoint (oscillation.ipp:110-119): the middle
// value is a peak when it equals the window's maximum and not its minimum,
// a trough when it equals the minimum -- that is, a peak when no live value
// lies above it and some lies below, a trough when none lies below.  The
// window is scanned from both ends inwards, four values from each end at a
// time, and the scan stops as soon as values above and below have both been
// seen, so only an extreme middle value costs a whole pass -- and a flat
// window (every live value equal, known from the run of equal newest
// values, and equal to the middle value) none: the middle value is then a
// trough.  A middle index
// of -1 (DENSE reads contents[-1]), an empty window or a NaN middle value
// gives no critical point; NaN values in the window compare neither above
// nor below (DENSE keeps them in a std::multiset, whose order NaN breaks).
__device__ __forceinline__ void osc_check(const OscRef& o, const OscQueue& q, const double* win, int m, int w,
                                          double samples, const AnalysisDesc& A) {
  if (q.current < 0 || q.live <= 0) return;
  const double mid = win[static_cast<size_t>(q.current) * m];
  if (isnan(mid)) return;
  bool above = false, below = false;
  if (q.same >= q.live && mid == win[static_cast<size_t>(q.end) * m]) {
    // every live value equals the newest one, and so mid (a run of equal
    // values holds no NaN)
    double t = (samples - static_cast<double>(A.range_steps / 2)) * A.interval + A.t0;
    t = (0.0 < t) ? t : 0.0;
    osc_add_crit(o, t, mid, false);
    return;
  }
  long lo = q.start, hi = q.end;  // oldest and newest live slots
  long left = q.live;             // live values not yet looked at
  while (left > 0 && !(above && below)) {
    // slots past the live values hold mid, which is neither above nor below
    double x[8];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool a0 = left > 2 * u, a1 = left > 2 * u + 1;
      x[2 * u] = a0 ? win[static_cast<size_t>(lo) * m] : mid;
      x[2 * u + 1] = a1 ? win[static_cast<size_t>(hi) * m] : mid;
      if (a0) lo = (lo == w - 1) ? 0 : lo + 1;
      if (a1) hi = (hi == 0) ? w - 1 : hi - 1;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      above = above || (x[u] > mid);
      below = below || (x[u] < mid);
    }
    left -= 8;
  }
  if (above && below) return;
  double t = (samples - static_cast<double>(A.range_steps / 2)) * A.interval + A.t0;
  t = (0.0 < t) ? t : 0.0;
  if (!above && below) osc_add_crit(o, t, mid, true);
  else if (!below) osc_add_crit(o, t, mid, false);
}

__device__ __forceinline__ OscRef osc_ref(double* st, const AnalysisDesc& A, int i, int cc) {
  const size_t nm = static_cast<size_t>(A.nsp) * (A.cmax - A.cmin);
  return OscRef{st + 2 + static_cast<size_t>(i) * (A.cmax - A.cmin) + cc, nm};
}

__device__ __forceinline__ double* osc_window(double* st, const AnalysisDesc& A, int i, int cc) {
  const int m = A.cmax - A.cmin, w = A.range_steps + 1;
  const size_t nm = static_cast<size_t>(A.nsp) * m;
  return st + 2 + nm * kOscFields + static_cast<size_t>(i) * w * m + cc;
}

// OscillationAnalysis::update / get_peaks_and_troughs (oscillation.ipp:
// 86-103, 154-160) for thread c's cell, species in observation order,
// stopping at the first species whose window is still short.
template <typename Vals>
__device__ __forceinline__ void osc_cell_update(double* st, const AnalysisDesc& A, const Vals& vals, int c,
                                                double samples) {
  if (c < A.cmin || c >= A.cmax) return;
  const int n = A.nsp, m = A.cmax - A.cmin, w = A.range_steps + 1;
  const int cc = c - A.cmin;
  for (int i = 0; i < n; ++i) {
    const OscRef o = osc_ref(st, A, i, cc);
    double* win = osc_window(st, A, i, cc);
    const double added = vals(A.slot[i], c);
    OscQueue q;
    q.load(o);
    // the run of equal newest values (NaN equals nothing)
    const double newest = q.live > 0 ? win[static_cast<size_t>(q.end) * m] : added;
    q.same = (q.live > 0 && newest == added) ? q.same + 1 : (added == added ? 1 : 0);
    // Queue::enqueue; the multiset gains `added`
    q.end = (q.end == w - 1) ? 0 : q.end + 1;
    win[static_cast<size_t>(q.end) * m] = added;
    q.live += 1;
    if (2 * q_size(q.start, q.end, w) >= w) {
      q.current = q.current + 1;
      if (q.current == w) q.current = 0;
    }
    if (q_size(q.start, q.end, w) == A.range_steps + 1) q.dequeue(w);
    const bool stop = q_size(q.start, q.end, w) < A.range_steps / 2;
    if (!stop) osc_check(o, q, win, m, w, samples, A);
    q.store(o);
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
  double samples = samples0;
  for (int i = 0; i < n; ++i) {
    const OscRef o = osc_ref(st, A, i, cc);
    double* win = osc_window(st, A, i, cc);
    samples = samples0;
    OscQueue q;
    q.load(o);
    for (;;) {
      if (!(q_size(q.start, q.end, w) >= (A.range_steps / 2) && q.live > 0)) break;
      q.dequeue(w);
      osc_check(o, q, win, m, w, samples, A);
      samples += 1.0;
    }
    q.store(o);
    osc_fold_last(o);
    const double np = o.f(kOscNumPeaks), nt = o.f(kOscNumTroughs);
    o.f(kOscAmp) = ((o.f(kOscPeakSum) / np) - (o.f(kOscTroughSum) / nt)) / 2;
    o.f(kOscPer) = o.f(kOscCycleSum) / o.f(kOscCycles);
    o.f(kOscAvgPeak) = (np != 0.0) ? o.f(kOscPeakSum) / np : o.f(kOscPeakSum);
  }
  if (cc == m - 1) st[0] = samples;
}

// Where the analyses read the sampled state: the shared staging buffer of
// the register kernel, or the lag-0 rows of the rings in the memory kernel.
struct SmemVals {
  const double* base;
  int blk;
  __device__ __forceinline__ double operator()(int slot, int cell) const { return base[slot * blk + cell]; }
};

template <typename T>
struct RingVals {
  T* const* rows;  // lag-0 row of each observed species (shared)
  T* const* comp;  // FP32 Kahan: compensation row of each observed species (shared), else null
  __device__ __forceinline__ double operator()(int slot, int cell) const {
    // with Kahan compensation the analyses see the compensated value,
    // state minus its running error, in double
    const double v = static_cast<double>(rows[slot][cell]);
    return comp ? v - static_cast<double>(comp[slot][cell]) : v;
  }
};

// One analysis sample of a set at `age` (measurement/base.ipp:4-9): every
// analysis records the time; those whose window contains it update, over
// the cells c0, c0 + stride, ... this thread handles.  Returns whether a
// concentration check failed for one of them.
template <typename Vals>
__device__ __forceinline__ bool analyses_sample(const StepArgs& a, double* anl, const Vals& vals, int tid, int c0,
                                                int stride, int n, double age, const double* samples) {
  bool bad = false;
  for (int ai = 0; ai < a.n_analyses; ++ai) {
    const AnalysisDesc& A = a.analyses[ai];
    double* st = anl + A.off;
    const bool in_range = !(age < A.t0 || age >= A.t1);
    if (A.kind == kBasic) {
      if (tid == 0) st[3 * A.nsp + 1] = age;
      if (!in_range) continue;
      for (int c = c0; c < n; c += stride) basic_cell_update(st, A, vals, c);
      if (tid < 32) basic_range_fold(st, A, vals, tid);
      if (tid == 0) st[3 * A.nsp] += 1.0;
    } else if (A.kind == kOscillation) {
      if (tid == 0) st[1] = age;
      if (!in_range) continue;
      for (int c = c0; c < n; c += stride) osc_cell_update(st, A, vals, c, samples[ai]);
      if (tid == 0) st[0] = samples[ai] + 1.0;
    } else if (A.kind == kTrajectory) {
      // csvw_sim::update (io/csvw_sim.ipp:17-91): every observed species
      // of every analysed cell at every sample
      if (tid == 0) st[1] = age;
      if (!in_range) continue;
      const long k = static_cast<long>(st[0]);
      if (k < A.range_steps) {
        const int m = A.cmax - A.cmin;
        double* vals_k = st + 2 + A.range_steps + static_cast<size_t>(k) * A.nsp * m;
        for (int c = c0; c < n; c += stride) {
          if (c < A.cmin || c >= A.cmax) continue;
          for (int i = 0; i < A.nsp; ++i) vals_k[static_cast<size_t>(i) * m + (c - A.cmin)] = vals(A.slot[i], c);
        }
        if (tid == 0) st[2 + k] = age;
      }
      if (tid == 0) st[0] = static_cast<double>(k + 1);
    } else if (A.kind == kConcCheck) {
      if (tid == 0) st[0] = age;
      if (!in_range) continue;
      for (int c = c0; c < n; c += stride) {
        if (c < A.cmin || c >= A.cmax) continue;
        for (int i = 0; i < A.nsp; ++i) {
          const double x = vals(A.slot[i], c);
          if (x < A.lo || x > A.hi) bad = true;
        }
      }
    }
  }
  return bad;
}

// ---------------------------------------------------------------- kernel

// kThreads / kMinBlocks: 224 threads with two resident CTAs per SM for sets
// of up to 224 cells (128 registers: the fourteen warps put four on the
// busiest of the SM's four sub-partitions, whose register file holds
// 16384), 256 threads with one CTA per SM above that.
template <typename T, bool kKahan, int kThreads, int kMinBlocks, bool kUniform>
__global__ void __launch_bounds__(kThreads, kMinBlocks) dense_step_kernel(const StepArgs a, const int* set_list) {
  // dynamic shared memory: sampled state [NS][blockDim] (doubles, only with
  // analyses) | truncated delays [ND][blockDim] | the set's CSR lists
  extern __shared__ double s_dyn[];
  double* s_vals = s_dyn;
  __shared__ int s_S[kNS], s_mask[kNS];
  __shared__ int64_t s_roff[kNS];
  __shared__ T s_prm[kNP];
  __shared__ int s_flags;
  __shared__ double s_samples[kMaxAnalyses];
  __shared__ int s_olag[kND > 0 ? kND * kNS : 1], s_nlag[kND > 0 ? kND * kNS : 1];

  const int set = set_list[blockIdx.x];
  const SetDesc& sd = a.sets[set];
  const int n = sd.n_cells;
  const int blk = blockDim.x;
  const int c = threadIdx.x;
  const bool active = c < n;

  const SetProgress pg = a.prog[set];
  if ((pg.status & (kSetDropped | kSetNotRunnable)) || pg.finalized) return;

  const int pstride = sd.param_stride;
  if (c < kNS) {
    s_S[c] = sd.S[c];
    s_mask[c] = sd.D[c] - 1;
    s_roff[c] = sd.ring_off[c];
  }
  const T* P = static_cast<const T*>(a.params) + sd.param_base;
  if (pstride == 0) {
    for (int i = c; i < kNP; i += blk) s_prm[i] = P[i];
  }
  if (c == 0) s_flags = 0;
  double* anl = a.anl + sd.anl_base;
  if (c < a.n_analyses) s_samples[c] = anl[a.analyses[c].off];
  __syncthreads();

  const int cell = active ? c : 0;
  // parameters: the shared row of the set, or this cell's column of the
  // set's [NP][n] block (read through L1)
  const T* prm = pstride == 0 ? s_prm : P + cell;
  const int ps = pstride == 0 ? 1 : n;
  if (kUniform) {
    // lag tables of this set, with the exact lag rules of the checked path
    for (int i = c; i < kND * kNS; i += blk) {
      const int d = i / kNS, sp = i % kNS;
      const int k = static_cast<int>(s_prm[kNR + d]);
      const int S = s_S[sp], m = s_mask[sp];
      int ol = -1, nl = -1;
      if (k >= 0 && k <= S) {  // else: the checked path records a bad delay
        ol = k - 1 < 0 ? S - 1 : k - 1;
        if (ol != 0 && ol > m) ol = -1;
        nl = k == S ? 0 : k;
        if (nl >= m || nl == S - 1) nl = -1;
      }
      s_olag[i] = ol;
      s_nlag[i] = nl;
    }
  }
  int* s_kd = reinterpret_cast<int*>(s_dyn + (a.n_analyses > 0 ? a.n_vals * blk : 0));
  int* s_csr = s_kd + kND * blk;
#pragma unroll
  for (int d = 0; d < kND; ++d) s_kd[d * blk + c] = static_cast<int>(prm[(kNR + d) * ps]);

  T cur[kNS];
  T comp[kNS];
  T* state = static_cast<T*>(a.state) + sd.cell_base * (2 * kNS);
#pragma unroll
  for (int sp = 0; sp < kNS; ++sp) {
    cur[sp] = state[static_cast<size_t>(sp) * n + cell];
    comp[sp] = kKahan ? state[static_cast<size_t>(kNS + sp) * n + cell] : T(0);
  }
  const int* nbr_off = a.nbr_off + sd.nbr_base;
  const int nb0 = nbr_off[cell];
  const int nnbr = nbr_off[cell + 1] - nb0;
  const int* nbr = a.nbr_idx + nb0;
  if (a.csr_in_smem) {
    // the set's neighbour ids, [edges], in shared memory
    const int e0 = nbr_off[0], ne = nbr_off[n] - e0;
    for (int e = c; e < ne; e += blk) s_csr[e] = a.nbr_idx[e0 + e];
    nbr = s_csr + (nb0 - e0);
  }
  __syncthreads();

  int err = 0;
  T* ring = static_cast<T*>(a.ring) + sd.ring_base;
  int64_t step = pg.step;
  // per-set constants of the history reads in registers (only the entries
  // the model's reads use stay live); through shared memory they would be
  // reloaded after every ring store
  int64_t lroff[kNS];
  int lmask[kNS];
#pragma unroll
  for (int sp = 0; sp < kNS; ++sp) {
    lroff[sp] = s_roff[sp];
    lmask[sp] = s_mask[sp];
  }
  int lolag[kND > 0 ? kND * kNS : 1], lnlag[kND > 0 ? kND * kNS : 1];
#pragma unroll
  for (int i = 0; i < kND * kNS; ++i) {
    lolag[i] = s_olag[i];
    lnlag[i] = s_nlag[i];
  }
  DeviceContext<T, kUniform> ctx{cur,  prm,    ps,   s_kd + cell, blk,    s_S,    lmask, lroff, ring,
                                 static_cast<int>(step), nbr, nnbr, T(1) / static_cast<T>(nnbr), lolag, lnlag,
                                 false, n, cell, &err};

  const T dt = static_cast<T>(a.dt);
  int chunk = pg.chunk;
  const int chunk_end = (a.chunk_count < 0 || sd.n_chunks - chunk < a.chunk_count)
                            ? sd.n_chunks
                            : chunk + a.chunk_count;
  double age = pg.age;
  bool dropped = false;

  for (; chunk < chunk_end; ++chunk) {
    // ---- analyses sample the state at `age` (measurement/base.ipp:4-9)
    if (a.n_analyses > 0) {
#pragma unroll
      for (int sp = 0; sp < kNS; ++sp) {
        const int row = a.val_slot[sp];
        if (row >= 0)
          s_vals[row * blk + c] = static_cast<double>(cur[sp]) - (kKahan ? static_cast<double>(comp[sp]) : 0.0);
      }
      __syncthreads();
      const bool bad = analyses_sample(a, anl, SmemVals{s_vals, blk}, c, c, n + blk, n, age, s_samples);
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
        // DENSE evaluates every rate, then adds rate * delta reaction by
        // reaction (determ.cpp:58-72).  Each species' accumulator sees the
        // same additions in the same order when each rate is folded in as
        // soon as it is known, which keeps one rate live instead of all.
        T dsp[kNS];
#pragma unroll
        for (int sp = 0; sp < kNS; ++sp) dsp[sp] = T(0);
#define REACTION(name)                                                        \
  {                                                                           \
    const T rate_ = reaction<name>::active_rate(ctx);                         \
    _Pragma("unroll") for (int j = 0; j < num_deltas_##name; j++)             \
        dsp[delta_ids_##name[j]] += rate_ * static_cast<T>(deltas_##name[j]); \
  }
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
        const int w = ctx.step + 1;
#pragma unroll
        for (int sp = 0; sp < kNS; ++sp) {
          const int m = s_mask[sp];
          if (m >= 0) ring[s_roff[sp] + static_cast<int64_t>(w & m) * n + c] = nxt[sp];
        }
      }
      __syncthreads();
      ctx.step += 1;
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

// Lag tables of one set (kUniform sets), with the lag rules of the checked
// path: own reads (k-1) mod S, neighbour reads k mod S; -1 where the
// checked path must run (out-of-range delay, unstaged lag, same-step row).
template <typename T>
__device__ __forceinline__ void fill_lag_tables(const T* s_prm, const int* s_S, const int* s_mask, int* s_olag,
                                                int* s_nlag, int tid, int nthreads) {
  for (int i = tid; i < kND * kNS; i += nthreads) {
    const int d = i / kNS, sp = i % kNS;
    const int k = static_cast<int>(s_prm[kNR + d]);
    const int S = s_S[sp], m = s_mask[sp];
    int ol = -1, nl = -1;
    if (k >= 0 && k <= S) {
      ol = k - 1 < 0 ? S - 1 : k - 1;
      if (ol != 0 && ol > m) ol = -1;
      nl = k == S ? 0 : k;
      if (nl >= m || nl == S - 1) nl = -1;
    }
    s_olag[i] = ol;
    s_nlag[i] = nl;
  }
}

// The memory-state step kernel: one CTA per set, any number of cells, and
// cell-dependency levels.  Every species lives in its ring (the lag-0 row
// is the state); each step visits the levels in order, the cells of a level
// in parallel (thread t takes the level's cells t, t + blockDim, ...), with
// a barrier after each level.  A set whose neighbour reads see the row
// written in the same step gets one level per step of its lower-numbered
// neighbour chain (level(c) = 1 + max level of its lower-numbered
// neighbours), which reproduces DENSE's cell-ordered loop; other sets have
// one level holding every cell.
template <typename T, bool kKahan, bool kUniform>
__global__ void __launch_bounds__(256, 2) dense_step_mem_kernel(const StepArgs a, const int* set_list) {
  __shared__ T s_rc[kRcTable];  // RN(1 / count) for neighbour counts below kRcTable
  __shared__ int s_S[kNS], s_mask[kNS];
  __shared__ int64_t s_roff[kNS];
  __shared__ T s_prm[kNP];
  __shared__ int s_flags;
  __shared__ double s_samples[kMaxAnalyses];
  __shared__ int s_olag[kND > 0 ? kND * kNS : 1], s_nlag[kND > 0 ? kND * kNS : 1];
  __shared__ T* s_rows[kNS];
  __shared__ T* s_crows[kNS];

  const int set = set_list[blockIdx.x];
  const SetDesc& sd = a.sets[set];
  const int n = sd.n_cells;
  const int blk = blockDim.x;
  const int tid = threadIdx.x;

  const SetProgress pg = a.prog[set];
  if ((pg.status & (kSetDropped | kSetNanParam)) || pg.finalized) return;

  const int pstride = sd.param_stride;
  const T* P = static_cast<const T*>(a.params) + sd.param_base;
  for (int i = tid; i < kRcTable; i += blk) s_rc[i] = i > 0 ? T(1) / static_cast<T>(i) : T(0);
  for (int i = tid; i < kNS; i += blk) {  // blocks may be a single warp
    s_S[i] = sd.S[i];
    s_mask[i] = sd.D[i] - 1;
    s_roff[i] = sd.ring_off[i];
  }
  if (pstride == 0)
    for (int i = tid; i < kNP; i += blk) s_prm[i] = P[i];
  if (tid == 0) s_flags = 0;
  double* anl = a.anl + sd.anl_base;
  if (tid < a.n_analyses) s_samples[tid] = anl[a.analyses[tid].off];
  __syncthreads();
  if (kUniform) fill_lag_tables(s_prm, s_S, s_mask, s_olag, s_nlag, tid, blk);
  __syncthreads();

  T* ring = static_cast<T*>(a.ring) + sd.ring_base;
  T* comp_base = static_cast<T*>(a.state) + sd.cell_base * (2 * kNS) + static_cast<int64_t>(kNS) * n;
  const int* nbr_off = a.nbr_off + sd.nbr_base;
  const int* lvl_off = a.lvl_off + sd.lvl_base;
  const int* lvl_cells = a.lvl_cells + sd.cell_base;
  const int n_levels = sd.n_levels;
  const bool ordered = sd.ordered != 0;
  int err = 0;
  const T dt = static_cast<T>(a.dt);
  int chunk = pg.chunk;
  const int chunk_end = (a.chunk_count < 0 || sd.n_chunks - chunk < a.chunk_count)
                            ? sd.n_chunks
                            : chunk + a.chunk_count;
  double age = pg.age;
  int64_t step = pg.step;
  bool dropped = false;

  for (; chunk < chunk_end; ++chunk) {
    if (a.n_analyses > 0) {
      for (int i = tid; i < kNS; i += blk) {
        const int row = a.val_slot[i];
        if (row >= 0) {
          s_rows[row] = ring + s_roff[i] + static_cast<int64_t>(step & s_mask[i]) * n;
          s_crows[row] = comp_base + static_cast<int64_t>(i) * n;
        }
      }
      __syncthreads();
      const bool bad =
          analyses_sample(a, anl, RingVals<T>{s_rows, kKahan ? s_crows : nullptr}, tid, tid, blk, n, age, s_samples);
      if (bad) atomicOr(&s_flags, 1);
      __syncthreads();
      if (tid < a.n_analyses) s_samples[tid] = anl[a.analyses[tid].off];
      if (s_flags & 1) {
        dropped = true;
        break;
      }
    }
    for (int s = 0; s < sd.steps_per_chunk; ++s) {
      const int st32 = static_cast<int>(step);
      for (int l = 0; l < n_levels; ++l) {
        for (int i = lvl_off[l] + tid; i < lvl_off[l + 1]; i += blk) {
          const int cell = lvl_cells[i];
          T cur[kNS];
#pragma unroll
          for (int sp = 0; sp < kNS; ++sp)
            cur[sp] = ring[s_roff[sp] + static_cast<int64_t>(st32 & s_mask[sp]) * n + cell];
          const T* prm = pstride == 0 ? s_prm : P + cell;
          const int ps = pstride == 0 ? 1 : n;
          const int nb0 = nbr_off[cell];
          const int cnt = nbr_off[cell + 1] - nb0;
          DeviceContext<T, kUniform> ctx{cur,    prm,    ps,     nullptr, 0,      s_S,  s_mask, s_roff,
                                         ring,   st32,   a.nbr_idx + nb0, cnt,
                                         cnt < kRcTable ? s_rc[cnt] : T(1) / static_cast<T>(cnt),
                                         s_olag, s_nlag, ordered, n,      cell,   &err};
          T dsp[kNS];
#pragma unroll
          for (int sp = 0; sp < kNS; ++sp) dsp[sp] = T(0);
#define REACTION(name)                                                        \
  {                                                                           \
    const T rate_ = reaction<name>::active_rate(ctx);                         \
    _Pragma("unroll") for (int j = 0; j < num_deltas_##name; j++)             \
        dsp[delta_ids_##name[j]] += rate_ * static_cast<T>(deltas_##name[j]); \
  }
#include "reactions_list.hpp"
#undef REACTION
#pragma unroll
          for (int sp = 0; sp < kNS; ++sp) {
            T nxt;
            if (kKahan) {
              T& cp = comp_base[static_cast<int64_t>(sp) * n + cell];
              const T y = dt * dsp[sp] - cp;
              const T t = cur[sp] + y;
              cp = (t - cur[sp]) - y;
              nxt = t;
            } else {
              nxt = cur[sp] + dt * dsp[sp];
            }
            ring[s_roff[sp] + static_cast<int64_t>((st32 + 1) & s_mask[sp]) * n + cell] = nxt;
          }
        }
        __syncthreads();
      }
      ++step;
    }
    age += a.interval;
  }

  // lag-0 state to the state block (what read_state returns)
  T* state = static_cast<T*>(a.state) + sd.cell_base * (2 * kNS);
  for (int i = tid; i < kNS * n; i += blk) {
    const int sp = i / n, cell = i % n;
    state[i] = ring[s_roff[sp] + static_cast<int64_t>(step & s_mask[sp]) * n + cell];
  }
  if (err) atomicOr(&s_flags, err << 1);
  if (tid < a.n_analyses) s_samples[tid] = anl[a.analyses[tid].off];
  __syncthreads();
  const int status = pg.status | (dropped ? kSetDropped : 0) | (s_flags >> 1);
  const bool finish = !dropped && chunk >= sd.n_chunks;
  if (finish) {
    for (int ai = 0; ai < a.n_analyses; ++ai) {
      const AnalysisDesc& A = a.analyses[ai];
      if (A.kind == kOscillation)
        for (int c = tid; c < n; c += blk) osc_cell_finalize(anl + A.off, A, c, s_samples[ai]);
    }
  }
  if (tid == 0) {
    SetProgress out = pg;
    out.step = step;
    out.chunk = chunk;
    out.age = age;
    out.status = status;
    out.finalized = finish ? 1 : 0;
    a.prog[set] = out;
  }
}

// ------------------------------------------------------------ wave kernel
// Context of the wave kernel.  Rows are indexed modulo each species' row
// count D (not a power of two: a species read by neighbours at lag S-1
// keeps exactly S + 1 rows), from the lag-0 row r0 the kernel advances per
// step; every species' rows sit behind a base pointer, in shared or global
// memory; a cell's neighbour ids come from its 16-byte record.
template <typename T, bool kUniform>
struct WaveContext {
  const T* cur;            // this cell's lag-0 state [NS] (registers)
  const T* prm;            // parameters: shared row (pstride 1) or this cell's column (pstride n)
  int pstride;
  const int* S;            // DENSE ring sizes (registers)
  const int* D;            // rows kept per species (registers)
  const int* r0;           // row holding lag 0, per species (registers)
  T* const* base;          // row 0 of each species, shared or global (registers)
  T* const* wrow;          // the row this step writes, per species (registers)
  const uint16_t* nbr;     // this cell's neighbour ids, ascending (registers)
  int nnbr;
  T rc;                    // RN(1 / nnbr)
  const int* olag;         // kUniform: own-read lag table [ND][NS] (shared)
  const int* nlag;         // kUniform: neighbour-read lag table [ND][NS] (shared)
  int n_cells;
  int cell;
  int* err;

  // DENSE's ring size: max delay / dt + 2, so 2 for every species of a
  // model without delay reactions
  __device__ __forceinline__ int ring_size(specie_id sp) const { return kND == 0 ? 2 : S[sp]; }

  __device__ __forceinline__ const T* row(specie_id sp, int lag) const {
    const int r = r0[sp] - lag;
    return base[sp] + (r < 0 ? r + D[sp] : r) * n_cells;
  }

  __device__ __forceinline__ T average(T sum) const {
    const T avg = div_by_count(sum, static_cast<T>(nnbr), rc);
    return isnan(avg) ? T(0) : avg;
  }

  // (checks set error bits without leaving the straight-line path; a set
  // with an error bit is reported, not its values)
  __device__ __forceinline__ T own(specie_id sp, int k) const {
    const int s = ring_size(sp);
    int lag = k - 1;
    if (lag < 0) lag += s;
    if (static_cast<unsigned>(k) > static_cast<unsigned>(s)) {
      if (k < 0 || k > s + 1) *err |= kSetBadDelay;
      lag = ((k - 1) % s + s) % s;
    }
    if (lag == 0) return cur[sp];
    *err |= lag >= D[sp] ? kSetUnstagedLag : 0;
    return row(sp, lag)[cell];
  }

  __device__ __forceinline__ T own_lag(specie_id sp, int lag) const {
    if (lag == 0) return cur[sp];
    return row(sp, lag)[cell];
  }

  __device__ __forceinline__ T nbr_lag(specie_id sp, int lag) const {
    const T* r = row(sp, lag);
    T sum = T(0);
#pragma unroll
    for (int e = 0; e < kWaveMaxNbrs; ++e)
      if (e < nnbr) sum += r[nbr[e]];
    return average(sum);
  }

  // Lag k mod S.  Lag S-1 is the row DENSE's cell-ordered loop is writing
  // in this step: lower-numbered neighbours (all in lower levels) have
  // their new value there, the others the value of S steps back.
  __device__ __forceinline__ T nbr_avg(specie_id sp, int k) const {
    const int s = ring_size(sp);
    int lag = k;
    if (static_cast<unsigned>(k) >= static_cast<unsigned>(s)) {
      if (k < 0 || k > s) *err |= kSetBadDelay;
      lag = (k % s + s) % s;
    }
    if (lag == s - 1 && s > 1) {
      *err |= D[sp] < s + 1 ? kSetOrderedReads : 0;
      const T* fresh = wrow[sp];
      const T* old = row(sp, lag);
      T sum = T(0);
#pragma unroll
      for (int e = 0; e < kWaveMaxNbrs; ++e) {
        const int v = nbr[e];
        if (e < nnbr) sum += (v < cell ? fresh : old)[v];
      }
      return average(sum);
    }
    *err |= lag >= D[sp] - 1 ? kSetUnstagedLag : 0;
    return nbr_lag(sp, lag);
  }

  __device__ __forceinline__ T getCon(specie_id sp) const { return cur[sp]; }
  __device__ __forceinline__ T getCon(specie_id sp, int k) const { return own(sp, k); }
  __device__ __forceinline__ T getCon(specie_id sp, DelayArg<T> d) const {
    if (kUniform) {
      const int lag = olag[d.dr * kNS + sp];
      if (lag >= 0) return own_lag(sp, lag);
    }
    return own(sp, d.k);
  }
  __device__ __forceinline__ T calculateNeighborAvg(specie_id sp, int k = 0) const { return nbr_avg(sp, k); }
  __device__ __forceinline__ T calculateNeighborAvg(specie_id sp, DelayArg<T> d) const {
    if (kUniform) {
      const int lag = nlag[d.dr * kNS + sp];
      if (lag >= 0) return nbr_lag(sp, lag);
    }
    return nbr_avg(sp, d.k);
  }
  __device__ __forceinline__ T getRate(reaction_id r) const { return prm[r * pstride]; }
  __device__ __forceinline__ DelayArg<T> getDelay(delay_reaction_id d) const {
    return DelayArg<T>{prm, pstride, static_cast<int>(d), static_cast<int>(prm[(kNR + d) * pstride])};
  }
  __device__ __forceinline__ T getCritVal(critspecie_id c) const { return prm[(kNR + kND + c) * pstride]; }
};

// The wave kernel: one CTA per ordered set (neighbour reads of the row
// being written, as in DENSE's cell-ordered loop), one barrier per
// dependency level, a thread per cell of a level.  The set's level offsets
// and as many species' rows (and then its cell records) as fit stay in
// shared memory for the whole launch: loaded from the set's history block
// at entry, stored back at exit.  Records left in global memory are
// fetched one level ahead.
// kThreads / kMinBlocks: 256 threads, two CTAs per SM (128 registers), or
// single-warp CTAs with up to 32 per SM (64 registers) for sets whose rows
// stay in global memory.  kAllShared: every species' rows and the records
// are in shared memory (the compiler then addresses them as such).
template <typename T, bool kKahan, bool kUniform, int kThreads, int kMinBlocks, bool kAllShared>
__global__ void __launch_bounds__(kThreads, kMinBlocks) dense_step_wave_kernel(const StepArgs a, const int* set_list) {
  extern __shared__ __align__(16) unsigned char w_dyn[];
  __shared__ int s_S[kNS], s_D[kNS];
  __shared__ T* s_base[kNS];
  __shared__ T s_prm[kNP];
  __shared__ int s_flags;
  __shared__ double s_samples[kMaxAnalyses];
  __shared__ int s_olag[kND > 0 ? kND * kNS : 1], s_nlag[kND > 0 ? kND * kNS : 1];
  __shared__ T* s_rows[kNS];
  __shared__ T* s_crows[kNS];
  __shared__ T s_rc[kWaveMaxNbrs + 1];  // RN(1 / count)

  const int set = set_list[blockIdx.x];
  const SetDesc& sd = a.sets[set];
  const int n = sd.n_cells;
  const int blk = blockDim.x;
  const int tid = threadIdx.x;

  const SetProgress pg = a.prog[set];
  if ((pg.status & (kSetDropped | kSetNotRunnable)) || pg.finalized) return;

  const int pstride = sd.param_stride;
  const T* P = static_cast<const T*>(a.params) + sd.param_base;
  T* ring = static_cast<T*>(a.ring) + sd.ring_base;
  for (int i = tid; i <= kWaveMaxNbrs; i += blk) s_rc[i] = i > 0 ? T(1) / static_cast<T>(i) : T(0);
  for (int i = tid; i < kNS; i += blk) {
    s_S[i] = sd.S[i];
    s_D[i] = sd.D[i];
    s_base[i] = sd.smem_off[i] >= 0 ? reinterpret_cast<T*>(w_dyn + sd.smem_off[i]) : ring + sd.ring_off[i];
  }
  if (pstride == 0)
    for (int i = tid; i < kNP; i += blk) s_prm[i] = P[i];
  if (tid == 0) s_flags = 0;
  double* anl = a.anl + sd.anl_base;
  if (tid < a.n_analyses) s_samples[tid] = anl[a.analyses[tid].off];

  // level offsets (16-bit) and cell records: shared, or records global
  const int n_levels = sd.n_levels;
  uint16_t* t_lvl = reinterpret_cast<uint16_t*>(w_dyn + sd.lvl_smem_off);
  {
    const int* lvl_off = a.lvl_off + sd.lvl_base;
    for (int i = tid; i <= n_levels; i += blk) t_lvl[i] = static_cast<uint16_t>(lvl_off[i]);
  }
  const uint4* g_rec = a.wave_rec + sd.rec_base;
  const bool rec_shared = sd.topo_off >= 0;
  const uint4* recs = kAllShared ? reinterpret_cast<const uint4*>(w_dyn + sd.topo_off)
                                 : (rec_shared ? reinterpret_cast<const uint4*>(w_dyn + sd.topo_off) : g_rec);
  if (rec_shared) {
    uint4* dst = reinterpret_cast<uint4*>(w_dyn + sd.topo_off);
    for (int i = tid; i < n; i += blk) dst[i] = g_rec[i];
  }
  for (int sp = 0; sp < kNS; ++sp) {
    if (sd.smem_off[sp] < 0) continue;
    T* dst = reinterpret_cast<T*>(w_dyn + sd.smem_off[sp]);
    const T* src = ring + sd.ring_off[sp];
    const int rows = sd.D[sp] * n;
    for (int i = tid; i < rows; i += blk) dst[i] = src[i];
  }
  // FP32 Kahan terms [kNS][n]: staged in shared memory when planned there
  T* const comp_g = static_cast<T*>(a.state) + sd.cell_base * (2 * kNS) + static_cast<int64_t>(kNS) * n;
  const bool comp_shared = kKahan && sd.comp_smem_off >= 0;
  T* const comp_base = comp_shared ? reinterpret_cast<T*>(w_dyn + sd.comp_smem_off) : comp_g;
  if (comp_shared)
    for (int i = tid; i < kNS * n; i += blk) comp_base[i] = comp_g[i];
  __syncthreads();
  if (kUniform) {
    // the lag tables' bound checks take the row count as D - 1
    for (int i = tid; i < kND * kNS; i += blk) {
      const int d = i / kNS, sp = i % kNS;
      const int k = static_cast<int>(s_prm[kNR + d]);
      const int S = s_S[sp], m = s_D[sp] - 1;
      int ol = -1, nl = -1;
      if (k >= 0 && k <= S) {
        ol = k - 1 < 0 ? S - 1 : k - 1;
        if (ol != 0 && ol > m) ol = -1;
        nl = k == S ? 0 : k;
        if (nl >= m || nl == S - 1) nl = -1;
      }
      s_olag[i] = ol;
      s_nlag[i] = nl;
    }
  }
  __syncthreads();

  int err = 0;
  const T dt = static_cast<T>(a.dt);
  int chunk = pg.chunk;
  const int chunk_end = (a.chunk_count < 0 || sd.n_chunks - chunk < a.chunk_count)
                            ? sd.n_chunks
                            : chunk + a.chunk_count;
  double age = pg.age;
  int64_t step = pg.step;
  bool dropped = false;
  // per-set constants and per-step row pointers in registers
  int lS[kNS], lD[kNS], r0[kNS];
  T* lbase[kNS];
  T* lcur[kNS];
  T* lw[kNS];
#pragma unroll
  for (int sp = 0; sp < kNS; ++sp) {
    lS[sp] = s_S[sp];
    lD[sp] = s_D[sp];
    lbase[sp] = kAllShared ? reinterpret_cast<T*>(w_dyn + sd.smem_off[sp]) : s_base[sp];
    r0[sp] = 0;
    lcur[sp] = lw[sp] = lbase[sp];
  }
  // thread groups, one per wavefront
  const int fronts = sd.wave_fronts;
  const int delta = sd.wave_delta;
  const int gsz = blk / fronts;
  const int grp = tid / gsz, gtid = tid % gsz;

  for (; chunk < chunk_end; ++chunk) {
    if (a.n_analyses > 0) {
      for (int i = tid; i < kNS; i += blk) {
        const int row = a.val_slot[i];
        if (row >= 0) {
          s_rows[row] = s_base[i] + static_cast<int64_t>(step % s_D[i]) * n;
          s_crows[row] = comp_base + static_cast<int64_t>(i) * n;
        }
      }
      __syncthreads();
      const bool bad =
          analyses_sample(a, anl, RingVals<T>{s_rows, kKahan ? s_crows : nullptr}, tid, tid, blk, n, age, s_samples);
      if (bad) atomicOr(&s_flags, 1);
      __syncthreads();
      if (tid < a.n_analyses) s_samples[tid] = anl[a.analyses[tid].off];
      if (s_flags & 1) {
        dropped = true;
        break;
      }
    }
    // the chunk's steps as overlapping wavefronts: in interval tau, group g
    // runs level tau - k * delta of the one step k in flight with
    // k = g (mod fronts); a barrier closes each interval
    const int S_chunk = sd.steps_per_chunk;
    const int n_intervals = S_chunk > 0 ? (S_chunk - 1) * delta + n_levels : 0;
    int kcur = -1;
    int rw[kNS];
    for (int tau = 0; tau < n_intervals; ++tau) {
      int kk = tau / delta;
      kk -= ((kk - grp) % fronts + fronts) % fronts;
      const int l = tau - kk * delta;
      if (grp < fronts && kk >= 0 && kk < S_chunk && l < n_levels) {
        if (kk != kcur) {
          // rows of step `step + kk`
          kcur = kk;
#pragma unroll
          for (int sp = 0; sp < kNS; ++sp) {
            r0[sp] = static_cast<int>((step + kk) % lD[sp]);
            rw[sp] = r0[sp] + 1 == lD[sp] ? 0 : r0[sp] + 1;
            lcur[sp] = lbase[sp] + r0[sp] * n;
            lw[sp] = lbase[sp] + rw[sp] * n;
          }
        }
        const int i1 = t_lvl[l + 1];
        for (int i = t_lvl[l] + gtid; i < i1; i += gsz) {
          const uint4 raw = recs[i];
          const int cell = static_cast<int>(raw.x & 0xFFFFu);
          const int cnt = static_cast<int>(raw.x >> 16);
          const uint16_t nb[6] = {static_cast<uint16_t>(raw.y & 0xFFFFu), static_cast<uint16_t>(raw.y >> 16),
                                  static_cast<uint16_t>(raw.z & 0xFFFFu), static_cast<uint16_t>(raw.z >> 16),
                                  static_cast<uint16_t>(raw.w & 0xFFFFu), static_cast<uint16_t>(raw.w >> 16)};
          T cur[kNS];
#pragma unroll
          for (int sp = 0; sp < kNS; ++sp) cur[sp] = lcur[sp][cell];
          const T* prm = pstride == 0 ? s_prm : P + cell;
          const int ps = pstride == 0 ? 1 : n;
          WaveContext<T, kUniform> ctx{cur,    prm,    ps, lS,   lD,   r0,  lbase, lw, nb, cnt, s_rc[cnt],
                                       s_olag, s_nlag, n,  cell, &err};
          T dsp[kNS];
#pragma unroll
          for (int sp = 0; sp < kNS; ++sp) dsp[sp] = T(0);
#define REACTION(name)                                                        \
  {                                                                           \
    const T rate_ = reaction<name>::active_rate(ctx);                         \
    _Pragma("unroll") for (int j = 0; j < num_deltas_##name; j++)             \
        dsp[delta_ids_##name[j]] += rate_ * static_cast<T>(deltas_##name[j]); \
  }
#include "reactions_list.hpp"
#undef REACTION
#pragma unroll
          for (int sp = 0; sp < kNS; ++sp) {
            T nxt;
            if (kKahan) {
              T& cp = comp_base[static_cast<int64_t>(sp) * n + cell];
              const T y = dt * dsp[sp] - cp;
              const T t = cur[sp] + y;
              cp = (t - cur[sp]) - y;
              nxt = t;
            } else {
              nxt = cur[sp] + dt * dsp[sp];
            }
            lw[sp][cell] = nxt;
          }
        }
      }
      __syncthreads();
    }
    step += S_chunk;
    age += a.interval;
  }

  // lag-0 state to the state block (what read_state returns), shared rows
  // back to the history block
  T* state = static_cast<T*>(a.state) + sd.cell_base * (2 * kNS);
  for (int i = tid; i < kNS * n; i += blk) {
    const int sp = i / n, cell = i % n;
    state[i] = s_base[sp][static_cast<int64_t>(step % s_D[sp]) * n + cell];
  }
  for (int sp = 0; sp < kNS; ++sp) {
    if (sd.smem_off[sp] < 0) continue;
    const T* src = reinterpret_cast<const T*>(w_dyn + sd.smem_off[sp]);
    T* dst = ring + sd.ring_off[sp];
    const int rows = sd.D[sp] * n;
    for (int i = tid; i < rows; i += blk) dst[i] = src[i];
  }
  if (comp_shared)
    for (int i = tid; i < kNS * n; i += blk) comp_g[i] = comp_base[i];
  if (err) atomicOr(&s_flags, err << 1);
  if (tid < a.n_analyses) s_samples[tid] = anl[a.analyses[tid].off];
  __syncthreads();
  const int status = pg.status | (dropped ? kSetDropped : 0) | (s_flags >> 1);
  const bool finish = !dropped && chunk >= sd.n_chunks;
  if (finish) {
    for (int ai = 0; ai < a.n_analyses; ++ai) {
      const AnalysisDesc& A = a.analyses[ai];
      if (A.kind == kOscillation)
        for (int c = tid; c < n; c += blk) osc_cell_finalize(anl + A.off, A, c, s_samples[ai]);
    }
  }
  if (tid == 0) {
    SetProgress out = pg;
    out.step = step;
    out.chunk = chunk;
    out.age = age;
    out.status = status;
    out.finalized = finish ? 1 : 0;
    a.prog[set] = out;
  }
}

// Analysis of imported samples (simulation -i): the set's analyses see
// `num_samples` sampled states read from `samples` ([sample][slot][cell],
// the rows of the sampled-state buffer) instead of simulated ones, at the
// ages time_start, time_start + interval, ... (accumulated as DENSE's
// age_by does), then the oscillation analyses are finalized.  One CTA runs
// the one set `set`; a failed concentration check stops it as a drop.
struct ImportVals {
  const double* base;
  int n;
  __device__ __forceinline__ double operator()(int slot, int cell) const { return base[slot * n + cell]; }
};

// (T: the batch's precision; the analyses work in double either way)
template <typename T>
__global__ void dense_import_kernel(const StepArgs a, int set, const double* samples, int num_samples,
                                    double time_start) {
  __shared__ double s_samples[kMaxAnalyses];
  __shared__ int s_flags;
  const SetDesc& sd = a.sets[set];
  const int n = sd.n_cells;
  const int tid = threadIdx.x, blk = blockDim.x;
  double* anl = a.anl + sd.anl_base;
  if (tid < a.n_analyses) s_samples[tid] = anl[a.analyses[tid].off];
  if (tid == 0) s_flags = 0;
  __syncthreads();
  double age = time_start;
  int k = 0;
  bool dropped = false;
  for (; k < num_samples; ++k) {
    const ImportVals vals{samples + static_cast<size_t>(k) * a.n_vals * n, n};
    const bool bad = analyses_sample(a, anl, vals, tid, tid, blk, n, age, s_samples);
    if (bad) atomicOr(&s_flags, 1);
    __syncthreads();
    if (tid < a.n_analyses) s_samples[tid] = anl[a.analyses[tid].off];
    if (s_flags & 1) {
      dropped = true;
      break;
    }
    age += a.interval;
  }
  __syncthreads();
  if (!dropped) {
    for (int ai = 0; ai < a.n_analyses; ++ai) {
      const AnalysisDesc& A = a.analyses[ai];
      if (A.kind == kOscillation)
        for (int c = tid; c < n; c += blk) osc_cell_finalize(anl + A.off, A, c, s_samples[ai]);
    }
  }
  if (tid == 0) {
    SetProgress out = a.prog[set];
    out.chunk = k;
    out.age = age;
    out.status |= dropped ? kSetDropped : 0;
    out.finalized = dropped ? 0 : 1;
    a.prog[set] = out;
  }
}

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
      const int64_t nm = static_cast<int64_t>(nsp) * m;
      const int64_t total = 2 + nm * kOscFields + static_cast<int64_t>(nsp) * (A.range_steps + 1) * m;
      for (int64_t i = threadIdx.x; i < total; i += blockDim.x) {
        double v = 0.0;
        if (i >= 2 + kOscEnd * nm && i < 2 + (kOscCurrent + 1) * nm) v = -1.0;  // end = current = -1
        st[i] = v;
      }
    } else if (A.kind == kTrajectory) {
      if (threadIdx.x < 2) st[threadIdx.x] = 0.0;
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

// Streaming multiprocessors of the current device (looked up once).
inline int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
      n = v;
  }
  return n > 0 ? n : 148;
}

// Launchers, named by the including translation unit's precision suffix.
#define DENSE_B200_STEP_VARIANT(T, KAHAN, THREADS, BLOCKS, UNIFORM, SMEM_CAP)                     \
  {                                                                                             \
    auto k = dense_step_kernel<T, KAHAN, THREADS, BLOCKS, UNIFORM>;                             \
    static bool configured = false;                                                             \
    if (!configured) {                                                                          \
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_CAP); \
      if (e != cudaSuccess) return e;                                                           \
      configured = true;                                                                        \
    }                                                                                           \
    k<<<n_sets, a.block_threads, smem, s>>>(a, set_list);                                       \
    return cudaGetLastError();                                                                  \
  }

#define DENSE_B200_WAVE_VARIANT(T, KAHAN, UNIFORM, THREADS, MINB, SHARED)                       \
  {                                                                                             \
    cudaError_t e = cudaFuncSetAttribute(dense_step_wave_kernel<T, KAHAN, UNIFORM, THREADS, MINB, SHARED>, \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,           \
                                         kWaveSmemBudget);                                       \
    if (e != cudaSuccess) return e;                                                             \
    dense_step_wave_kernel<T, KAHAN, UNIFORM, THREADS, MINB, SHARED><<<n_sets, block, smem, s>>>(a, set_list); \
  }

#define DENSE_B200_DEFINE_LAUNCHERS(SUFFIX, T, KAHAN)                                             \
  namespace dense_b200 {                                                                        \
  cudaError_t launch_init_##SUFFIX(const StepArgs& a, const double* init_conc,                   \
                                   const int* init_status, cudaStream_t s) {                    \
    dense_init_kernel<T><<<a.num_sets, 256, 0, s>>>(a, init_conc, init_status);                  \
    return cudaGetLastError();                                                                  \
  }                                                                                             \
  cudaError_t launch_import_##SUFFIX(const StepArgs& a, int set, const double* samples, int num_samples, \
                                     double time_start, cudaStream_t s) {                       \
    dense_import_kernel<T><<<1, 256, 0, s>>>(a, set, samples, num_samples, time_start);         \
    return cudaGetLastError();                                                                  \
  }                                                                                             \
  cudaError_t launch_step_mem_##SUFFIX(const StepArgs& a, const int* set_list, int n_sets,       \
                                       int block, cudaStream_t s) {                             \
    if (n_sets <= 0) return cudaSuccess;                                                        \
    if (a.uniform_params)                                                                       \
      dense_step_mem_kernel<T, KAHAN, true><<<n_sets, block, 0, s>>>(a, set_list);               \
    else                                                                                        \
      dense_step_mem_kernel<T, KAHAN, false><<<n_sets, block, 0, s>>>(a, set_list);              \
    return cudaGetLastError();                                                                  \
  }                                                                                             \
  cudaError_t launch_step_wave_##SUFFIX(const StepArgs& a, const int* set_list, int n_sets,      \
                                        int block, int smem, int all_shared, cudaStream_t s) {  \
    if (n_sets <= 0) return cudaSuccess;                                                        \
    if (all_shared) {                                                                           \
      if (a.uniform_params) DENSE_B200_WAVE_VARIANT(T, KAHAN, true, 256, 2, true)               \
      else DENSE_B200_WAVE_VARIANT(T, KAHAN, false, 256, 2, true)                               \
    } else if (block == 32 && smem <= 2 * 1024) {                                               \
      if (a.uniform_params) DENSE_B200_WAVE_VARIANT(T, KAHAN, true, 32, 32, false)              \
      else DENSE_B200_WAVE_VARIANT(T, KAHAN, false, 32, 32, false)                              \
    } else {                                                                                    \
      if (a.uniform_params) DENSE_B200_WAVE_VARIANT(T, KAHAN, true, 256, 2, false)              \
      else DENSE_B200_WAVE_VARIANT(T, KAHAN, false, 256, 2, false)                              \
    }                                                                                           \
    return cudaGetLastError();                                                                  \
  }                                                                                             \
  cudaError_t launch_step_##SUFFIX(const StepArgs& a, const int* set_list, int n_sets, size_t smem, \
                                   cudaStream_t s) {                                            \
    if (n_sets <= 0) return cudaSuccess;                                                        \
    /* two 224-thread CTAs per SM (128 registers) when the sets fill more  \
       than one CTA per SM; else one CTA per SM with every register */     \
    if (a.block_threads <= 224 && n_sets > sm_count()) {                                        \
      if (a.uniform_params) DENSE_B200_STEP_VARIANT(T, KAHAN, 224, 2, true, 100000)              \
      else DENSE_B200_STEP_VARIANT(T, KAHAN, 224, 2, false, 100000)                               \
    } else {                                                                                    \
      if (a.uniform_params) DENSE_B200_STEP_VARIANT(T, KAHAN, 256, 1, true, 200000)              \
      else DENSE_B200_STEP_VARIANT(T, KAHAN, 256, 1, false, 200000)                               \
    }                                                                                           \
  }                                                                                             \
  }
