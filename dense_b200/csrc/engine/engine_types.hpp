// Device-side descriptors shared by the step kernels and the host engine.
// Compiled once per DENSE model (NUM_SPECIES etc. come from the model's
// headers through dense_model_api.hpp).
#ifndef DENSE_B200_ENGINE_TYPES_HPP
#define DENSE_B200_ENGINE_TYPES_HPP

#include <vector_types.h>

#include <cstdint>

#include "dense_model_api.hpp"

namespace dense_b200 {

constexpr int kNS = NUM_SPECIES;
constexpr int kNR = NUM_REACTIONS;
constexpr int kND = NUM_DELAY_REACTIONS;
constexpr int kNP = NUM_PARAMS;
constexpr int kMaxAnalyses = 8;
constexpr int kStepThreads = 256;  // register kernel: one thread per cell, one CTA per set
constexpr int kMaxCells = 65536;   // memory kernel: cells per set

// Per-set status bits (also the public DENSE_SET_* values).
enum : int {
  kSetDropped = 1,       // a concentration check rejected the set
  kSetNanParam = 2,      // a rate or delay parameter is NaN
  kSetUnstagedLag = 4,   // a read hit a lag the history staging did not keep
  kSetBadDelay = 8,      // a delay DENSE would turn into an out-of-bounds read
  kSetOrderedReads = 16, // neighbour reads of rows written in the same step
  kSetNotRunnable = kSetNanParam | kSetOrderedReads,
};

enum AnalysisKind : int { kBasic = 1, kOscillation = 2, kConcCheck = 3, kTrajectory = 4 };

// One analysis, identical for every set of the batch.
struct AnalysisDesc {
  int kind;
  int nsp;              // observed species count (ConcCheck: 1, or NS for all)
  int sp[kNS];          // observed species ids, in observation order
  int slot[kNS];        // row of each observed species in the kernel's sampled-state buffer
  int cmin, cmax;       // cell range [cmin, cmax)
  double t0, t1;        // time range [t0, t1)
  int range_steps;      // oscillation window (range / anlys-intvl, truncated)
  double interval;      // oscillation anlys-intvl
  double lo, hi;        // concentration check bounds
  int64_t off;          // offset of this analysis' state inside a set's block
};

// Layout of one analysis' per-set state (doubles), relative to
// AnalysisDesc::off.  n = nsp, m = cmax - cmin, w = range_steps + 1.
//  Basic:       mins[n] maxs[n] sums[n] samples time | cmins[n][m] cmaxs[n][m] csums[n][m]
//  Oscillation: samples time | field[kOscFields][n][m] | window[n][w][m]
//  ConcCheck:   time
//  Trajectory:  samples time | sample_time[cap] | values[cap][n][m]  (cap = range_steps)
enum OscField : int {
  kOscStart, kOscEnd, kOscCurrent,  // queue indices (core/queue.hpp)
  kOscLive,                         // values in the window
  kOscLastTime, kOscLastConc, kOscLastPeak, kOscNcrit,
  kOscTm2, kOscTm1,                 // times of critical points ncrit-3 and ncrit-2
  kOscPeakSum, kOscTroughSum, kOscNumPeaks, kOscNumTroughs, kOscCycleSum, kOscCycles,
  kOscAmp, kOscPer, kOscAvgPeak,    // results, written by finalize
  kOscSame,                         // length of the run of equal values that ends at the newest one
  kOscFields
};

// One parameter set of the batch.
struct SetDesc {
  int n_cells;
  int n_chunks;          // analysis chunks of this set's horizon
  int steps_per_chunk;   // (int)(interval / dt)
  int param_stride;      // 0: one parameter row for every cell; n_cells: [NP][n] per cell
  int64_t param_base;    // first double of this set's parameters
  int64_t cell_base;     // first cell of this set in the per-cell arrays
  int64_t nbr_base;      // offset of this set's CSR row offsets (n_cells + 1)
  int64_t ring_base;     // first element of this set's history block
  int64_t anl_base;      // first double of this set's analysis block
  int S[kNS];            // DENSE ring size per species (baby_cl.cpp:10)
  int D[kNS];            // staged history depth, a power of two (0: lag-0 only, kept in registers)
  int64_t ring_off[kNS]; // offset of each staged ring inside the set's block
  int64_t lvl_base;      // memory kernel: offset of this set's level offsets (n_levels + 1)
  int n_levels;          // memory kernel: cell-dependency levels per step
  int ordered;           // neighbour reads of the row written in the same step (DENSE's cell order)
  // wave kernel (ordered sets): rows indexed modulo D (not a power of two),
  // cells as 16-byte records {cell, neighbour count, up to 6 neighbour ids}
  // in level order
  int wave;
  int smem_off[kNS];     // byte offset of the species' rows in shared memory, -1: global
  int lvl_smem_off;      // byte offset of the 16-bit level offsets in shared memory
  int topo_off;          // byte offset of the records in shared memory, -1: global
  int comp_smem_off;     // FP32: byte offset of the Kahan terms [kNS][n] in shared memory, -1: global
  int smem_bytes;        // dynamic shared memory the set needs
  int64_t rec_base;      // first record of the set in StepArgs::wave_rec
  // time pipelining: step k + 1 runs wave_delta levels behind step k, so
  // wave_fronts consecutive steps are in flight, one thread group each
  int wave_delta;
  int wave_fronts;
};

// Dynamic shared memory a wave-kernel CTA may use (the 227 KB opt-in limit
// of sm_100 less room for the kernel's static shared memory), and the
// neighbours a wave-kernel cell record holds.
constexpr int kWaveSmemBudget = 227 * 1024 - 8 * 1024;
constexpr int kWaveMaxNbrs = 6;
constexpr int kWaveMaxFronts = 4;   // steps in flight in the wave kernel

// Mutable per-set progress, updated by the kernels.
struct SetProgress {
  int64_t step;   // Euler steps done
  int chunk;      // chunks done
  int status;     // kSet* bits
  double age;     // simulated minutes (DENSE Simulation::age_)
  int finalized;
  int pad;
};

struct StepArgs {
  const SetDesc* sets;
  SetProgress* prog;
  const void* params;       // per set, in the batch's precision: [NP] (param_stride 0) or [NP][n_cells]
  const int* nbr_off;       // per set: n_cells + 1 absolute offsets into nbr_idx
  const int* nbr_idx;       // neighbour cell ids, local to the set, ascending
  void* state;              // per set: [NS][n_cells] lag-0 state (T), then [NS][n_cells] Kahan terms
  void* ring;               // history rings (T)
  double* anl;              // analysis state
  AnalysisDesc analyses[kMaxAnalyses];
  int n_analyses;
  int num_sets;
  double dt;
  double interval;
  int chunk_count;          // chunks to run in this launch (-1: to the end)
  int block_threads;
  int csr_in_smem;          // copy each set's neighbour ids into shared memory
  int uniform_params;       // every set has one parameter row for all its cells
  const int* lvl_off;       // memory kernel: per set, first index of each level in lvl_cells
  const int* lvl_cells;     // memory kernel: per set, its cells in level order
  const uint4* wave_rec;    // wave kernel: per set, [n_cells] cell records in level order
  int n_vals;               // species the analyses observe (rows of the sampled-state buffer)
  int val_slot[kNS];        // row of each species in that buffer, -1 when no analysis observes it
};

}  // namespace dense_b200

#endif
