/*
 * dense_b200 -- C ABI of the B200 engine for DENSE's deterministic
 * delay-differential simulation path.
 *
 * One shared library per DENSE model (libdense_b200_<model>.so): the model's
 * specie_list.hpp, reactions_list.hpp, reaction_deltas.hpp and
 * model_impl.hpp are compiled into it, as DENSE compiles one simulator per
 * model (source/CMakeLists.txt:146-188).
 *
 * The entry points replace, for a whole batch of parameter sets at once,
 * what DENSE does per set on the CPU:
 *
 *   dense_engine_create   Simulation / Deterministic_Simulation constructors
 *                         (sim/base.cpp:35-140, sim/determ/determ.cpp:31-52,
 *                         baby_cl.cpp:5-15) and the analysis constructors
 *                         built by parse_analysis_entries
 *                         (parse_analysis_entries.hpp:64-126)
 *   dense_engine_run      run_simulation's chunk loop
 *                         (run_simulation.hpp:127-157): analysis callbacks,
 *                         bad-set drop, age_by -> step (determ.cpp:8-88)
 *   dense_engine_read_*   Deterministic_Simulation::get_concentration
 *                         (determ.hpp:73-79), BasicAnalysis and
 *                         OscillationAnalysis results (basic.ipp:38-75,
 *                         oscillation.ipp:6-77)
 *   dense_engine_status   the Bad_Simulation_Error drop of run_simulation
 *                         (run_simulation.hpp:131-150), as a per-set word
 *
 * Conventions: plain pointers and sizes; the caller owns host buffers, the
 * engine owns device buffers; every function returns a DENSE_* status code
 * (0 = OK) and no exception crosses the ABI; dense_last_error() describes
 * the last failure of the calling thread.  Runs are stream-ordered: only
 * dense_engine_read_* and dense_engine_sync wait for the device.
 */
#ifndef DENSE_B200_H
#define DENSE_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define DENSE_API __attribute__((visibility("default")))
#else
#define DENSE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* return codes */
#define DENSE_OK 0
#define DENSE_ERR_INVALID 1     /* bad argument */
#define DENSE_ERR_CUDA 2        /* CUDA runtime failure */
#define DENSE_ERR_MEMORY 3      /* device allocation failed */
#define DENSE_ERR_UNSUPPORTED 4 /* a batch the engine does not run */
#define DENSE_ERR_SCRATCH_TOO_SMALL 5 /* dense_simulate_noalloc: the batch exceeds its fixed scratch */

/* per-set status bits (dense_engine_status) */
#define DENSE_SET_OK 0
#define DENSE_SET_DROPPED 1        /* a concentration check rejected the set */
#define DENSE_SET_NAN_PARAM 2      /* a rate or delay is NaN (DENSE throws) */
#define DENSE_SET_UNSTAGED_LAG 4   /* a read needed history the staging did not keep */
#define DENSE_SET_BAD_DELAY 8      /* a delay DENSE would read out of bounds with */
#define DENSE_SET_ORDERED_READS 16 /* neighbour reads of rows written in the same step */

/* schedule hint of a set (dense_set_desc.schedule) */
#define DENSE_SCHEDULE_AUTO 0              /* register kernel when the set fits one, else memory kernel */
#define DENSE_SCHEDULE_MEMORY 1            /* memory-state kernel; sets with in-order neighbour reads in
                                              the wave kernel, rows in shared memory as far as they fit */
#define DENSE_SCHEDULE_GLOBAL 2            /* memory-state kernel with every row in global memory */
#define DENSE_SCHEDULE_SHARED_NEIGHBOUR 3  /* as MEMORY, but only neighbour-read species in shared memory */
#define DENSE_SCHEDULE_WAVE_GLOBAL 4       /* as MEMORY, but rows and cell records in global memory: more
                                              sets per SM (single-warp CTAs up to 32 per SM) */
#define DENSE_SCHEDULE_SHARED_ROWS 5       /* a set without in-order neighbour reads in the wave kernel: its
                                              history rows in shared memory as far as they fit, one level
                                              per step */
#define DENSE_SCHEDULE_REGISTER 6          /* register kernel (one thread per cell) */

/* arithmetic of a batch */
#define DENSE_FP64 0        /* matches DENSE's CPU path bit for bit */
#define DENSE_FP32_KAHAN 1  /* FP32 rates, Kahan-compensated FP32 state */

/* analysis kinds */
#define DENSE_ANALYSIS_BASIC 1        /* BasicAnalysis (measurement/basic.hpp) */
#define DENSE_ANALYSIS_OSCILLATION 2  /* OscillationAnalysis (measurement/oscillation.hpp) */
#define DENSE_ANALYSIS_CONCCHECK 3    /* ConcentrationCheck (measurement/conccheck.hpp) */
#define DENSE_ANALYSIS_TRAJECTORY 4   /* csvw_sim data export (io/csvw_sim.ipp) */

typedef struct dense_model_info {
  int num_species;
  int num_reactions;
  int num_delay_reactions;
  int num_critical_species;
  int num_params; /* rates | delays | critical values (core/parameter_set.hpp:9-13) */
} dense_model_info;

/* One parameter set (one DENSE Simulation). */
typedef struct dense_set_desc {
  int num_cells;              /* <= 65536 */
  const int* nbr_offsets;     /* [num_cells + 1] CSR row offsets */
  const int* nbr_ids;         /* neighbour cell ids, ascending per cell (std::set order) */
  const double* set_params;   /* [num_params]: the Parameter_Set; ring sizes derive from it */
  const double* cell_params;  /* [num_cells][num_params] per-cell parameters, or NULL:
                                 every cell uses set_params */
  const double* init_conc;    /* [num_species] initial value of every history row, or NULL (zeros) */
  const double* perturb;      /* [num_reactions] -b factors entering the ring sizes, or NULL */
  double duration;            /* simulated minutes (-t) */
  /* Schedule hints, 0 = the engine's choice (results do not depend on them;
     dense_b200.autotune picks them by timing): */
  int schedule;               /* DENSE_SCHEDULE_MEMORY: run the set in the memory-state kernel */
  int mem_block;              /* memory-state kernel threads per CTA: 32..256, a multiple of 32 */
} dense_set_desc;

/* One analysis, applied to every set (an <anlys> entry of analyses.xml). */
typedef struct dense_analysis_desc {
  int kind;                   /* DENSE_ANALYSIS_* */
  int num_species;            /* observed species; CONCCHECK: 0 = all species */
  const int* species;         /* [num_species] species ids */
  int cell_start, cell_end;   /* [cell_start, cell_end) */
  double time_start, time_end;/* [time_start, time_end) */
  double win_range;           /* OSCILLATION: <win-range> */
  double anlys_intvl;         /* OSCILLATION: <anlys-intvl> */
  double lower, upper;        /* CONCCHECK bounds */
} dense_analysis_desc;

typedef struct dense_run_desc {
  int precision;              /* DENSE_FP64 or DENSE_FP32_KAHAN */
  double step_size;           /* dt in minutes (-s) */
  double analysis_interval;   /* minutes between analysis samples (-u) */
  int num_analyses;
  const dense_analysis_desc* analyses;
  int device;                 /* CUDA device ordinal */
} dense_run_desc;

typedef struct dense_engine dense_engine;

/* The compiled model's counts: NUM_SPECIES (core/specie.hpp:25),
   NUM_REACTIONS (core/reaction.hpp:19), NUM_DELAY_REACTIONS
   (core/reaction.hpp:29-36), NUM_CRITICAL_SPECIES (core/specie.hpp:28-35),
   NUM_PARAMS (core/parameter_set.hpp:10). */
DENSE_API int dense_model_get_info(dense_model_info* out);
/* specie_str[species] (core/specie.hpp:19) and reaction_str[reaction]
   (core/reaction.hpp:23); NULL out of range. */
DENSE_API const char* dense_model_specie_name(int species);
DENSE_API const char* dense_model_reaction_name(int reaction);
/* Reaction name of delay reaction d (reactions_list.hpp order of the
   DELAY_REACTION entries), and species name of critical species c
   (specie_list.hpp order of the CRITICAL_SPECIE entries); NULL out of range. */
DENSE_API const char* dense_model_delay_reaction_name(int d);
DENSE_API const char* dense_model_critical_specie_name(int c);
/* Text of the last failure on this thread (what DENSE's exceptions carry
   in what()). */
DENSE_API const char* dense_last_error(void);

/* Validate and stage a batch on the device (host buffers are copied).
   Replaces Sim_Builder::get_simulations and the Deterministic_Simulation
   constructor per set (deterministic_main.cpp:53, sim/determ/determ.cpp:31-52)
   and the analyses parse_analysis_entries builds (deterministic_main.cpp:54). */
DENSE_API int dense_engine_create(const dense_run_desc* run, int num_sets, const dense_set_desc* sets,
                        dense_engine** out);

/* Run the next `num_chunks` analysis chunks of every set (-1: to the end of
   each set's horizon), on `stream` (a cudaStream_t, or NULL for the
   engine's own stream).  Sets finishing their horizon are finalized.
   Replaces run_simulation's chunk loop (run_simulation.hpp:84-165) over
   Deterministic_Simulation::age_by (sim/determ/determ.cpp:9-21). */
DENSE_API int dense_engine_run(dense_engine* e, int num_chunks, void* stream);

/* Same, replayed from a CUDA graph captured on first use for this chunk
   count (no counterpart in DENSE). */
DENSE_API int dense_engine_run_graph(dense_engine* e, int num_chunks, void* stream);

/* Wait for the engine's stream (no counterpart in DENSE, which is
   synchronous). */
DENSE_API int dense_engine_sync(dense_engine* e);

/* Reset every set to its initial state (same inputs; no reallocation; in
   DENSE a new Simulation object). */
DENSE_API int dense_engine_reset(dense_engine* e, void* stream);

/* Analysis of an imported trajectory, what DENSE's [-i | --data-import]
   flag was meant to do (main.cpp:160-175 with CSV_Streamed_Simulation,
   io/csvr_sim.cpp:7-96, which never worked: its age_by calls itself): the
   set's analyses, as created, see `num_samples` sampled states taken from
   `samples` ([num_samples][num_species][num_cells]; species no analysis
   observes are not read) instead of simulated ones, at the ages
   time_start, time_start + analysis_interval, ... (each the previous plus
   the interval, as age_by accumulates them), and the oscillation analyses
   are then finalized; the results are read as after a run.  Call it on an
   engine fresh from dense_engine_create or dense_engine_reset; it returns
   when the analyses are done. */
DENSE_API int dense_engine_analyze_samples(dense_engine* e, int set, const double* samples, int num_samples,
                                           double time_start);

/* Checkpoint and resume (no counterpart in DENSE, whose only record of a
   run is its trajectory export).  A batch's whole mutable run state --
   per-set progress and status, lag-0 state (and FP32 Kahan terms),
   history rings and analysis state -- is copied into a caller buffer of
   dense_engine_checkpoint_size bytes (a header that identifies the batch's
   layout, then the four device blocks), after the engine's work so far
   has finished.  dense_engine_restore puts such a snapshot back into an
   engine created from the same inputs (the same sets, analyses, step
   size, interval and precision, in this process or another one), which
   then continues exactly where the checkpointed engine was: the rest of
   the run gives the same results bit for bit as an uninterrupted one.  A
   buffer too small, or a snapshot of a batch with another layout, returns
   DENSE_ERR_INVALID and leaves the engine unchanged. */
DENSE_API int dense_engine_checkpoint_size(dense_engine* e, int64_t* bytes);
DENSE_API int dense_engine_checkpoint(dense_engine* e, void* buf, int64_t bytes);
DENSE_API int dense_engine_restore(dense_engine* e, const void* buf, int64_t bytes);

/* Per-set status words (DENSE_SET_* bits), [num_sets]: the drop that
   run_simulation makes when an analysis throws Bad_Simulation_Error
   (run_simulation.hpp:131-150, measurement/conccheck.hpp:48), as a word. */
DENSE_API int dense_engine_status(dense_engine* e, int32_t* out);

/* Chunks done and simulated age per set, [num_sets] each
   (Simulation::age, sim/base.hpp:124). */
DENSE_API int dense_engine_progress(dense_engine* e, int32_t* chunks, double* age);

/* Lag-0 concentrations of one set, [num_species][num_cells]:
   Deterministic_Simulation::get_concentration(cell, species)
   (sim/determ/determ.hpp:73-75) for every cell and species. */
DENSE_API int dense_engine_read_state(dense_engine* e, int set, double* out);

/* BasicAnalysis `analysis` of one set: mins/sums/maxs [n], per-cell
   [cells][n] (any may be NULL), samples and time.  sums are the raw sums
   DENSE keeps in `means` (basic.ipp:22-36); show() divides by
   samples * cells. */
DENSE_API int dense_engine_read_basic(dense_engine* e, int analysis, int set, double* mins, double* sums,
                            double* maxs, double* cell_mins, double* cell_sums, double* cell_maxs,
                            int* samples, double* time);

/* OscillationAnalysis `analysis` of one set, [n][cells] each: average
   amplitude, average period, mean peak ("avg peak" of show()), number of
   critical points; plus samples and time.  Valid once the set finished. */
DENSE_API int dense_engine_read_oscillation(dense_engine* e, int analysis, int set, double* amps,
                                  double* periods, double* avg_peaks, int* num_crit, int* samples,
                                  double* time);

/* Trajectory analysis `analysis` of one set: sample times [capacity] and
   values [capacity][n][cells] of the observed species at every sample, as
   csvw_sim::update writes them (io/csvw_sim.ipp:17-91); *samples is the
   number recorded. */
DENSE_API int dense_engine_read_trajectory(dense_engine* e, int analysis, int set, double* times, double* values,
                                           int capacity, int* samples);

/* Batched reads (no counterpart in DENSE, which reads one simulation at a
   time): every set's Oscillation amplitudes and periods, [sets][species]
   [cells] (either pointer may be NULL); every set's recorded Trajectory
   values, [sets][capacity][species][cells], into device memory (on_device)
   or host memory, with each set's sample count (samples[sets], or NULL),
   ordered on `stream`; the capacity (samples room per set). */
DENSE_API int dense_engine_read_oscillation_all(dense_engine* e, int analysis, double* amps, double* periods);
DENSE_API int dense_engine_copy_trajectory(dense_engine* e, int analysis, void* dst, int on_device, int* samples,
                                           void* stream);
DENSE_API int dense_engine_trajectory_capacity(dense_engine* e, int analysis, int* capacity);

/* Batch facts: cell-steps per full run, device bytes held, threads per
   CTA of the register kernel (no counterpart in DENSE). */
DENSE_API int dense_engine_info(dense_engine* e, int64_t* total_cell_steps, int64_t* device_bytes,
                      int* max_block_threads);

/* Staged history depth (D) and DENSE ring size (S) per species of a set;
   S is baby_cl's per-species row count (sim/determ/baby_cl.cpp:10). */
DENSE_API int dense_engine_ring_info(dense_engine* e, int set, int* S, int* D);

/* Free the batch's device buffers (the simulations' destruction at the end
   of run_simulation). */
DENSE_API int dense_engine_destroy(dense_engine* e);

/* One CUDA graph over several batches, possibly of different models (no
   counterpart in DENSE, which runs one model per process): run_fns[i] is
   the dense_engine_run of engines[i]'s model library; every engine advances
   num_chunks chunks on a branch of its own, kernels keep their stream
   priorities.  Run each engine once (e.g. num_chunks 0) before capturing.
   Launch with dense_graph_launch, free with dense_graph_destroy. */
DENSE_API int dense_graph_capture(int num_engines, void* const* run_fns, dense_engine* const* engines,
                                  int num_chunks, int device, void** graph_exec);
DENSE_API int dense_graph_launch(void* graph_exec, void* stream);
DENSE_API int dense_graph_destroy(void* graph_exec);

/* Planning without a GPU (no counterpart in DENSE, whose Simulation objects
   size themselves, sim/base.cpp:55-140): per set, the device bytes
   dense_engine_create would hold for it (set_bytes, or NULL) and the kernel
   it would run in (set_kernel: 0 = register kernel, else the memory-state
   kernel's threads per CTA; or NULL) and the dependency levels of one of
   its steps (set_levels: 1 unless neighbour reads see rows written in the
   same step, DENSE's in-order cell loop; or NULL).  Used to size waves and
   to bucket sets for schedule tuning. */
DENSE_API int dense_engine_plan(const dense_run_desc* run, int num_sets, const dense_set_desc* sets,
                                int64_t* set_bytes, int* set_kernel, int* set_levels);

/* No counterpart in DENSE: an addition of this library for callers that may
   not allocate device memory -- code running inside a framework that owns
   the GPU's whole memory through its own pool, or a service loop that must
   not call cudaMalloc after start-up because it can synchronize the device.

   Runs an FP64 batch without analyses from host inputs to the final lag-0
   state (final_state: the sets' [num_species][num_cells] blocks one after
   another; status: [num_sets] DENSE_SET_* words, or NULL) and returns when
   the results are on the host.  It allocates nothing: every device buffer
   lives in one fixed 16 MiB array inside this library, which every GPU that
   loads the library holds until the process exits.  Limits: at most 64 sets
   of at most 256 cells, and the batch's descriptors, parameters, neighbour
   lists, state and history rings must fit in 16 MiB; a larger batch returns
   DENSE_ERR_SCRATCH_TOO_SMALL.  precision must be DENSE_FP64 and
   num_analyses 0, and no set may have neighbour reads of the row written in
   the same step (DENSE's in-order cell loop, e.g. Turing-Pattern): those
   need the memory or wave kernel of dense_engine_create, and such a batch
   returns DENSE_ERR_UNSUPPORTED before the device is touched.
   Every call looks up the array's device address on run->device (a lookup
   that allocates nothing); the first call on a device may load this
   library's device code there, so make it before any stream capture on the
   device.  The call makes run->device current while it works and restores
   the caller's current device before it returns.  All calls share the
   array: calls that overlap on the GPU (two host threads, or two streams
   not ordered against each other) race and must not be made.  Every region
   a call reads is written by the same call first, so the array's previous
   contents never leak into results. */
DENSE_API int dense_simulate_noalloc(const dense_run_desc* run, int num_sets, const dense_set_desc* sets,
                                     double* final_state, int32_t* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DENSE_B200_H */
