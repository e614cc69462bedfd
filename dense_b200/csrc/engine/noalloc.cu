// dense_simulate_noalloc: the FP64 engine for callers that cannot allocate
// device memory.
//
// Some callers of this library are not allowed to call cudaMalloc: a host
// framework that owns all of the GPU's memory through its own pool (and
// would see a foreign allocation as an out-of-memory fault or as
// fragmentation), or a latency-bound service loop that must not allocate
// after start-up because cudaMalloc may synchronize the whole device.  This
// entry point serves them: it runs a small FP64 batch with no analyses and
// returns the final state, using only the fixed scratch array below for
// every device-side buffer (set descriptors, parameters, neighbour lists,
// state, history rings).  It calls no cudaMalloc, cudaFree or other
// allocating routine.
//
// The array is a file-scope __device__ variable of kScratchBytes (16 MiB);
// every GPU that loads this library keeps it until the process exits.  In
// host code the name g_noalloc_scratch is only a stand-in for the device
// symbol, never a usable address, so every call (with the run's device
// current) asks the runtime for the real address with cudaGetSymbolAddress,
// which allocates nothing; asking on every call rather than caching keeps
// the address right if the device's context is ever re-created.  The first
// call on a device may load this library's device code there, so it should
// come before any stream capture on the device.
//
// The call makes run->device current while it works and makes the caller's
// current device current again before it returns.
//
// It runs sets in the register kernel only.  A set whose neighbour reads
// see the row written in the same step (DENSE's in-order cell loop, as in
// Turing-Pattern) needs the memory or wave kernel and is refused with
// DENSE_ERR_UNSUPPORTED before the device is touched.
//
// All calls share the one array and it keeps the previous call's contents.
// Everything the kernels read is written by the call itself before the
// kernels run (descriptors, parameters, neighbour lists; the init kernel
// writes state, history rows and progress), so nothing has to start at
// zero.  Calls that overlap on the GPU -- from two host threads, or on two
// streams without ordering between them -- race on the array and must not
// be issued.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "dense_model_api.hpp"
#include "reaction_deltas.hpp"
#include "model_impl.hpp"

#include "dense_b200.h"
#include "engine_launch.hpp"
#include "engine_types.hpp"
#include "lag_trace.hpp"

using namespace dense_b200;

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;
constexpr int kMaxNoallocSets = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Failures are reported by return code only (the message names the case
// for readers of this file).
int nfail(int code, const char*) { return code; }

// Device address of the scratch array on the current device.
int scratch_address(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) return nfail(DENSE_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
  *out = static_cast<unsigned char*>(p);
  return DENSE_OK;
}

// Makes the caller's current device current again when the call returns.
struct DeviceRestore {
  int prev = -1;
  DeviceRestore() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceRestore() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceRestore(const DeviceRestore&) = delete;
  DeviceRestore& operator=(const DeviceRestore&) = delete;
};

// Writes the [NP][n] parameter layout of one set from its raw rows.
__global__ void noalloc_param_layout(double* dst, const double* src, int n, int per_cell) {
  const int total = NUM_PARAMS * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int p = i / n, c = i % n;
    dst[i] = per_cell ? src[static_cast<size_t>(c) * NUM_PARAMS + p] : src[p];
  }
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" DENSE_API int dense_simulate_noalloc(const dense_run_desc* run, int num_sets, const dense_set_desc* sets,
                                                double* final_state, int32_t* status, void* stream) {
  if (!run || !sets || !final_state || num_sets <= 0) return nfail(DENSE_ERR_INVALID, "null argument or no sets");
  if (num_sets > kMaxNoallocSets) return nfail(DENSE_ERR_SCRATCH_TOO_SMALL, "more than 64 sets");
  if (run->precision != DENSE_FP64 || run->num_analyses != 0)
    return nfail(DENSE_ERR_UNSUPPORTED, "the no-allocation entry point runs FP64 batches without analyses");
  if (!(run->step_size > 0.0) || !(run->analysis_interval > 0.0))
    return nfail(DENSE_ERR_INVALID, "step size and analysis interval must be positive");
  const double dt = run->step_size, interval = run->analysis_interval;
  const double steps_d = interval / dt;
  if (!(steps_d < 2147483647.0)) return nfail(DENSE_ERR_INVALID, "interval / step size too large");
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  // ---- plan every set on the host (stack memory only)
  SetDesc desc[kMaxNoallocSets];
  double init_conc[kMaxNoallocSets][NUM_SPECIES];
  int init_status[kMaxNoallocSets];
  int64_t cells_total = 0, ring_total = 0, edges_total = 0;
  int max_cells = 0;
  for (int si = 0; si < num_sets; ++si) {
    const dense_set_desc& in = sets[si];
    if (in.num_cells <= 0 || in.num_cells > 256 || !in.nbr_offsets || !in.nbr_ids || !in.set_params ||
        !(in.duration >= 0.0))
      return nfail(DENSE_ERR_INVALID, "bad set (1..256 cells, CSR and parameters required)");
    const int n = in.num_cells;
    if (in.nbr_offsets[0] != 0) return nfail(DENSE_ERR_INVALID, "CSR offsets must start at 0");
    for (int c = 0; c < n; ++c)
      if (in.nbr_offsets[c + 1] < in.nbr_offsets[c]) return nfail(DENSE_ERR_INVALID, "CSR offsets decrease");
    for (int c = 0; c < n; ++c)
      for (int k = in.nbr_offsets[c]; k < in.nbr_offsets[c + 1]; ++k)
        if (in.nbr_ids[k] < 0 || in.nbr_ids[k] >= n || (k > in.nbr_offsets[c] && in.nbr_ids[k - 1] >= in.nbr_ids[k]))
          return nfail(DENSE_ERR_INVALID, "neighbour ids must be ascending cell ids of the tissue");
    SetDesc& d = desc[si];
    std::memset(&d, 0, sizeof(d));
    d.n_cells = n;
    if (!ring_sizes(in, dt, d.S)) return nfail(DENSE_ERR_INVALID, "ring size is not a positive int");
    int status0 = 0;
    const int traced = in.cell_params ? n : 1;
    const double* prm0 = in.cell_params ? in.cell_params : in.set_params;
    for (int c = 0; c < traced; ++c)
      for (int i = 0; i < NUM_REACTIONS + NUM_DELAY_REACTIONS; ++i)
        if (std::isnan(prm0[static_cast<size_t>(c) * NUM_PARAMS + i])) status0 |= kSetNanParam;
    // the same tracing as dense_engine_create, so the rings have the same depths
    LagTrace tr;
    trace_lags(prm0, traced, NUM_PARAMS, 1, d.S, tr);
    if (tr.ordered)
      return nfail(DENSE_ERR_UNSUPPORTED,
                   "neighbour reads of the row written in the same step need the memory or wave kernel");
    if (tr.bad) status0 |= kSetBadDelay;
    const int* own_max = tr.own_max;
    const int* nbr_max = tr.nbr_max;
    int64_t off = 0;
    for (int sp = 0; sp < NUM_SPECIES; ++sp) {
      int depth = 0;
      if (own_max[sp] >= 1) depth = own_max[sp] + 1;
      if (nbr_max[sp] >= 0 && nbr_max[sp] + 2 > depth) depth = nbr_max[sp] + 2;
      int pow2 = depth > 0 ? 1 : 0;
      while (pow2 < depth) pow2 <<= 1;
      depth = pow2;
      d.D[sp] = depth;
      d.ring_off[sp] = off;
      off += static_cast<int64_t>(depth) * n;
    }
    const double chunks = in.duration / interval;
    if (!(chunks < 2147483647.0)) return nfail(DENSE_ERR_INVALID, "too many chunks");
    d.n_chunks = static_cast<int>(std::ceil(chunks));
    d.steps_per_chunk = static_cast<int>(steps_d);
    d.cell_base = cells_total;
    d.param_base = cells_total * NUM_PARAMS;  // [NP][n] per set
    d.param_stride = n;
    d.nbr_base = cells_total + si;  // offsets region: n + 1 entries per set
    d.ring_base = ring_total;
    d.anl_base = 0;
    for (int sp = 0; sp < NUM_SPECIES; ++sp) init_conc[si][sp] = in.init_conc ? in.init_conc[sp] : 0.0;
    init_status[si] = status0;
    cells_total += n;
    edges_total += in.nbr_offsets[n];
    ring_total = (ring_total + off + 31) & ~int64_t(31);
    if (n > max_cells) max_cells = n;
  }

  // ---- carve the scratch array
  size_t o = 0;
  const size_t o_sets = o;     o = align256(o + sizeof(SetDesc) * num_sets);
  const size_t o_prog = o;     o = align256(o + sizeof(SetProgress) * num_sets);
  const size_t o_params = o;   o = align256(o + sizeof(double) * NUM_PARAMS * cells_total);
  const size_t o_raw = o;      o = align256(o + sizeof(double) * NUM_PARAMS * 256);
  const size_t o_off = o;      o = align256(o + sizeof(int) * (cells_total + num_sets));
  const size_t o_idx = o;      o = align256(o + sizeof(int) * (edges_total > 0 ? edges_total : 1));
  const size_t o_state = o;    o = align256(o + sizeof(double) * 2 * NUM_SPECIES * cells_total);
  const size_t o_ring = o;     o = align256(o + sizeof(double) * (ring_total > 0 ? ring_total : 1));
  const size_t o_conc = o;     o = align256(o + sizeof(double) * NUM_SPECIES * num_sets);
  const size_t o_status = o;   o = align256(o + sizeof(int) * num_sets);
  const size_t o_list = o;     o = align256(o + sizeof(int) * num_sets);
  if (o > kScratchBytes)
    return nfail(DENSE_ERR_SCRATCH_TOO_SMALL, "batch needs more than the 16 MiB scratch array");
  // every check above runs on the host; the device is touched from here on
  DeviceRestore restore_;
  if (cudaSetDevice(run->device) != cudaSuccess) return nfail(DENSE_ERR_CUDA, "cudaSetDevice failed");
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc != DENSE_OK) return rc;

#define NA_TRY(x) do { if ((x) != cudaSuccess) return nfail(DENSE_ERR_CUDA, #x " failed"); } while (0)
  NA_TRY(cudaMemcpyAsync(base + o_sets, desc, sizeof(SetDesc) * num_sets, cudaMemcpyHostToDevice, s));
  NA_TRY(cudaMemcpyAsync(base + o_conc, init_conc, sizeof(double) * NUM_SPECIES * num_sets, cudaMemcpyHostToDevice, s));
  NA_TRY(cudaMemcpyAsync(base + o_status, init_status, sizeof(int) * num_sets, cudaMemcpyHostToDevice, s));
  int list[kMaxNoallocSets];
  for (int si = 0; si < num_sets; ++si) list[si] = si;
  NA_TRY(cudaMemcpyAsync(base + o_list, list, sizeof(int) * num_sets, cudaMemcpyHostToDevice, s));
  int64_t edge_base = 0;
  for (int si = 0; si < num_sets; ++si) {
    const dense_set_desc& in = sets[si];
    const int n = in.num_cells;
    int offs[257];
    for (int c = 0; c <= n; ++c) offs[c] = static_cast<int>(edge_base + in.nbr_offsets[c]);
    NA_TRY(cudaMemcpyAsync(base + o_off + sizeof(int) * desc[si].nbr_base, offs, sizeof(int) * (n + 1),
                           cudaMemcpyHostToDevice, s));
    if (in.nbr_offsets[n] > 0)
      NA_TRY(cudaMemcpyAsync(base + o_idx + sizeof(int) * edge_base, in.nbr_ids, sizeof(int) * in.nbr_offsets[n],
                             cudaMemcpyHostToDevice, s));
    edge_base += in.nbr_offsets[n];
    // raw parameter rows -> [NP][n] layout (the staging area is reused per set)
    const size_t raw = in.cell_params ? sizeof(double) * NUM_PARAMS * n : sizeof(double) * NUM_PARAMS;
    NA_TRY(cudaMemcpyAsync(base + o_raw, in.cell_params ? in.cell_params : in.set_params, raw,
                           cudaMemcpyHostToDevice, s));
    noalloc_param_layout<<<8, 256, 0, s>>>(reinterpret_cast<double*>(base + o_params) + desc[si].cell_base * NUM_PARAMS,
                                           reinterpret_cast<const double*>(base + o_raw), n, in.cell_params ? 1 : 0);
    NA_TRY(cudaGetLastError());
  }

  StepArgs a{};
  a.sets = reinterpret_cast<const SetDesc*>(base + o_sets);
  a.prog = reinterpret_cast<SetProgress*>(base + o_prog);
  a.params = base + o_params;
  a.nbr_off = reinterpret_cast<const int*>(base + o_off);
  a.nbr_idx = reinterpret_cast<const int*>(base + o_idx);
  a.state = base + o_state;
  a.ring = base + o_ring;
  a.anl = reinterpret_cast<double*>(base + o_state);  // unused: no analyses
  a.n_analyses = 0;
  a.num_sets = num_sets;
  a.dt = dt;
  a.interval = interval;
  a.chunk_count = -1;
  a.block_threads = max_cells < 32 ? 32 : (max_cells + 31) / 32 * 32;
  NA_TRY(launch_init_fp64(a, reinterpret_cast<const double*>(base + o_conc),
                          reinterpret_cast<const int*>(base + o_status), s));
  a.csr_in_smem = 0;
  a.uniform_params = 0;  // parameters are laid out per cell here
  NA_TRY(launch_step_fp64(a, reinterpret_cast<const int*>(base + o_list), num_sets,
                          sizeof(int) * NUM_DELAY_REACTIONS * a.block_threads, s));

  // ---- results to the caller's buffers
  size_t out_off = 0;
  for (int si = 0; si < num_sets; ++si) {
    const size_t cnt = static_cast<size_t>(NUM_SPECIES) * desc[si].n_cells;
    NA_TRY(cudaMemcpyAsync(final_state + out_off,
                           reinterpret_cast<double*>(base + o_state) + desc[si].cell_base * 2 * NUM_SPECIES,
                           sizeof(double) * cnt, cudaMemcpyDeviceToHost, s));
    out_off += cnt;
  }
  if (status) {
    SetProgress prog[kMaxNoallocSets];
    NA_TRY(cudaMemcpyAsync(prog, base + o_prog, sizeof(SetProgress) * num_sets, cudaMemcpyDeviceToHost, s));
    NA_TRY(cudaStreamSynchronize(s));
    for (int si = 0; si < num_sets; ++si) status[si] = prog[si].status;
  } else {
    NA_TRY(cudaStreamSynchronize(s));
  }
#undef NA_TRY
  return DENSE_OK;
}
