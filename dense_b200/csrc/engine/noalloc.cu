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
// symbol, never a usable address, so the first call on each device (with
// that device current) asks the runtime for the real address with
// cudaGetSymbolAddress and keeps it.  That first call should therefore come
// before any stream capture on the device.
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
#include <mutex>
#include <string>

#include "dense_model_api.hpp"
#include "reaction_deltas.hpp"
#include "model_impl.hpp"

#include "dense_b200.h"
#include "engine_launch.hpp"
#include "engine_types.hpp"

using namespace dense_b200;

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;
constexpr int kMaxNoallocSets = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Failures are reported by return code only (the message names the case
// for readers of this file).
int nfail(int code, const char*) { return code; }

// Device address of the scratch array on the current device (set-up on
// first use per device).
int scratch_address(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return nfail(DENSE_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return nfail(DENSE_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    g_scratch_ptr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_ptr[device]);
  return DENSE_OK;
}

struct Dep {
  bool* deps;
  double getCon(specie_id sp, int = 0) const { deps[sp] = true; return 0.0; }
  double calculateNeighborAvg(specie_id sp, int = 0) const { deps[sp] = true; return 0.0; }
  double getRate(reaction_id) const { return 0.0; }
  double getDelay(delay_reaction_id) const { return 0.0; }
  double getCritVal(critspecie_id) const { return 0.0; }
};

struct Lags {
  const double* prm;
  const int* S;
  int* own_max;
  int* nbr_max;
  bool* ordered;
  double getCon(specie_id) const { return 0.0; }
  double getCon(specie_id sp, int k) const {
    const int s = S[sp];
    const int lag = (((k - 1) % s) + s) % s;
    if (lag > own_max[sp]) own_max[sp] = lag;
    return 0.0;
  }
  double calculateNeighborAvg(specie_id sp, int k = 0) const {
    const int s = S[sp];
    const int lag = ((k % s) + s) % s;
    if (lag == s - 1 && s > 1) *ordered = true;
    if (lag > nbr_max[sp]) nbr_max[sp] = lag;
    return 0.0;
  }
  double getRate(reaction_id r) const { return prm[r]; }
  double getDelay(delay_reaction_id d) const { return prm[NUM_REACTIONS + d]; }
  double getCritVal(critspecie_id c) const { return prm[NUM_REACTIONS + NUM_DELAY_REACTIONS + c]; }
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
    bool deps[NUM_REACTIONS][NUM_SPECIES] = {};
#define REACTION(name) { Dep c{deps[name]}; reaction<name>::active_rate(c); }
#include "reactions_list.hpp"
#undef REACTION
    double md[NUM_SPECIES] = {};
    for (int dr = 0; dr < NUM_DELAY_REACTIONS; ++dr) {
      const int r = dense_delay_reaction_of[dr];
      const double pert = in.perturb ? in.perturb[r] : 0.0;
      for (int sp = 0; sp < NUM_SPECIES; ++sp)
        if (deps[r][sp]) {
          const double v = in.set_params[NUM_REACTIONS + dr] * 1.0 * (1.0 + pert);
          md[sp] = (v < md[sp]) ? md[sp] : v;
        }
    }
    for (int sp = 0; sp < NUM_SPECIES; ++sp) {
      const double v = md[sp] / dt + 2;
      if (!(v >= 1.0 && v < 2147483647.0)) return nfail(DENSE_ERR_INVALID, "ring size is not a positive int");
      d.S[sp] = static_cast<int>(v);
    }
    int own_max[NUM_SPECIES], nbr_max[NUM_SPECIES];
    for (int sp = 0; sp < NUM_SPECIES; ++sp) { own_max[sp] = 0; nbr_max[sp] = -1; }
    bool ordered = false;
    int status0 = 0;
    for (int c = 0; c < (in.cell_params ? n : 1); ++c) {
      const double* prm = in.cell_params ? in.cell_params + static_cast<size_t>(c) * NUM_PARAMS : in.set_params;
      for (int i = 0; i < NUM_REACTIONS + NUM_DELAY_REACTIONS; ++i)
        if (std::isnan(prm[i])) status0 |= kSetNanParam;
      Lags t{prm, d.S, own_max, nbr_max, &ordered};
#define REACTION(name) reaction<name>::active_rate(t);
#include "reactions_list.hpp"
#undef REACTION
    }
    if (ordered) status0 |= kSetOrderedReads;
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
  if (cudaSetDevice(run->device) != cudaSuccess) return nfail(DENSE_ERR_CUDA, "cudaSetDevice failed");
  unsigned char* base = nullptr;
  int rc = scratch_address(run->device, &base);
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
