// Persistent form of the tensor-core GEMM of umma_gemm.cuh (same product,
// same shape rules, N a multiple of 32):
//
//   D[M][N] (FP32) = A[M][K] . B[N][K]^T (+ bias, GELU -> H in BF16)
//
// One CTA per SM walks the work units u = blockIdx.x, += gridDim.x.  A unit
// is a 128-row tile of D, or with split-K a tile and a range of K chunks,
// or with column blocks (few row tiles, K too short to split) a tile and a
// block of N / nsplit columns.
// Ten warps with fixed roles:
//
//   warp 0     one thread drives the Tensor Memory Accelerator: A chunks of
//              {64 K, 128 rows} into a ring of shared-memory stages ("full"
//              mbarrier per stage, byte-counted; "empty" mbarrier released by
//              the MMAs that read it).  B is either loaded once and kept
//              (resident: N x K x 2 bytes fit) or streamed beside A.
//   warp 1     owns the tensor memory (two accumulators of N columns) and one
//              thread issues tcgen05.mma (M = 128, N, K = 16) for a unit into
//              accumulator t & 1, then commits to that accumulator's "full"
//              barrier; before reusing it, it waits for its "empty" barrier.
//   warps 2-9  the epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 and
//              every other 32-column group (two warps per lane quadrant),
//              releases the accumulator as soon as its last columns are in
//              registers (so the next unit's MMAs run under this unit's
//              stores), adds bias / GELU and writes 32 x 32 boxes through
//              swizzled staging buffers with TMA stores (bulk-group waits
//              before a buffer is reused).
//
// Split-K (units of the same tile over disjoint K ranges, for products
// with few row tiles and a long K such as the weight gradients): each unit
// stores its FP32 partial through the same epilogue into a workspace
// [splits][M][N]; splitk_reduce_kernel then sums the partials in split
// order (deterministic), applies the bias / GELU epilogue and writes D.
//
// Every mbarrier wait has an iteration limit and gives up when another
// role has given up (shared abort flag); on giving up the kernel records
// kErrTimeout, waits (bounded) for its copies and MMAs in flight and frees
// its tensor memory.  No load uses cluster multicast.
#pragma once

#include "umma_gemm.cuh"

namespace dense_b200 {
namespace mlp {

constexpr int kEpiWarps = 8;
constexpr int kPersThreads = 64 + 32 * kEpiWarps;
constexpr int kMaxStages = 8;
constexpr int kStoreBox = 32;                    // rows and columns of one epilogue store box
constexpr uint32_t kADim = kTileM * kChunkK * 2;  // bytes of one A chunk (16 KB)
constexpr uint32_t kStageD = kStoreBox * kStoreBox * 4;  // FP32 staging box, 128-byte swizzle
constexpr uint32_t kStageH = kStoreBox * kStoreBox * 2;  // BF16 staging box, 64-byte swizzle

struct PersistentArgs {
  int M, N, K;
  int tiles;             // M / 128
  int splits;            // K ranges per tile (1: no split)
  int nsplit;            // column blocks per tile (1: the whole N)
  int n_blk;             // columns of one block, N / nsplit (a multiple of 32)
  int chunks_per_split;  // K chunks of 64 per unit
  int stages;            // shared-memory ring depth
  int resident_b;        // B loaded once for the whole launch
  int out_bufs;          // staging buffers per epilogue warp (1 or 2)
  uint32_t b_bytes;      // resident B region (bytes, 1024-aligned)
  uint32_t stage_bytes;  // one ring stage
  const float* bias;
  int* err;
};

// Dynamic shared memory the persistent kernel needs (its layout plus 1 KB
// to align the layout's base to 1024 bytes), 0 when the shape does not
// fit in `limit` bytes of dynamic shared memory.  Prefers, in order: B
// resident with two staging buffers per epilogue warp, B resident with
// one, B streamed with two, then with one; at least three ring stages when
// B is resident, two when streamed.  Fills stages /
// resident_b / out_bufs / b_bytes / stage_bytes of `a`; `epi` is the
// epilogue the kernel itself applies.
inline size_t persistent_smem(PersistentArgs& a, int epi, size_t limit) {
  if (limit < 1024 + kADim) return 0;
  const size_t room = limit - 1024;
  const size_t b_all = static_cast<size_t>(a.n_blk) * static_cast<size_t>(a.K) * 2;
  const size_t b_chunk = static_cast<size_t>(a.n_blk) * kChunkK * 2;
  const size_t per_buf = kStageD + (epi == kEpiBiasGelu ? kStageH : 0);
  struct Option {
    bool resident;
    int bufs;
  };
  const Option options[4] = {{true, 2}, {true, 1}, {false, 2}, {false, 1}};
  for (const Option& o : options) {
    const size_t staging = static_cast<size_t>(kEpiWarps) * o.bufs * per_buf;
    const size_t b_bytes = o.resident ? ((b_all + 1023) & ~static_cast<size_t>(1023)) : 0;
    const size_t stage = kADim + (o.resident ? 0 : b_chunk);
    const int min_stages = o.resident ? 3 : 2;
    if (o.resident && (a.splits > 1 || a.nsplit > 1 || b_all > 128 * 1024)) continue;
    if (staging + b_bytes + min_stages * stage > room) continue;
    int st = static_cast<int>((room - staging - b_bytes) / stage);
    if (st > kMaxStages) st = kMaxStages;
    a.resident_b = o.resident;
    a.out_bufs = o.bufs;
    a.b_bytes = static_cast<uint32_t>(b_bytes);
    a.stage_bytes = static_cast<uint32_t>(stage);
    a.stages = st;
    return b_bytes + static_cast<size_t>(st) * stage + staging + 1024;
  }
  return 0;
}

// Waits on an mbarrier phase for at most ~2^31 clock cycles, or until
// another role of the CTA has given up.
__device__ __forceinline__ bool mbar_wait_or_abort(uint32_t bar, uint32_t parity, const volatile int* abort) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort) return false;
    if (clock64() - t0 > (1ll << 31)) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(src)
               : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int EPI>
__device__ __forceinline__ void epilogue_values(const uint32_t (&r)[32], const float* s_bias, int c0, float (&v)[32]) {
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]) + (EPI != kEpiStore ? s_bias[c0 + j] : 0.f);
}

// tmD covers D, or with split-K the workspace [splits * M][N] (partial of
// split s of tile t at rows s * M + 128 t); EPI is then kEpiStore.
template <int EPI>
__global__ void __launch_bounds__(kPersThreads, 1)
    umma_gemm_persistent_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                                const __grid_constant__ CUtensorMap tmD, const __grid_constant__ CUtensorMap tmH,
                                const PersistentArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kMaxStages], empty_bar[kMaxStages];
  __shared__ __align__(8) uint64_t bres_bar, mma_done_bar, acc_full[2], acc_empty[2];
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_flag;
  __shared__ float s_bias[256];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // N: the columns of one unit's accumulator (a block of the output's)
  const int N = p.n_blk, S = p.stages, splits = p.splits, cps = p.chunks_per_split, nsplit = p.nsplit;
  const int n_chunks = p.K / kChunkK;
  const int per_tile = splits * nsplit;  // units per 128-row tile: K ranges x column blocks
  const int units = p.tiles * per_tile;
  // the 128-byte swizzle of the staging boxes repeats every 1024 bytes of
  // shared-memory address: the layout starts on such a boundary
  unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  unsigned char* sBres = smem;
  unsigned char* ring = smem + p.b_bytes;
  unsigned char* staging = ring + static_cast<size_t>(S) * p.stage_bytes;

  uint32_t ncols = 32;
  while (ncols < static_cast<uint32_t>(2 * N)) ncols <<= 1;
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < S; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full_bar[i])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty_bar[i])));
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bres_bar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mma_done_bar)));
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&acc_full[i])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&acc_empty[i])), "r"(kEpiWarps));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  if (EPI != kEpiStore)
    for (int i = tid; i < p.N; i += kPersThreads) s_bias[i] = p.bias[i];
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_sh;

  if (warp == 0) {
    if (lane == 0) {
      // ---------------------------------------------------------- producer
      uint32_t it = 0;
      bool bad = false;
      if (p.resident_b) {
        const uint32_t bar = smem_u32(&bres_bar);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(static_cast<uint32_t>(N) * static_cast<uint32_t>(p.K) * 2u)
                     : "memory");
        for (int g = 0; g < p.K / 8; ++g)
          tma_load_2d(smem_u32(sBres + static_cast<size_t>(g) * N * 16), &tmB, g * 8, 0, bar);
      }
      for (int u = blockIdx.x; u < units && !bad; u += gridDim.x) {
        const int tile = u / per_tile, c0 = ((u % per_tile) / nsplit) * cps, nb = u % nsplit;
        const int c1 = min(c0 + cps, n_chunks);
        for (int c = c0; c < c1; ++c, ++it) {
          const int s = static_cast<int>(it % static_cast<uint32_t>(S));
          if (it >= static_cast<uint32_t>(S) &&
              !mbar_wait_or_abort(smem_u32(&empty_bar[s]), ((it / S) - 1) & 1u, &abort_flag)) {
            bad = true;
            break;
          }
          unsigned char* sA = ring + static_cast<size_t>(s) * p.stage_bytes;
          const uint32_t fb = smem_u32(&full_bar[s]);
          asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(p.stage_bytes)
                       : "memory");
#pragma unroll
          for (int j = 0; j < kChunkK / 8; ++j)
            tma_load_2d(smem_u32(sA + j * kTileM * 16), &tmA, c * kChunkK + j * 8, tile * kTileM, fb);
          if (!p.resident_b) {
            unsigned char* sB = sA + kADim;
#pragma unroll
            for (int j = 0; j < kChunkK / 8; ++j)
              tma_load_2d(smem_u32(sB + j * N * 16), &tmB, c * kChunkK + j * 8, nb * N, fb);
          }
        }
      }
      if (bad) {
        atomicOr(p.err, kErrTimeout);
        abort_flag = 1;
      }
      // the copies issued last into each stage (and B) land before the CTA
      // gives up its shared memory (at once when the MMAs consumed them)
      for (int s = 0; s < S; ++s) {
        if (static_cast<uint32_t>(s) >= it) break;
        const uint32_t last = it - 1u - ((it - 1u - static_cast<uint32_t>(s)) % static_cast<uint32_t>(S));
        mbar_wait_bounded(smem_u32(&full_bar[s]), (last / S) & 1u);
      }
      if (p.resident_b) mbar_wait_bounded(smem_u32(&bres_bar), 0u);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------------------------------------------------- MMA issuer
      const uint32_t idesc = umma_idesc_bf16(kTileM, N);
      uint32_t it = 0;
      bool bad = false;
      if (p.resident_b && !mbar_wait_or_abort(smem_u32(&bres_bar), 0u, &abort_flag)) bad = true;
      int t = 0;
      for (int u = blockIdx.x; u < units && !bad; u += gridDim.x, ++t) {
        const int a = t & 1, use = t >> 1;
        if (use >= 1 && !mbar_wait_or_abort(smem_u32(&acc_empty[a]), (use - 1) & 1, &abort_flag)) {
          bad = true;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t acc = tmem + static_cast<uint32_t>(a * N);
        const int c0 = ((u % per_tile) / nsplit) * cps;
        const int c1 = min(c0 + cps, n_chunks);
        for (int c = c0; c < c1; ++c, ++it) {
          const int s = static_cast<int>(it % static_cast<uint32_t>(S));
          if (!mbar_wait_or_abort(smem_u32(&full_bar[s]), (it / S) & 1u, &abort_flag)) {
            bad = true;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t sA = smem_u32(ring + static_cast<size_t>(s) * p.stage_bytes);
          const uint32_t sB = p.resident_b ? smem_u32(sBres) + static_cast<uint32_t>(c * (kChunkK / 8) * N * 16)
                                           : sA + kADim;
#pragma unroll
          for (int j = 0; j < kChunkK / 16; ++j) {
            const uint64_t da = umma_desc(sA + j * 2 * kTileM * 16, kTileM * 16, 128);
            const uint64_t db = umma_desc(sB + j * 2 * N * 16, N * 16, 128);
            const uint32_t accumulate = (c > c0 || j > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(acc),
                "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
          }
          asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                           smem_u32(&empty_bar[s]))
                       : "memory");
        }
        if (bad) break;
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&acc_full[a]))
                     : "memory");
      }
      if (bad) {
        atomicOr(p.err, kErrTimeout);
        abort_flag = 1;
      }
      // every MMA issued has completed before the tensor memory is freed
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mma_done_bar))
                   : "memory");
      mbar_wait_bounded(smem_u32(&mma_done_bar), 0u);
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int q = warp & 3;          // TMEM lane quadrant this warp may read
    const int half = (warp - 2) >> 2;  // which of every two column groups
    const int n_groups = N / kStoreBox;
    const uint32_t per_buf = kStageD + (EPI == kEpiBiasGelu ? kStageH : 0);
    unsigned char* st_warp = staging + static_cast<size_t>(warp - 2) * p.out_bufs * per_buf;
    uint32_t groups = 0;  // store groups this warp committed
    int t = 0;
    for (int u = blockIdx.x; u < units; u += gridDim.x, ++t) {
      const int a = t & 1, use = t >> 1;
      if (!mbar_wait_or_abort(smem_u32(&acc_full[a]), use & 1, &abort_flag)) {
        atomicOr(p.err, kErrTimeout);
        abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int tile = u / per_tile, split = (u % per_tile) / nsplit, col0 = (u % nsplit) * N;
      const int out_row = split * p.M + tile * kTileM + q * 32;  // first row of this warp's boxes
      const uint32_t tacc = tmem + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>(a * N);
      if (half >= n_groups) {  // no column group for this warp (N = 32)
        __syncwarp();
        if (lane == 0)
          asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[a])) : "memory");
        continue;
      }
      for (int g = half; g < n_groups; g += 2) {
        const int c0 = g * kStoreBox;
        uint32_t r[32];
        tmem_ld32(tacc + static_cast<uint32_t>(c0), r);
        if (g + 2 >= n_groups) {  // this warp's share of the accumulator drained
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncwarp();
          if (lane == 0)
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[a])) : "memory");
        }
        float v[32];
        epilogue_values<EPI>(r, s_bias, col0 + c0, v);
        const int buf = static_cast<int>(groups % static_cast<uint32_t>(p.out_bufs));
        // the store issued from this buffer last time has read it
        if (lane == 0) {
          if (p.out_bufs == 2)
            asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
          else
            asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        }
        __syncwarp();
        unsigned char* bd = st_warp + buf * per_buf;
#pragma unroll
        for (int j = 0; j < 8; ++j)  // 128-byte swizzle: 16-byte chunk j of row r at chunk j ^ (r & 7)
          *reinterpret_cast<float4*>(bd + lane * 128 + ((j ^ (lane & 7)) << 4)) =
              make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        unsigned char* bh = bd + kStageD;
        if (EPI == kEpiBiasGelu) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {  // 64-byte swizzle: chunk j of row r at chunk j ^ ((r >> 1) & 3)
            uint32_t hp[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const __nv_bfloat162 h2 = __floats2bfloat162_rn(gelu(v[8 * j + 2 * k]), gelu(v[8 * j + 2 * k + 1]));
              hp[k] = *reinterpret_cast<const uint32_t*>(&h2);
            }
            *reinterpret_cast<uint4*>(bh + lane * 64 + ((j ^ ((lane >> 1) & 3)) << 4)) =
                make_uint4(hp[0], hp[1], hp[2], hp[3]);
          }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) {
          tma_store_2d(&tmD, col0 + c0, out_row, smem_u32(bd));
          if (EPI == kEpiBiasGelu) tma_store_2d(&tmH, col0 + c0, out_row, smem_u32(bh));
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
        ++groups;
      }
    }
    // stores complete before the CTA's shared memory is released
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    __syncwarp();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// D = sum over splits (in split order) of the partials [splits][M][N],
// plus the bias / GELU epilogue; one thread per four columns.
template <int EPI>
__global__ void splitk_reduce_kernel(const float* __restrict__ ws, int splits, int M, int N, float* __restrict__ D,
                                     int ldd, const float* __restrict__ bias, __nv_bfloat16* __restrict__ H,
                                     int ldh) {
  const int64_t quads = static_cast<int64_t>(M) * (N / 4);
  const size_t plane = static_cast<size_t>(M) * N;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < quads;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int row = static_cast<int>(i / (N / 4)), c0 = static_cast<int>(i % (N / 4)) * 4;
    const float* src = ws + static_cast<size_t>(row) * N + c0;
    float4 acc = __ldcs(reinterpret_cast<const float4*>(src));
    for (int s = 1; s < splits; ++s) {
      const float4 x = __ldcs(reinterpret_cast<const float4*>(src + s * plane));
      acc.x += x.x;
      acc.y += x.y;
      acc.z += x.z;
      acc.w += x.w;
    }
    if (EPI != kEpiStore) {
      acc.x += bias[c0];
      acc.y += bias[c0 + 1];
      acc.z += bias[c0 + 2];
      acc.w += bias[c0 + 3];
    }
    *reinterpret_cast<float4*>(D + static_cast<size_t>(row) * ldd + c0) = acc;
    if (EPI == kEpiBiasGelu) {
      const __nv_bfloat162 h0 = __floats2bfloat162_rn(gelu(acc.x), gelu(acc.y));
      const __nv_bfloat162 h1 = __floats2bfloat162_rn(gelu(acc.z), gelu(acc.w));
      *reinterpret_cast<uint2*>(H + static_cast<size_t>(row) * ldh + c0) =
          make_uint2(*reinterpret_cast<const uint32_t*>(&h0), *reinterpret_cast<const uint32_t*>(&h1));
    }
  }
}

}  // namespace mlp
}  // namespace dense_b200
