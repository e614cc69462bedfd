// BF16 GEMM on the 5th-generation tensor cores (tcgen05), for the MLP
// surrogate of the parameter search:
//
//   D[M][N] (FP32) = A[M][K] (BF16, row-major) . B[N][K]^T (BF16, row-major)
//
// with M a multiple of 128, N a multiple of 16 in [16, 256], K a multiple
// of 64, and 16-byte aligned rows (lda, ldb, ldh multiples of 8, ldd of 4).
// One CTA of 128 threads computes a 128 x N tile: the accumulator lives in
// tensor memory (N columns, one TMEM lane per output row), A and B stream
// through shared memory in chunks of 64 along K in the no-swizzle K-major
// layout the UMMA descriptors expect (8-row x 16-byte core matrices; the
// two core matrices of one K=16 step 128 bytes apart, 8-row groups 1024
// bytes apart).  One elected thread issues four tcgen05.mma (M=128, N,
// K=16) per chunk and commits them to an mbarrier; every thread waits on it
// (with an iteration limit) before the chunk buffer is refilled.  The
// epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31), adds the layer's bias and activation and writes 16-byte
// vectors.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace dense_b200 {
namespace mlp {

constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr int kGemmThreads = 128;

enum Epilogue : int {
  kEpiStore = 0,      // D -> FP32
  kEpiBiasGelu = 1,   // Z = D + bias -> FP32 (kept for the backward pass), H = GELU(Z) -> BF16
  kEpiBias = 2,       // D + bias -> FP32
};

enum : int { kErrTimeout = 1, kErrShape = 2 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, no swizzle, K-major: start address, leading
// byte offset (between the two K core matrices of a K=16 step), stride byte
// offset (between 8-row groups), all in 16-byte units; descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr & 0x3FFFF) >> 4) | (static_cast<uint64_t>(lbo >> 4) << 16) |
         (static_cast<uint64_t>(sbo >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulate, BF16 A and B, both
// K-major, N and M as given.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits on the mbarrier phase for at most ~2^31 clock cycles.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > (1ll << 31)) return false;
  }
  return true;
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.3989422804014327f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}

template <int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    umma_gemm_kernel(const __nv_bfloat16* __restrict__ A, int lda, const __nv_bfloat16* __restrict__ B, int ldb,
                     float* __restrict__ D, int ldd, int M, int N, int K, const float* __restrict__ bias,
                     __nv_bfloat16* __restrict__ H, int ldh, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  // A chunk: 128 x 64 BF16 = 16 KB; B chunk: N x 64 BF16 <= 32 KB
  unsigned char* sA = smem;
  unsigned char* sB = smem + kTileM * kChunkK * 2;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_flag;
  __shared__ float s_bias[256];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row0 = blockIdx.x * kTileM;
  if ((M % kTileM) || (N % 16) || N < 16 || N > 256 || (K % kChunkK)) {
    if (tid == 0) atomicOr(err, kErrShape);
    return;
  }
  uint32_t ncols = 32;
  while (ncols < static_cast<uint32_t>(N)) ncols <<= 1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    abort_flag = 0;
  }
  if (EPI != kEpiStore)
    for (int i = tid; i < N; i += kGemmThreads) s_bias[i] = bias[i];
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_sh;
  const uint32_t bar = smem_u32(&mbar);
  const uint32_t idesc = umma_idesc_bf16(kTileM, N);

  uint32_t phase = 0;
  for (int kc = 0; kc < K; kc += kChunkK) {
    // A chunk: 128 rows x 8 vectors of 8 BF16; vector (r, c) -> group r/8,
    // core matrix c, row r%8: byte (r/8)*1024 + c*128 + (r%8)*16
    for (int v = tid; v < kTileM * 8; v += kGemmThreads) {
      const int r = v >> 3, c = v & 7;
      const uint4 x = *reinterpret_cast<const uint4*>(A + static_cast<size_t>(row0 + r) * lda + kc + c * 8);
      *reinterpret_cast<uint4*>(sA + (r >> 3) * 1024 + c * 128 + (r & 7) * 16) = x;
    }
    for (int v = tid; v < N * 8; v += kGemmThreads) {
      const int r = v >> 3, c = v & 7;
      const uint4 x = *reinterpret_cast<const uint4*>(B + static_cast<size_t>(r) * ldb + kc + c * 8);
      *reinterpret_cast<uint4*>(sB + (r >> 3) * 1024 + c * 128 + (r & 7) * 16) = x;
    }
    // make the generic-proxy stores visible to the tensor cores
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int j = 0; j < kChunkK / 16; ++j) {
        const uint64_t da = umma_desc(smem_u32(sA) + j * 256, 128, 1024);
        const uint64_t db = umma_desc(smem_u32(sB) + j * 256, 128, 1024);
        const uint32_t accumulate = (kc > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                   : "memory");
    }
    // the chunk buffers are reused: wait until the MMAs reading them are done
    if (!mbar_wait_bounded(bar, phase)) {
      atomicOr(err, kErrTimeout);
      abort_flag = 1;
    }
    phase ^= 1u;
    __syncthreads();
    if (abort_flag) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (!abort_flag) {
    // epilogue: warp w reads TMEM lanes 32w..32w+31 = output rows
    // warp w reads TMEM lanes 32w..32w+31, the accumulator rows of its threads
    const int row = row0 + warp * 32 + lane;
    for (int c0 = 0; c0 < N; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      // 16 consecutive columns of this thread's row: four 16-byte stores
      // (and two for the BF16 activations)
      float v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]) + (EPI != kEpiStore ? s_bias[c0 + j] : 0.f);
      float4* drow = reinterpret_cast<float4*>(D + static_cast<size_t>(row) * ldd + c0);
#pragma unroll
      for (int j = 0; j < 4; ++j) drow[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
      if (EPI == kEpiBiasGelu) {
        uint32_t hp[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const __nv_bfloat162 h2 = __floats2bfloat162_rn(gelu(v[2 * j]), gelu(v[2 * j + 1]));
          hp[j] = *reinterpret_cast<const uint32_t*>(&h2);
        }
        uint4* hrow = reinterpret_cast<uint4*>(H + static_cast<size_t>(row) * ldh + c0);
        hrow[0] = make_uint4(hp[0], hp[1], hp[2], hp[3]);
        hrow[1] = make_uint4(hp[4], hp[5], hp[6], hp[7]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// The same product with the operands brought in by the Tensor Memory
// Accelerator: per 64-wide K chunk, 8 boxes of {8 K-elements, 128 rows} of A
// and 8 of {8, N} of B land as columns of core matrices (row r of box c at
// c * rows * 16 + r * 16), so a K=16 step's two core matrices are
// rows * 16 bytes apart (leading byte offset) and 8-row groups 128 bytes
// apart (stride byte offset).  Two chunk buffers: thread 0 loads chunk k+1
// while the tensor cores multiply chunk k; each buffer has a "full"
// mbarrier (TMA bytes landed) and an "empty" one (the MMAs reading it
// committed).  Every wait is bounded.
template <int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    umma_gemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                         float* __restrict__ D, int ldd, int M, int N, int K, const float* __restrict__ bias,
                         __nv_bfloat16* __restrict__ H, int ldh, int* err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const int stage_bytes = (kTileM + N) * kChunkK * 2;
  __shared__ __align__(8) uint64_t full_bar[2], empty_bar[2];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_flag;
  __shared__ uint32_t s_final;  // stage and barrier parity of the last chunk's MMA commit
  __shared__ float s_bias[256];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row0 = blockIdx.x * kTileM;
  if ((M % kTileM) || (N % 16) || N < 16 || N > 256 || (K % kChunkK)) {
    if (tid == 0) atomicOr(err, kErrShape);
    return;
  }
  uint32_t ncols = 32;
  while (ncols < static_cast<uint32_t>(N)) ncols <<= 1;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_sh)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int i = 0; i < 2; ++i) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full_bar[i])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty_bar[i])));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  if (EPI != kEpiStore)
    for (int i = tid; i < N; i += kGemmThreads) s_bias[i] = bias[i];
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_sh;
  const uint32_t idesc = umma_idesc_bf16(kTileM, N);
  const int n_chunks = K / kChunkK;

  if (tid == 0) {
    uint32_t full_ph[2] = {0u, 0u}, empty_ph[2] = {0u, 0u};
    int loads[2] = {0, 0}, landed[2] = {0, 0};  // per buffer: loads issued, loads waited for
    bool bad = false;
    auto load = [&](int c) {
      const int st = c & 1;
      ++loads[st];
      unsigned char* sA = smem + st * stage_bytes;
      unsigned char* sB = sA + kTileM * kChunkK * 2;
      const uint32_t fb = smem_u32(&full_bar[st]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fb), "r"(stage_bytes)
                   : "memory");
#pragma unroll
      for (int j = 0; j < kChunkK / 8; ++j) {
        const int x = c * kChunkK + j * 8;
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(smem_u32(sA + j * kTileM * 16)),
            "l"(reinterpret_cast<uint64_t>(&tmA)), "r"(x), "r"(row0), "r"(fb)
            : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(smem_u32(sB + j * N * 16)),
            "l"(reinterpret_cast<uint64_t>(&tmB)), "r"(x), "r"(0), "r"(fb)
            : "memory");
      }
    };
    load(0);
    for (int c = 0; c < n_chunks && !bad; ++c) {
      const int st = c & 1;
      if (c + 1 < n_chunks) {
        const int ns = (c + 1) & 1;
        if (c + 1 >= 2) {  // the buffer's previous MMAs must have finished reading it
          if (!mbar_wait_bounded(smem_u32(&empty_bar[ns]), empty_ph[ns])) bad = true;
          empty_ph[ns] ^= 1u;
        }
        if (!bad) load(c + 1);
      }
      if (bad) break;
      if (!mbar_wait_bounded(smem_u32(&full_bar[st]), full_ph[st])) {
        bad = true;
        break;
      }
      full_ph[st] ^= 1u;
      ++landed[st];
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* sA = smem + st * stage_bytes;
      unsigned char* sB = sA + kTileM * kChunkK * 2;
#pragma unroll
      for (int j = 0; j < kChunkK / 16; ++j) {
        const uint64_t da = umma_desc(smem_u32(sA) + j * 2 * kTileM * 16, kTileM * 16, 128);
        const uint64_t db = umma_desc(smem_u32(sB) + j * 2 * N * 16, N * 16, 128);
        const uint32_t accumulate = (c > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&empty_bar[st]))
                   : "memory");
    }
    if (bad) {
      atomicOr(err, kErrTimeout);
      abort_flag = 1;
      // copies still in flight land before the CTA gives up its shared memory
      for (int st = 0; st < 2; ++st)
        if (loads[st] > landed[st]) mbar_wait_bounded(smem_u32(&full_bar[st]), full_ph[st]);
    }
    // the last chunk's commit: its buffer, and the parity of that barrier's
    // last phase (every earlier phase of it was waited for above)
    const int last_stage = (n_chunks - 1) & 1;
    s_final = static_cast<uint32_t>(last_stage) | (empty_ph[last_stage] << 1);
  }
  __syncthreads();
  if (!abort_flag) {
    const uint32_t code = s_final;
    if (!mbar_wait_bounded(smem_u32(&empty_bar[code & 1]), (code >> 1) & 1u)) {
      atomicOr(err, kErrTimeout);
      abort_flag = 1;
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  if (!abort_flag) {
    const int row = row0 + warp * 32 + lane;
    for (int c0 = 0; c0 < N; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      float v[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]) + (EPI != kEpiStore ? s_bias[c0 + j] : 0.f);
      float4* drow = reinterpret_cast<float4*>(D + static_cast<size_t>(row) * ldd + c0);
#pragma unroll
      for (int j = 0; j < 4; ++j) drow[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
      if (EPI == kEpiBiasGelu) {
        uint32_t hp[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const __nv_bfloat162 h2 = __floats2bfloat162_rn(gelu(v[2 * j]), gelu(v[2 * j + 1]));
          hp[j] = *reinterpret_cast<const uint32_t*>(&h2);
        }
        uint4* hrow = reinterpret_cast<uint4*>(H + static_cast<size_t>(row) * ldh + c0);
        hrow[0] = make_uint4(hp[0], hp[1], hp[2], hp[3]);
        hrow[1] = make_uint4(hp[4], hp[5], hp[6], hp[7]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

inline size_t umma_gemm_tma_smem(int n) {
  return 2 * (static_cast<size_t>(kTileM) + static_cast<size_t>(n)) * kChunkK * 2;
}

inline size_t umma_gemm_smem(int n) { return static_cast<size_t>(kTileM) * kChunkK * 2 + static_cast<size_t>(n) * kChunkK * 2; }

}  // namespace mlp
}  // namespace dense_b200
