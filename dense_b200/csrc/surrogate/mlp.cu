// Kernels of the MLP surrogate that pre-screens parameter-search
// candidates (an addition of this project: DENSE's search scores every
// candidate by simulating it, search/sres.cpp:328-345).
//
// The network maps a candidate's log-parameters to oscillation features;
// its matrix products run on the tensor cores through umma_gemm.cuh, the
// rest is elementwise.  The C ABI takes device pointers and a stream; the
// host sequences forward and backward passes (dense_b200/surrogate.py).

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "dense_b200_surrogate.h"

#include <cooperative_groups.h>

#include <atomic>
#include <cstdint>
#include <mutex>

#include "umma_gemm.cuh"
#include "umma_gemm_persistent.cuh"

#if defined(__GNUC__)
#define MLP_API extern "C" __attribute__((visibility("default")))
#else
#define MLP_API extern "C"
#endif

using namespace dense_b200::mlp;

namespace {

__global__ void transpose_bf16_kernel(const __nv_bfloat16* __restrict__ src, int rows, int cols, int lds,
                                      __nv_bfloat16* __restrict__ dst, int ldd) {
  __shared__ __nv_bfloat16 tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = by + i, c = bx + threadIdx.x;
    if (r < rows && c < cols) tile[i][threadIdx.x] = src[static_cast<size_t>(r) * lds + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = bx + i, r = by + threadIdx.x;
    if (r < rows && c < cols) dst[static_cast<size_t>(c) * ldd + r] = tile[threadIdx.x][i];
  }
}

// FP32 [rows][cols] -> BF16, optionally transposed.
__global__ void cast_bf16_kernel(const float* __restrict__ src, int rows, int cols, __nv_bfloat16* __restrict__ dst,
                                 int transpose) {
  const int64_t total = static_cast<int64_t>(rows) * cols;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / cols), c = static_cast<int>(i % cols);
    dst[transpose ? static_cast<int64_t>(c) * rows + r : i] = __float2bfloat16(src[i]);
  }
}

// dZ = dH * GELU'(Z): BF16 [rows][cols] and FP32 copies.
__global__ void gelu_backward_kernel(const float* __restrict__ dH, const float* __restrict__ Z, int64_t n,
                                     float* __restrict__ dZ, __nv_bfloat16* __restrict__ dZb) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float g = dH[i] * gelu_grad(Z[i]);
    dZ[i] = g;
    dZb[i] = __float2bfloat16(g);
  }
}

// Masked mean squared error over the first `nout` of `ldy` outputs:
// loss += sum mask (y - t)^2 / count; dY = 2 mask (y - t) / count.
// With inv_count_dev non-null the scale is read from device memory (a
// value that changes per step inside a captured graph).
__global__ void mse_kernel(const float* __restrict__ Y, int ldy, const float* __restrict__ T,
                           const float* __restrict__ mask, int rows, int nout, float inv_count,
                           const float* __restrict__ inv_count_dev, float* __restrict__ dY,
                           __nv_bfloat16* __restrict__ dYb, float* __restrict__ loss) {
  if (inv_count_dev) inv_count = *inv_count_dev;
  float acc = 0.f;
  const int64_t total = static_cast<int64_t>(rows) * ldy;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / ldy), c = static_cast<int>(i % ldy);
    float g = 0.f;
    if (c < nout) {
      const float m = mask[static_cast<int64_t>(r) * nout + c];
      const float d = Y[i] - T[static_cast<int64_t>(r) * nout + c];
      acc += m * d * d * inv_count;
      g = 2.f * m * d * inv_count;
    }
    dY[i] = g;
    dYb[i] = __float2bfloat16(g);
  }
  // one atomic per block: warp sums, then the block's warps in order
  __shared__ float warp_sum[32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float b = 0.f;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) b += warp_sum[w];
    atomicAdd(loss, b);
  }
}

// db[c] = sum_r dZ[r][c].  A cluster of kColSlices CTAs per 32 columns:
// CTA rank k sums the k-th slice of the rows (32 row lanes x 32 columns,
// eight independent partial sums per thread, combined in a fixed order),
// then rank 0 adds the ranks' column sums in rank order, read from their
// shared memory over the cluster's distributed shared memory.  The order
// of every addition is fixed: the result does not depend on timing.
constexpr int kColSlices = 8;

__global__ void __cluster_dims__(1, kColSlices, 1) __launch_bounds__(1024)
    colsum_kernel(const float* __restrict__ dZ, int rows, int cols, float* __restrict__ db) {
  __shared__ float part[32][33];
  __shared__ float slice_sum[32];
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int x = threadIdx.x, y = threadIdx.y;
  const int c = blockIdx.x * 32 + x;
  const int per = (rows + kColSlices - 1) / kColSlices;
  const int r0 = blockIdx.y * per, r1 = min(rows, r0 + per);
  float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (c < cols) {
    int r = r0 + y;
    for (; r + 7 * 32 < r1; r += 8 * 32) {
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[j] += dZ[static_cast<int64_t>(r + j * 32) * cols + c];
    }
    for (; r < r1; r += 32) acc[0] += dZ[static_cast<int64_t>(r) * cols + c];
  }
  part[y][x] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
  __syncthreads();
  if (y == 0) {
    float s = 0.f;
    for (int i = 0; i < 32; ++i) s += part[i][x];
    slice_sum[x] = s;
  }
  cluster.sync();
  if (cluster.block_rank() == 0 && y == 0) {
    float s = 0.f;
    for (int k = 0; k < kColSlices; ++k) s += cluster.map_shared_rank(slice_sum, k)[x];
    if (c < cols) db[c] = s;
  }
  cluster.sync();  // every rank's shared memory stays until rank 0 has read it
}

// Adam (Kingma & Ba, 2015) with bias correction.  With hyper non-null the
// step's {lr, b1, b2, eps, c1, c2} are read from device memory (a captured
// graph replays the same launch every step).
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2, const float* __restrict__ hyper) {
  if (hyper) {
    lr = hyper[0];
    b1 = hyper[1];
    b2 = hyper[2];
    eps = hyper[3];
    c1 = hyper[4];
    c2 = hyper[5];
  }
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// One training batch gathered from the device-resident training set:
// Xb[r] = BF16 of X[idx[r]] padded with zeros to in_pad columns, Tb[r] and
// Mb[r] the row's targets and mask; rows B..Bp-1 (padding up to the GEMM's
// 128-row tile) and out-of-range indices give zeros.
__global__ void gather_rows_kernel(const float* __restrict__ X, int n_rows, int n_in, const float* __restrict__ T,
                                   const float* __restrict__ Mk, int n_out, const int* __restrict__ idx, int B,
                                   int Bp, __nv_bfloat16* __restrict__ Xb, int in_pad, float* __restrict__ Tb,
                                   float* __restrict__ Mb) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  for (int64_t i = t0; i < static_cast<int64_t>(Bp) * in_pad; i += stride) {
    const int r = static_cast<int>(i / in_pad), c = static_cast<int>(i % in_pad);
    float v = 0.f;
    if (r < B && c < n_in) {
      const int src = idx[r];
      if (src >= 0 && src < n_rows) v = X[static_cast<int64_t>(src) * n_in + c];
    }
    Xb[i] = __float2bfloat16(v);
  }
  for (int64_t i = t0; i < static_cast<int64_t>(Bp) * n_out; i += stride) {
    const int r = static_cast<int>(i / n_out), c = static_cast<int>(i % n_out);
    float tv = 0.f, mv = 0.f;
    if (r < B) {
      const int src = idx[r];
      if (src >= 0 && src < n_rows) {
        tv = T[static_cast<int64_t>(src) * n_out + c];
        mv = Mk[static_cast<int64_t>(src) * n_out + c];
      }
    }
    Tb[i] = tv;
    Mb[i] = mv;
  }
}

int grid_for(int64_t n) {
  int64_t g = (n + 255) / 256;
  return static_cast<int>(g < 4096 ? (g > 0 ? g : 1) : 4096);
}

// Blocks for the loss kernel: a few per SM, each thread several elements
// (one atomic per block).
int grid_for_reduce(int64_t n) {
  int64_t g = (n + 1023) / 1024;
  return static_cast<int>(g < 592 ? (g > 0 ? g : 1) : 592);
}

// cuTensorMapEncodeTiled, reached through the runtime's driver entry point
// (no link against the driver library); null when unavailable.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// Tensor map of a row-major BF16 matrix [rows][k] (leading dimension ld)
// read in boxes of {8 K-elements, box_rows rows}, no swizzle.
bool bf16_map(CUtensorMap* m, const void* base, int rows, int k, int ld, int box_rows) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(k), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
  const cuuint32_t box[2] = {8, static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, elem,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor map of a row-major 2-D matrix [rows][cols] (leading dimension ld
// elements of elem_bytes) written in boxes of {box_cols, box_rows} with
// the given shared-memory swizzle.
bool store_map(CUtensorMap* m, CUtensorMapDataType type, int elem_bytes, const void* base, int rows, int cols,
               int ld, int box_cols, int box_rows, CUtensorMapSwizzle swizzle) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * static_cast<cuuint64_t>(elem_bytes)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(box_cols), static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t elem[2] = {1, 1};
  return fn(m, type, 2, const_cast<void*>(base), dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle,
            CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// SMs of the current device, queried once per device.
int sm_count() {
  constexpr int kMaxDevices = 64;
  static std::atomic<int> cached[kMaxDevices] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
  int n = cached[dev].load(std::memory_order_relaxed);
  if (n > 0) return n;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  cached[dev].store(n, std::memory_order_relaxed);
  return n;
}

// Dynamic shared memory a CTA of the persistent kernel may take: the
// device's opt-in limit per block less the kernel's static shared memory.
template <int EPI>
size_t query_persistent_smem_limit() {
  int dev = 0, optin = 0;
  cudaFuncAttributes fa;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, umma_gemm_persistent_kernel<EPI>) != cudaSuccess ||
      static_cast<size_t>(optin) <= fa.sharedSizeBytes)
    return 0;
  return static_cast<size_t>(optin) - fa.sharedSizeBytes;
}

// The limit above, queried once per process (every GPU of one process is
// the same B200 part).
template <int EPI>
size_t persistent_smem_limit() {
  static std::once_flag once;
  static size_t limit = 0;
  std::call_once(once, [] { limit = query_persistent_smem_limit<EPI>(); });
  return limit;
}

// Raises a kernel's dynamic shared-memory opt-in on the current device to
// at least `bytes`, calling the runtime only when the size grows (so that
// launches inside a graph capture make no attribute calls); one record per
// kernel (the template argument).
template <auto kernel>
cudaError_t raise_smem_optin(size_t bytes) {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static size_t granted[kMaxDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (bytes <= granted[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  if (e == cudaSuccess) granted[dev] = bytes;
  return e;
}

template <int EPI>
cudaError_t launch_tma(const CUtensorMap& ma, const CUtensorMap& mb, float* D, int ldd, int M, int N, int K,
                       const float* bias, __nv_bfloat16* h, int ldh, int* err, cudaStream_t s) {
  const cudaError_t e = raise_smem_optin<umma_gemm_tma_kernel<EPI>>(umma_gemm_tma_smem(N));
  if (e != cudaSuccess) return e;
  umma_gemm_tma_kernel<EPI><<<M / kTileM, kGemmThreads, umma_gemm_tma_smem(N), s>>>(ma, mb, D, ldd, M, N, K, bias,
                                                                                     h, ldh, err);
  return cudaGetLastError();
}

template <int EPI>
cudaError_t launch_persistent(const CUtensorMap& ma, const CUtensorMap& mb, const CUtensorMap& md,
                              const CUtensorMap& mh, const PersistentArgs& a, size_t smem, int grid, cudaStream_t s) {
  const cudaError_t e = raise_smem_optin<umma_gemm_persistent_kernel<EPI>>(smem);
  if (e != cudaSuccess) return e;
  umma_gemm_persistent_kernel<EPI><<<grid, kPersThreads, smem, s>>>(ma, mb, md, mh, a);
  return cudaGetLastError();
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) % 16) == 0; }

// The persistent kernel when the shape, the alignment and the maps allow it
// (and with split-K the reduction after it): 0 launched, 1 not applicable,
// 2 launch error.
int try_persistent(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K,
                   int epilogue, const float* bias, void* H, int ldh, int* err, float* ws, size_t ws_bytes,
                   cudaStream_t s) {
  if ((N % kStoreBox) || !aligned16(A) || !aligned16(B) || !aligned16(D) ||
      (epilogue == kEpiBiasGelu && !aligned16(H)))
    return 1;
  const int sms = sm_count();
  if (sms <= 0) return 1;
  PersistentArgs a{};
  a.M = M;
  a.N = N;
  a.K = K;
  a.tiles = M / kTileM;
  a.bias = bias;
  a.err = err;
  const int n_chunks = K / kChunkK;
  a.splits = 1;
  a.chunks_per_split = n_chunks;
  a.nsplit = 1;
  a.n_blk = N;
  // split K when the row tiles leave most SMs idle and K is long: at least
  // four chunks per unit, partials in the caller's workspace
  if (ws && aligned16(ws) && a.tiles * 2 <= sms && n_chunks >= 8) {
    int splits = n_chunks / 4;
    if (splits > sms / a.tiles) splits = sms / a.tiles;
    const size_t per_split = static_cast<size_t>(M) * N * sizeof(float);
    if (static_cast<size_t>(splits) * per_split > ws_bytes) splits = static_cast<int>(ws_bytes / per_split);
    if (splits >= 2) {
      const int cps = (n_chunks + splits - 1) / splits;
      a.splits = (n_chunks + cps - 1) / cps;
      a.chunks_per_split = cps;
    }
  }
  // without a K split, few row tiles take column blocks instead (at least
  // 64 columns each), so that more SMs share the product
  if (a.splits == 1) {
    while (a.tiles * a.nsplit * 2 <= sms && (N / (a.nsplit * 2)) % kStoreBox == 0 && N / (a.nsplit * 2) >= 64)
      a.nsplit *= 2;
    a.n_blk = N / a.nsplit;
  }
  const int kernel_epi = a.splits > 1 ? kEpiStore : epilogue;
  const size_t limit = kernel_epi == kEpiStore      ? persistent_smem_limit<kEpiStore>()
                       : kernel_epi == kEpiBiasGelu ? persistent_smem_limit<kEpiBiasGelu>()
                                                    : persistent_smem_limit<kEpiBias>();
  const size_t smem = persistent_smem(a, kernel_epi, limit);
  if (!smem) return 1;
  CUtensorMap ma, mb, md, mh;
  if (!bf16_map(&ma, A, M, K, lda, kTileM) || !bf16_map(&mb, B, N, K, ldb, a.n_blk)) return 1;
  const bool mapped = a.splits > 1 ? store_map(&md, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ws, a.splits * M, N, N,
                                               kStoreBox, kStoreBox, CU_TENSOR_MAP_SWIZZLE_128B)
                                   : store_map(&md, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, D, M, N, ldd, kStoreBox,
                                               kStoreBox, CU_TENSOR_MAP_SWIZZLE_128B);
  if (!mapped) return 1;
  if (kernel_epi == kEpiBiasGelu) {
    if (!store_map(&mh, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, H, M, N, ldh, kStoreBox, kStoreBox,
                   CU_TENSOR_MAP_SWIZZLE_64B))
      return 1;
  } else {
    mh = md;
  }
  const int units = a.tiles * a.splits * a.nsplit;
  const int grid = units < sms ? units : sms;
  cudaError_t e = kernel_epi == kEpiStore ? launch_persistent<kEpiStore>(ma, mb, md, mh, a, smem, grid, s)
                  : kernel_epi == kEpiBiasGelu
                      ? launch_persistent<kEpiBiasGelu>(ma, mb, md, mh, a, smem, grid, s)
                      : launch_persistent<kEpiBias>(ma, mb, md, mh, a, smem, grid, s);
  if (e != cudaSuccess) return 2;
  if (a.splits > 1) {
    const int64_t quads = static_cast<int64_t>(M) * (N / 4);
    int blocks = static_cast<int>((quads + 255) / 256);
    if (blocks > 4 * sms) blocks = 4 * sms;
    auto* h = static_cast<__nv_bfloat16*>(H);
    if (epilogue == kEpiStore)
      splitk_reduce_kernel<kEpiStore><<<blocks, 256, 0, s>>>(ws, a.splits, M, N, D, ldd, bias, h, ldh);
    else if (epilogue == kEpiBiasGelu)
      splitk_reduce_kernel<kEpiBiasGelu><<<blocks, 256, 0, s>>>(ws, a.splits, M, N, D, ldd, bias, h, ldh);
    else
      splitk_reduce_kernel<kEpiBias><<<blocks, 256, 0, s>>>(ws, a.splits, M, N, D, ldd, bias, h, ldh);
    if (cudaGetLastError() != cudaSuccess) return 2;
  }
  return 0;
}

int gemm_impl(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K, int epilogue,
              const float* bias, void* H, int ldh, int* err, float* ws, size_t ws_bytes, void* stream) {
  if (M <= 0 || K <= 0 || (M % kTileM) || (N % 16) || N < 16 || N > 256 || (K % kChunkK) || (lda % 8) ||
      (ldb % 8) || (ldd % 4) || (epilogue == kEpiBiasGelu && (ldh % 8 || !H)) || epilogue < kEpiStore || epilogue > kEpiBias ||
      (epilogue != kEpiStore && !bias) || !A || !B || !D || !err)
    return 1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  {
    const int r = try_persistent(A, lda, B, ldb, D, ldd, M, N, K, epilogue, bias, H, ldh, err, ws, ws_bytes, s);
    if (r != 1) return r;
  }
  {
    // operands through the Tensor Memory Accelerator when its maps can be made
    CUtensorMap ma, mb;
    if (aligned16(A) && aligned16(B) && bf16_map(&ma, A, M, K, lda, kTileM) && bf16_map(&mb, B, N, K, ldb, N)) {
      auto* h = static_cast<__nv_bfloat16*>(H);
      const cudaError_t e =
          epilogue == kEpiStore      ? launch_tma<kEpiStore>(ma, mb, D, ldd, M, N, K, bias, h, ldh, err, s)
          : epilogue == kEpiBiasGelu ? launch_tma<kEpiBiasGelu>(ma, mb, D, ldd, M, N, K, bias, h, ldh, err, s)
                                     : launch_tma<kEpiBias>(ma, mb, D, ldd, M, N, K, bias, h, ldh, err, s);
      return e == cudaSuccess ? 0 : 2;
    }
  }
  const size_t smem = umma_gemm_smem(N);
  const auto* a = static_cast<const __nv_bfloat16*>(A);
  const auto* b = static_cast<const __nv_bfloat16*>(B);
  auto* h = static_cast<__nv_bfloat16*>(H);
  cudaError_t e;
  switch (epilogue) {
    case kEpiStore:
      e = raise_smem_optin<umma_gemm_kernel<kEpiStore>>(smem);
      if (e == cudaSuccess)
        umma_gemm_kernel<kEpiStore><<<M / kTileM, kGemmThreads, smem, s>>>(a, lda, b, ldb, D, ldd, M, N, K, bias, h,
                                                                           ldh, err);
      break;
    case kEpiBiasGelu:
      e = raise_smem_optin<umma_gemm_kernel<kEpiBiasGelu>>(smem);
      if (e == cudaSuccess)
        umma_gemm_kernel<kEpiBiasGelu><<<M / kTileM, kGemmThreads, smem, s>>>(a, lda, b, ldb, D, ldd, M, N, K, bias,
                                                                              h, ldh, err);
      break;
    case kEpiBias:
      e = raise_smem_optin<umma_gemm_kernel<kEpiBias>>(smem);
      if (e == cudaSuccess)
        umma_gemm_kernel<kEpiBias><<<M / kTileM, kGemmThreads, smem, s>>>(a, lda, b, ldb, D, ldd, M, N, K, bias, h,
                                                                          ldh, err);
      break;
    default:
      return 1;
  }
  if (e != cudaSuccess) return 2;
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace

// D = A . B^T (+ bias, GELU -> H) on the tensor cores; see umma_gemm.cuh
// for the shape rules.  err (device int) collects kErr* bits.  Returns 0
// launched, 1 shape / argument rejected, 2 launch error.
MLP_API int dense_mlp_gemm(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K,
                           int epilogue, const float* bias, void* H, int ldh, int* err, void* stream) {
  return gemm_impl(A, lda, B, ldb, D, ldd, M, N, K, epilogue, bias, H, ldh, err, nullptr, 0, stream);
}

// The same product with a split-K workspace: ws (ws_bytes of 16-byte
// aligned device memory, used by this call's launches only) holds the FP32
// partials when the K dimension is split across SMs (few 128-row tiles and
// K >= 512); calls sharing a workspace must be ordered on one stream.
MLP_API int dense_mlp_gemm_ws(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K,
                              int epilogue, const float* bias, void* H, int ldh, int* err, float* ws, size_t ws_bytes,
                              void* stream) {
  return gemm_impl(A, lda, B, ldb, D, ldd, M, N, K, epilogue, bias, H, ldh, err, ws, ws_bytes, stream);
}

MLP_API int dense_mlp_transpose_bf16(const void* src, int rows, int cols, int lds, void* dst, int ldd, void* stream) {
  dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
  transpose_bf16_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(src), rows, cols, lds, static_cast<__nv_bfloat16*>(dst), ldd);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

MLP_API int dense_mlp_cast_bf16(const float* src, int rows, int cols, void* dst, int transpose, void* stream) {
  cast_bf16_kernel<<<grid_for(static_cast<int64_t>(rows) * cols), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      src, rows, cols, static_cast<__nv_bfloat16*>(dst), transpose);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

MLP_API int dense_mlp_gelu_backward(const float* dH, const float* Z, int64_t n, float* dZ, void* dZb, void* stream) {
  gelu_backward_kernel<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(dH, Z, n, dZ,
                                                                                    static_cast<__nv_bfloat16*>(dZb));
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

MLP_API int dense_mlp_mse(const float* Y, int ldy, const float* T, const float* mask, int rows, int nout,
                          float inv_count, float* dY, void* dYb, float* loss, void* stream) {
  mse_kernel<<<grid_for_reduce(static_cast<int64_t>(rows) * ldy), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      Y, ldy, T, mask, rows, nout, inv_count, nullptr, dY, static_cast<__nv_bfloat16*>(dYb), loss);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// The same with the 1 / count scale read from device memory.
MLP_API int dense_mlp_mse_dev(const float* Y, int ldy, const float* T, const float* mask, int rows, int nout,
                              const float* inv_count_dev, float* dY, void* dYb, float* loss, void* stream) {
  if (!inv_count_dev) return 1;
  mse_kernel<<<grid_for_reduce(static_cast<int64_t>(rows) * ldy), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      Y, ldy, T, mask, rows, nout, 0.f, inv_count_dev, dY, static_cast<__nv_bfloat16*>(dYb), loss);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

MLP_API int dense_mlp_gather(const float* X, int n_rows, int n_in, const float* T, const float* mask, int n_out,
                             const int* idx, int B, int Bp, void* Xb, int in_pad, float* Tb, float* Mb, void* stream) {
  if (B < 0 || Bp < B || n_in > in_pad || n_rows <= 0 || n_out <= 0) return 1;
  gather_rows_kernel<<<grid_for(static_cast<int64_t>(Bp) * in_pad), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      X, n_rows, n_in, T, mask, n_out, idx, B, Bp, static_cast<__nv_bfloat16*>(Xb), in_pad, Tb, Mb);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

MLP_API int dense_mlp_colsum(const float* dZ, int rows, int cols, float* db, void* stream) {
  if (rows < 0 || cols <= 0) return 1;
  colsum_kernel<<<dim3((cols + 31) / 32, kColSlices), dim3(32, 32), 0, static_cast<cudaStream_t>(stream)>>>(
      dZ, rows, cols, db);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

MLP_API int dense_mlp_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2,
                           float eps, int step, void* stream) {
  float c1 = 1.f, c2 = 1.f, p1 = b1, p2 = b2;
  for (int i = 0; i < step; ++i) {  // 1 - beta^step
    c1 *= p1;
    c2 *= p2;
  }
  adam_kernel<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, g, m, v, n, lr, b1, b2, eps, 1.f - c1,
                                                                          1.f - c2, nullptr);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// The same with {lr, b1, b2, eps, 1 - b1^step, 1 - b2^step} read from
// device memory.
MLP_API int dense_mlp_adam_dev(float* w, const float* g, float* m, float* v, int64_t n, const float* hyper,
                               void* stream) {
  if (!hyper) return 1;
  adam_kernel<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(w, g, m, v, n, 0.f, 0.f, 0.f, 0.f, 1.f,
                                                                          1.f, hyper);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
