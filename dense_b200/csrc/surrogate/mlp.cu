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

#include <cstdint>
#include <mutex>

#include "umma_gemm.cuh"

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
__global__ void mse_kernel(const float* __restrict__ Y, int ldy, const float* __restrict__ T,
                           const float* __restrict__ mask, int rows, int nout, float inv_count,
                           float* __restrict__ dY, __nv_bfloat16* __restrict__ dYb, float* __restrict__ loss) {
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
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// db[c] = sum_r dZ[r][c]; one thread per column, rows in order.
__global__ void colsum_kernel(const float* __restrict__ dZ, int rows, int cols, float* __restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += dZ[static_cast<int64_t>(r) * cols + c];
  db[c] = s;
}

// Adam (Kingma & Ba, 2015) with bias correction.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
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

int grid_for(int64_t n) {
  int64_t g = (n + 255) / 256;
  return static_cast<int>(g < 4096 ? (g > 0 ? g : 1) : 4096);
}

// D = A . B^T (+ bias, GELU -> H) on the tensor cores; see umma_gemm.cuh
// for the shape rules.  err (device int) collects kErr* bits.
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

template <int EPI>
cudaError_t launch_tma(const CUtensorMap& ma, const CUtensorMap& mb, float* D, int ldd, int M, int N, int K,
                       const float* bias, __nv_bfloat16* h, int ldh, int* err, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(umma_gemm_tma_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       100 * 1024);
  if (e != cudaSuccess) return e;
  umma_gemm_tma_kernel<EPI><<<M / kTileM, kGemmThreads, umma_gemm_tma_smem(N), s>>>(ma, mb, D, ldd, M, N, K, bias,
                                                                                     h, ldh, err);
  return cudaGetLastError();
}

}  // namespace

MLP_API int dense_mlp_gemm(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K,
                           int epilogue, const float* bias, void* H, int ldh, int* err, void* stream) {
  if ((M % kTileM) || (N % 16) || N < 16 || N > 256 || (K % kChunkK) || (lda % 8) || (ldb % 8) || (ldd % 4) ||
      (epilogue == kEpiBiasGelu && (ldh % 8)) || epilogue < kEpiStore || epilogue > kEpiBias)
    return 1;
  {
    // operands through the Tensor Memory Accelerator when its maps can be made
    CUtensorMap ma, mb;
    if ((reinterpret_cast<uintptr_t>(A) % 16) == 0 && (reinterpret_cast<uintptr_t>(B) % 16) == 0 &&
        bf16_map(&ma, A, M, K, lda, kTileM) && bf16_map(&mb, B, N, K, ldb, N)) {
      cudaStream_t s = static_cast<cudaStream_t>(stream);
      auto* h = static_cast<__nv_bfloat16*>(H);
      const cudaError_t e =
          epilogue == kEpiStore      ? launch_tma<kEpiStore>(ma, mb, D, ldd, M, N, K, bias, h, ldh, err, s)
          : epilogue == kEpiBiasGelu ? launch_tma<kEpiBiasGelu>(ma, mb, D, ldd, M, N, K, bias, h, ldh, err, s)
                                     : launch_tma<kEpiBias>(ma, mb, D, ldd, M, N, K, bias, h, ldh, err, s);
      return e == cudaSuccess ? 0 : 2;
    }
  }
  const size_t smem = umma_gemm_smem(N);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const auto* a = static_cast<const __nv_bfloat16*>(A);
  const auto* b = static_cast<const __nv_bfloat16*>(B);
  auto* h = static_cast<__nv_bfloat16*>(H);
  cudaError_t e;
  switch (epilogue) {
    case kEpiStore:
      e = cudaFuncSetAttribute(umma_gemm_kernel<kEpiStore>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
      if (e == cudaSuccess)
        umma_gemm_kernel<kEpiStore><<<M / kTileM, kGemmThreads, smem, s>>>(a, lda, b, ldb, D, ldd, M, N, K, bias, h,
                                                                           ldh, err);
      break;
    case kEpiBiasGelu:
      e = cudaFuncSetAttribute(umma_gemm_kernel<kEpiBiasGelu>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               64 * 1024);
      if (e == cudaSuccess)
        umma_gemm_kernel<kEpiBiasGelu><<<M / kTileM, kGemmThreads, smem, s>>>(a, lda, b, ldb, D, ldd, M, N, K, bias,
                                                                              h, ldh, err);
      break;
    case kEpiBias:
      e = cudaFuncSetAttribute(umma_gemm_kernel<kEpiBias>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
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
  mse_kernel<<<grid_for(static_cast<int64_t>(rows) * ldy), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      Y, ldy, T, mask, rows, nout, inv_count, dY, static_cast<__nv_bfloat16*>(dYb), loss);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

MLP_API int dense_mlp_colsum(const float* dZ, int rows, int cols, float* db, void* stream) {
  colsum_kernel<<<(cols + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(dZ, rows, cols, db);
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
                                                                          1.f - c2);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
