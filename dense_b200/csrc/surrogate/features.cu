// Search-side kernels around the surrogate: the synchrony feature of a
// batch of simulated trajectories, the candidates' network inputs, and the
// ensemble's ranking score.  C ABI: device pointers and a stream.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "dense_b200_surrogate.h"

#include <cmath>
#include <cstdint>

#if defined(__GNUC__)
#define FEATURES_API extern "C" __attribute__((visibility("default")))
#else
#define FEATURES_API extern "C"
#endif

namespace {

constexpr int kSyncThreads = 256;
constexpr int kMaxSyncCells = 1024;

__device__ __forceinline__ double quiet_nan() { return __longlong_as_double(0x7FF8000000000000LL); }

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) t += red[i];  // warps in order
  return t;
}

__device__ __forceinline__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) t = fmax(t, red[i]);
  return t;
}

// Mean pairwise Pearson correlation across the cells of each set's
// trajectory X[set][t][cell] (t < counts[set]; cells contiguous), cells
// with a constant trace left out:
//   sum_{i != j} <z_i, z_j> = |sum_i z_i|^2 - n  for unit, zero-mean z_i,
// divided by n (n - 1); NaN when fewer than two cells remain.  One CTA per
// set: per cell the mean and the norm (two passes over the samples, in
// sample order), then per sample the sum over cells of z (a warp per
// sample, lanes over cells) and the sum of its squares.
__global__ void __launch_bounds__(kSyncThreads) synchrony_kernel(const double* __restrict__ X, int64_t set_stride,
                                                                 int64_t sample_stride, int cells,
                                                                 const int* __restrict__ counts,
                                                                 double* __restrict__ out) {
  __shared__ double mean[kMaxSyncCells], scale[kMaxSyncCells];
  __shared__ double red[kSyncThreads / 32];
  const int set = blockIdx.x;
  const int T = counts[set];
  const double* x = X + set * set_stride;
  double top = 0.0, nan_seen = 0.0;
  for (int c = threadIdx.x; c < cells; c += blockDim.x) {
    double s = 0.0;
    for (int t = 0; t < T; ++t) {
      const double v = x[t * sample_stride + c];
      s += v;
      top = fmax(top, fabs(v));
      if (isnan(v)) nan_seen = 1.0;
    }
    mean[c] = T > 0 ? s / T : 0.0;
  }
  top = block_max(top, red);
  // a NaN sample makes the largest magnitude NaN, and then no cell counts
  if (block_max(nan_seen, red) > 0.0) top = quiet_nan();
  double n_ok = 0.0;
  for (int c = threadIdx.x; c < cells; c += blockDim.x) {
    const double m = mean[c];
    double q = 0.0;
    for (int t = 0; t < T; ++t) {
      const double d = x[t * sample_stride + c] - m;
      q += d * d;
    }
    const double nrm = sqrt(q);
    const bool ok = nrm > 1e-12 * (1.0 + top);
    scale[c] = ok ? nrm : 0.0;
    n_ok += ok ? 1.0 : 0.0;
  }
  const double n = block_sum(n_ok, red);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
  double s2 = 0.0;
  for (int t = warp; t < T; t += warps) {
    double s = 0.0;
    for (int c = lane; c < cells; c += 32) {
      const double nrm = scale[c];
      if (nrm > 0.0) s += (x[t * sample_stride + c] - mean[c]) / nrm;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    s2 += s * s;
  }
  const double total = block_sum(lane == 0 ? s2 : 0.0, red);
  if (threadIdx.x == 0) out[set] = n >= 2.0 ? (total - n) / (n * (n - 1.0)) : quiet_nan();
}

// Network inputs of candidates P[r][ldp] (float64 parameters):
// Xb[r][j] = BF16(float32(log(P[r][idx[j]] / tmpl[j]) / log_spread)) for
// j < k, zeros in the padding columns and in rows n..Bp-1.
__global__ void encode_kernel(const double* __restrict__ P, int ldp, int n, const int* __restrict__ idx,
                              const double* __restrict__ tmpl, int k, double log_spread, __nv_bfloat16* __restrict__ Xb,
                              int in_pad, int Bp) {
  const int64_t total = static_cast<int64_t>(Bp) * in_pad;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / in_pad), j = static_cast<int>(i % in_pad);
    float v = 0.f;
    if (r < n && j < k) v = static_cast<float>(log(P[static_cast<int64_t>(r) * ldp + idx[j]] / tmpl[j]) / log_spread);
    Xb[i] = __float2bfloat16(v);
  }
}

// acc = Y (first network) or acc + Y, in float32, over [n][nout].
__global__ void ensemble_accumulate_kernel(const float* __restrict__ Y, int ldy, int n, int nout,
                                           float* __restrict__ acc, int first) {
  const int64_t total = static_cast<int64_t>(n) * nout;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int r = static_cast<int>(i / nout), c = static_cast<int>(i % nout);
    const float y = Y[static_cast<int64_t>(r) * ldy + c];
    acc[i] = first ? y : __fadd_rn(acc[i], y);
  }
}

// The ranking score of each candidate from the ensemble sum acc[n][nout]
// (outputs: log period, log amplitude, synchrony, oscillation indicator,
// acceptance indicator): y = (acc / nets) * sd + mu in float32, then in
// float64  y4 + w * (-|exp(clamp(y0, -10, 10)) - period| / tol
//                    + 0.5 clamp((y1 - log amp_min) / ramp + 0.5, 0, 1)
//                    + 0.5 clamp(y3, 0, 1)).
struct ScoreParams {
  float mu[8], sd[8];
  float nets;
  double weight, period, tol, log_amp_min, ramp;
};

__global__ void score_kernel(const float* __restrict__ acc, int n, int nout, const ScoreParams sp,
                             double* __restrict__ out) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double y[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const float a = __fdiv_rn(acc[static_cast<int64_t>(r) * nout + j], sp.nets);
      y[j] = static_cast<double>(__fadd_rn(__fmul_rn(a, sp.sd[j]), sp.mu[j]));
    }
    const double per = exp(fmin(fmax(y[0], -10.0), 10.0));
    const double amp_term = fmin(fmax((y[1] - sp.log_amp_min) / sp.ramp + 0.5, 0.0), 1.0);
    const double osc_term = fmin(fmax(y[3], 0.0), 1.0);
    const double region = -fabs(per - sp.period) / sp.tol + 0.5 * amp_term + 0.5 * osc_term;
    out[r] = y[4] + sp.weight * region;
  }
}

int blocks_for(int64_t n) {
  const int64_t b = (n + 255) / 256;
  return static_cast<int>(b < 4096 ? (b > 0 ? b : 1) : 4096);
}

}  // namespace

FEATURES_API int dense_features_synchrony(const double* X, int64_t set_stride, int64_t sample_stride, int cells,
                                          const int* counts, int n_sets, double* out, void* stream) {
  if (n_sets < 0 || cells < 0 || cells > kMaxSyncCells) return 1;
  if (n_sets == 0) return 0;
  synchrony_kernel<<<n_sets, kSyncThreads, 0, static_cast<cudaStream_t>(stream)>>>(X, set_stride, sample_stride, cells,
                                                                                  counts, out);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

FEATURES_API int dense_features_encode(const double* P, int ldp, int n, const int* idx, const double* tmpl, int k,
                                       double log_spread, void* Xb, int in_pad, int Bp, void* stream) {
  if (n < 0 || Bp < n || k > in_pad || k < 0 || !(log_spread != 0.0)) return 1;
  encode_kernel<<<blocks_for(static_cast<int64_t>(Bp) * in_pad), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      P, ldp, n, idx, tmpl, k, log_spread, static_cast<__nv_bfloat16*>(Xb), in_pad, Bp);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

FEATURES_API int dense_features_ensemble_accumulate(const float* Y, int ldy, int n, int nout, float* acc, int first,
                                                    void* stream) {
  if (n < 0 || nout <= 0 || ldy < nout) return 1;
  ensemble_accumulate_kernel<<<blocks_for(static_cast<int64_t>(n) * nout), 256, 0,
                               static_cast<cudaStream_t>(stream)>>>(Y, ldy, n, nout, acc, first);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// mu and sd (nout floats each) are host arrays.
FEATURES_API int dense_features_score(const float* acc, int n, int nout, int nets, const float* mu, const float* sd,
                                      double weight, double period, double tol, double amp_min, double ramp,
                                      double* out, void* stream) {
  if (n < 0 || nout < 5 || nout > 8 || nets <= 0 || !(amp_min > 0.0) || !(tol > 0.0) || !(ramp > 0.0)) return 1;
  ScoreParams sp{};
  for (int j = 0; j < nout; ++j) {
    sp.mu[j] = mu[j];
    sp.sd[j] = sd[j];
  }
  sp.nets = static_cast<float>(nets);
  sp.weight = weight;
  sp.period = period;
  sp.tol = tol;
  sp.log_amp_min = std::log(amp_min);
  sp.ramp = ramp;
  score_kernel<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(acc, n, nout, sp, out);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
