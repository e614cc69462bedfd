/* C ABI of the surrogate library (dense_b200/_lib/libdense_b200_surrogate.so,
 * built by dense_b200.surrogate.build()): the tensor-core kernels of the MLP
 * that pre-screens parameter-search candidates, and the search-side feature
 * and scoring kernels.  An addition of this project: DENSE's search scores
 * every candidate by simulating it (search/sres.cpp:328-345), so no DENSE
 * interface is replaced here.
 *
 * Every pointer argument is device memory unless stated; `stream` is a
 * cudaStream_t (NULL: the legacy default stream).  Every function returns
 * 0 when its kernels were launched, 1 when an argument is refused (before
 * any CUDA call), 2 on a launch error.  Matrices are row-major with the
 * given leading dimensions (elements).  BF16 arguments are void*. */
#ifndef DENSE_B200_SURROGATE_H
#define DENSE_B200_SURROGATE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Epilogues of the GEMM. */
enum {
  DENSE_MLP_EPI_STORE = 0,     /* D = A . B^T (FP32) */
  DENSE_MLP_EPI_BIAS_GELU = 1, /* D = A . B^T + bias (FP32), H = GELU(D) (BF16) */
  DENSE_MLP_EPI_BIAS = 2       /* D = A . B^T + bias (FP32) */
};

/* D[M][N] = A[M][K] . B[N][K]^T on the tcgen05 tensor cores, BF16 inputs,
 * FP32 accumulation.  M a positive multiple of 128, N a multiple of 16 in
 * [16, 256], K a positive multiple of 64; lda, ldb, ldh multiples of 8,
 * ldd of 4; bias (N floats) for the bias epilogues, H for GELU.  `err`
 * (one device int) collects error bits: 1 = a bounded wait gave up. */
int dense_mlp_gemm(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K,
                   int epilogue, const float* bias, void* H, int ldh, int* err, void* stream);

/* The same with a split-K workspace: `ws` (ws_bytes, 16-byte aligned)
 * holds FP32 partials when K is split across SMs (few 128-row tiles and
 * K >= 512); calls sharing a workspace must be ordered on one stream. */
int dense_mlp_gemm_ws(const void* A, int lda, const void* B, int ldb, float* D, int ldd, int M, int N, int K,
                      int epilogue, const float* bias, void* H, int ldh, int* err, float* ws, size_t ws_bytes,
                      void* stream);

/* BF16 copies: dst[c][r] = src[r][c] (transpose), and FP32 -> BF16
 * (optionally transposed into [cols][rows]). */
int dense_mlp_transpose_bf16(const void* src, int rows, int cols, int lds, void* dst, int ldd, void* stream);
int dense_mlp_cast_bf16(const float* src, int rows, int cols, void* dst, int transpose, void* stream);

/* dZ = dH * GELU'(Z) over n elements, FP32 and BF16 copies. */
int dense_mlp_gelu_backward(const float* dH, const float* Z, int64_t n, float* dZ, void* dZb, void* stream);

/* Masked squared error over the first nout of ldy outputs: loss (one
 * device float) += sum mask (Y - T)^2 * inv_count; dY = 2 mask (Y - T) *
 * inv_count in FP32 and BF16.  _dev reads inv_count from device memory. */
int dense_mlp_mse(const float* Y, int ldy, const float* T, const float* mask, int rows, int nout, float inv_count,
                  float* dY, void* dYb, float* loss, void* stream);
int dense_mlp_mse_dev(const float* Y, int ldy, const float* T, const float* mask, int rows, int nout,
                      const float* inv_count_dev, float* dY, void* dYb, float* loss, void* stream);

/* One training batch from a device-resident training set: rows idx[0..B)
 * of X [n_rows][n_in] to BF16 Xb [Bp][in_pad] (zero padded), of T and mask
 * [n_rows][n_out] to Tb and Mb [Bp][n_out]; rows B..Bp-1 are zeros. */
int dense_mlp_gather(const float* X, int n_rows, int n_in, const float* T, const float* mask, int n_out,
                     const int* idx, int B, int Bp, void* Xb, int in_pad, float* Tb, float* Mb, void* stream);

/* db[c] = sum over rows of dZ[r][c], in a fixed order (deterministic). */
int dense_mlp_colsum(const float* dZ, int rows, int cols, float* db, void* stream);

/* Adam with bias correction over n weights; _dev reads {lr, b1, b2, eps,
 * 1 - b1^t, 1 - b2^t} from device memory (for captured graphs). */
int dense_mlp_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                   int step, void* stream);
int dense_mlp_adam_dev(float* w, const float* g, float* m, float* v, int64_t n, const float* hyper, void* stream);

/* Mean pairwise Pearson correlation across the cells of each set's
 * trajectory X[set][t][cell] (cells contiguous, at most 1024; t <
 * counts[set]); NaN when fewer than two cells have a non-constant trace. */
int dense_features_synchrony(const double* X, int64_t set_stride, int64_t sample_stride, int cells,
                             const int* counts, int n_sets, double* out, void* stream);

/* Network inputs of candidates P[n][ldp] (FP64 parameters): BF16
 * log(P[r][idx[j]] / tmpl[j]) / log_spread for j < k, zero padded to
 * [Bp][in_pad]. */
int dense_features_encode(const double* P, int ldp, int n, const int* idx, const double* tmpl, int k,
                          double log_spread, void* Xb, int in_pad, int Bp, void* stream);

/* acc[n][nout] = Y (first != 0) or acc + Y, FP32. */
int dense_features_ensemble_accumulate(const float* Y, int ldy, int n, int nout, float* acc, int first,
                                       void* stream);

/* Ranking score per candidate from the ensemble sum acc[n][nout] of
 * `nets` networks (outputs: log period, log amplitude, synchrony,
 * oscillation indicator, acceptance indicator); mu and sd (nout floats,
 * HOST arrays) undo the outputs' standardisation:
 *   y4 + weight * (-|exp(y0) - period| / tol
 *                  + 0.5 clamp((y1 - log amp_min) / ramp + 0.5, 0, 1) + 0.5 clamp(y3, 0, 1)). */
int dense_features_score(const float* acc, int n, int nout, int nets, const float* mu, const float* sd, double weight,
                         double period, double tol, double amp_min, double ramp, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DENSE_B200_SURROGATE_H */
