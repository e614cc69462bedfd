// Host-side check of the persistent GEMM's shared-memory layout
// (persistent_smem in csrc/surrogate/umma_gemm_persistent.cuh) for the
// surrogate's shapes and the split-K / column-block forms: every layout
// fits the budget it was given, keeps the 1024-byte alignment the swizzled
// staging boxes need, has at least the stated ring depth, and prefers B
// resident where it fits.  Prints one line per case; exit 1 on a failure.
#include <cstdio>

#include "umma_gemm_persistent.cuh"

using namespace dense_b200::mlp;

static int fails = 0;

static void check(int M, int N, int K, int epi, int splits, int nsplit, size_t limit, bool expect_resident) {
  PersistentArgs a{};
  a.M = M;
  a.N = N;
  a.K = K;
  a.tiles = M / kTileM;
  a.splits = splits;
  a.nsplit = nsplit;
  a.n_blk = N / nsplit;
  a.chunks_per_split = (K / kChunkK + splits - 1) / splits;
  const size_t smem = persistent_smem(a, epi, limit);
  const size_t per_buf = kStageD + (epi == kEpiBiasGelu ? kStageH : 0);
  const size_t staging = static_cast<size_t>(kEpiWarps) * a.out_bufs * per_buf;
  bool ok = smem > 0 && smem <= limit;
  ok = ok && smem == a.b_bytes + static_cast<size_t>(a.stages) * a.stage_bytes + staging + 1024;
  ok = ok && a.b_bytes % 1024 == 0 && a.stage_bytes % 1024 == 0 && per_buf % 1024 == 0;
  ok = ok && a.stages >= (a.resident_b ? 3 : 2) && a.stages <= kMaxStages;
  ok = ok && (a.out_bufs == 1 || a.out_bufs == 2);
  ok = ok && (a.resident_b != 0) == expect_resident;
  std::printf("%s M=%d N=%d K=%d epi=%d splits=%d nsplit=%d smem=%zu resident=%d stages=%d bufs=%d\n",
              ok ? "ok" : "FAIL", M, N, K, epi, splits, nsplit, smem, a.resident_b, a.stages, a.out_bufs);
  if (!ok) ++fails;
}

int main() {
  // 227 KB per block less the kernel's static shared memory (at most 2 KB)
  const size_t limit = 232448 - 2048;
  for (int epi = 0; epi < 3; ++epi) {
    check(131072, 256, 64, epi, 1, 1, limit, true);    // first layer
    check(131072, 256, 256, epi, 1, 1, limit, true);   // hidden layers (B 128 KB)
    check(131072, 128, 256, epi, 1, 1, limit, true);   // output layer
    check(2048, 256, 256, epi, 1, 4, limit, false);    // column blocks stream B
    check(256, 256, 4096, epi, 16, 1, limit, false);   // split-K weight gradients
    check(128, 64, 8192, epi, 32, 1, limit, false);
    check(40960, 256, 512, epi, 1, 1, limit, false);   // B of 256 KB streams
    check(128, 32, 64, epi, 1, 1, limit, true);
  }
  return fails ? 1 : 0;
}
