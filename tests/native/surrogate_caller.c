/* A native caller of the surrogate library through
 * include/dense_b200_surrogate.h: argument checks that need no GPU. */
#include <stdio.h>

#include "dense_b200_surrogate.h"

int main(void) {
  static double buf[8] = {0};
  void* p = buf; /* never dereferenced: every call below is refused first */
  int refused = 0;
  refused += dense_mlp_gemm(p, 64, p, 64, (float*)p, 64, 100, 64, 64, DENSE_MLP_EPI_STORE, NULL, NULL, 0,
                            (int*)p, NULL) == 1;
  refused += dense_mlp_gemm_ws(p, 64, p, 64, (float*)p, 64, 128, 64, 64, DENSE_MLP_EPI_BIAS, NULL, NULL, 0,
                               (int*)p, NULL, 0, NULL) == 1;
  refused += dense_features_synchrony((const double*)p, 0, 0, 4096, (const int*)p, 1, (double*)p, NULL) == 1;
  refused += dense_mlp_adam_dev((float*)p, (const float*)p, (float*)p, (float*)p, 8, NULL, NULL) == 1;
  printf("%d\n", refused);
  return refused == 4 ? 0 : 1;
}
