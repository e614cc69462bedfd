/* A caller of the C ABI in plain C (also compiled as C++): model facts and
   a batch plan, the entry points that need no GPU.  Prints one line. */
#include <stdint.h>
#include <stdio.h>

#include "dense_b200.h"

int main(void) {
  dense_model_info info;
  if (dense_model_get_info(&info) != DENSE_OK) return 1;
  /* a 4-cell ring tissue: each cell's neighbours in ascending order */
  int off[5] = {0, 2, 4, 6, 8};
  int ids[8] = {1, 3, 0, 2, 1, 3, 0, 2};
  double params[256];
  for (int i = 0; i < info.num_params && i < 256; ++i) params[i] = 1.0;
  dense_set_desc set = {4, off, ids, params, NULL, NULL, NULL, 10.0, 0, 0};
  dense_run_desc run = {DENSE_FP64, 0.01, 0.1, 0, NULL, 0};
  int64_t bytes = 0;
  int kernel = -1, levels = -1;
  if (dense_engine_plan(&run, 1, &set, &bytes, &kernel, &levels) != DENSE_OK) {
    printf("plan failed: %s\n", dense_last_error());
    return 2;
  }
  /* a malformed set is refused with a code and a message */
  ids[1] = 9;
  int rc = dense_engine_plan(&run, 1, &set, NULL, NULL, NULL);
  printf("%d %d %s %lld %d %d %d %s\n", info.num_species, info.num_params, dense_model_specie_name(0),
         (long long)bytes, kernel, levels, rc, dense_last_error());
  return 0;
}
