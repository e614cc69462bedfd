// FP64 step kernel: the model is compiled with Real = double, and the file
// is built with --fmad=false so every multiply and add rounds on its own,
// as on DENSE's x86-64 build (no FMA contraction).
#define DENSE_B200_REAL double
#include "dense_model_api.hpp"
#include "reaction_deltas.hpp"
#include "model_impl.hpp"
#include "step_kernel.cuh"

DENSE_B200_DEFINE_LAUNCHERS(fp64, double, false)
