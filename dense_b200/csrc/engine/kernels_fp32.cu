// FP32 step kernel: the model is compiled with Real = float (DENSE's Real
// is configurable the same way, utility/configurable.hpp:30-45) and the
// state update is Kahan-compensated.  Analyses still run in FP64.
#define DENSE_B200_REAL float
#include "dense_model_api.hpp"
#include "reaction_deltas.hpp"
#include "model_impl.hpp"
#include "step_kernel.cuh"

DENSE_B200_DEFINE_LAUNCHERS(fp32, float, true)
