// Kernel launchers of the per-precision translation units.
#ifndef DENSE_B200_ENGINE_LAUNCH_HPP
#define DENSE_B200_ENGINE_LAUNCH_HPP

#include <cuda_runtime.h>

#include "engine_types.hpp"

namespace dense_b200 {
cudaError_t launch_init_fp64(const StepArgs& a, const double* init_conc, const int* init_status, cudaStream_t s);
cudaError_t launch_step_fp64(const StepArgs& a, const int* set_list, int n_sets, size_t smem, cudaStream_t s);
cudaError_t launch_step_mem_fp64(const StepArgs& a, const int* set_list, int n_sets, int block, cudaStream_t s);
cudaError_t launch_step_wave_fp64(const StepArgs& a, const int* set_list, int n_sets, int block, int smem,
                                  int all_shared, cudaStream_t s);
cudaError_t launch_import_fp64(const StepArgs& a, int set, const double* samples, int num_samples, double time_start,
                               cudaStream_t s);
cudaError_t launch_import_fp32(const StepArgs& a, int set, const double* samples, int num_samples, double time_start,
                               cudaStream_t s);
cudaError_t launch_init_fp32(const StepArgs& a, const double* init_conc, const int* init_status, cudaStream_t s);
cudaError_t launch_step_fp32(const StepArgs& a, const int* set_list, int n_sets, size_t smem, cudaStream_t s);
cudaError_t launch_step_mem_fp32(const StepArgs& a, const int* set_list, int n_sets, int block, cudaStream_t s);
cudaError_t launch_step_wave_fp32(const StepArgs& a, const int* set_list, int n_sets, int block, int smem,
                                  int all_shared, cudaStream_t s);
}  // namespace dense_b200

#endif
