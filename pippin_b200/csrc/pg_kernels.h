// Host-visible launchers of the device kernels (pg_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "pg_model.h"

namespace pg {

enum { K_STEP = 0, K_FORWARD = 1, K_SET_CONST = 2, K_POSES = 3 };

struct LaunchCfg {
  int G;                // lanes per environment (8, 16, 32)
  int tiles_per_block;  // environments resident per block
  int blocks;           // persistent grid size
};

const void* tile_kernel(int which, int G);
cudaError_t launch_step(const StepArgs& a, const LaunchCfg& c, cudaStream_t s);
cudaError_t launch_forward(const StepArgs& a, const LaunchCfg& c, double* dbg, int dbg_stride, int maxcon_out,
                           cudaStream_t s);
cudaError_t launch_set_const(const StepArgs& a, const LaunchCfg& c, const int* envs, int n, cudaStream_t s);
cudaError_t launch_poses(const StepArgs& a, const LaunchCfg& c, float* geoms, float* cams, cudaStream_t s);
cudaError_t launch_reset(const StepArgs& a, const int64_t* ids, int n, cudaStream_t s);

}  // namespace pg
