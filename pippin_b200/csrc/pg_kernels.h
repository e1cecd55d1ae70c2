// Host-visible launchers of the device kernels (pg_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include "pg_model.h"

namespace pg {

// tile kernels (one env per tile of G lanes, persistent over a work counter)
enum { K_SMOOTH = 0, K_COLLIDE = 1, K_NEWTON = 2, K_SET_CONST = 3, K_POSES = 4, K_NEWTON_PLAIN = 5, K_COUNT = 6 };

struct LaunchCfg {
  int G;                // lanes per environment (8, 16, 32)
  int tiles_per_block;  // environments resident per block
  int blocks;           // persistent grid size
};

// launch shapes of the three phases of a substep
struct SubstepCfg {
  LaunchCfg smooth, collide, newton;
};

const void* tile_kernel(int which, int G);
// shared bytes per block of kernel `which` for the given tiles per block
size_t kernel_smem(int which, const StepArgs& a, int tiles_per_block);

// One substep of envs [a.start, a.start + a.count): counter reset, then the
// smooth-dynamics, collision and Newton phase kernels, in stream order.
cudaError_t launch_substep(const StepArgs& a, const SubstepCfg& c, cudaStream_t s);
cudaError_t launch_smooth_collide(const StepArgs& a, const SubstepCfg& c, cudaStream_t s);
// the pieces of launch_substep: the counter reset and one phase kernel
cudaError_t reset_queue(const StepArgs& a, cudaStream_t s);
// the learned start's features (and, with infer, its predictions) over the
// collision phase's contact list; learn_prepare allows the kernel its
// shared memory (once, before launches or captures)
cudaError_t launch_learn(const StepArgs& a, bool infer, cudaStream_t s);
cudaError_t learn_prepare();
cudaError_t launch_phase(int which, const StepArgs& a, const LaunchCfg& c, cudaStream_t s);
cudaError_t launch_set_const(const StepArgs& a, const LaunchCfg& c, const int* envs, int n, cudaStream_t s);
cudaError_t launch_poses(const StepArgs& a, const LaunchCfg& c, float* geoms, float* cams, cudaStream_t s);
cudaError_t launch_reset(const StepArgs& a, const int64_t* ids, int n, cudaStream_t s);
// params[e * pstride ..] takes values v[e][w] of parameter p, element id, for e < count
cudaError_t launch_apply_param(const DModel& d, double* params, int64_t count, int p, int64_t id, const double* v, int w,
                               int nq, cudaStream_t s);
// vertex[i] = the hull support walk of mesh `mesh` along dirs[i] (mesh frame; device memory)
cudaError_t launch_hull_support(const DModel& m, int mesh, const double* dirs, int n, int* vertex, cudaStream_t s);

}  // namespace pg
