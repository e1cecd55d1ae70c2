// Kernels of the batched FP64 physics backend.
//
// step_kernel is persistent: a grid sized to the GPU's resident capacity,
// each tile of G lanes pops environment indices from a device work counter
// (one atomicAdd per env; nothing ever waits on another tile, so no spin
// can hang) and runs all `nstep` substeps of that env with its state held
// in shared memory. Envs with many contacts or Newton iterations hold only
// their own tile, never a whole block or the grid. Each block first copies
// the model (a few KB) into its shared memory, so the tree walks and the
// narrow phase read topology and constants at shared-memory latency.
#include <cuda_runtime.h>

#include "pg_kernels.h"
#include "pg_newton.cuh"

namespace pg {

// Copy the model arena into shared memory and rebase the DModel pointers
// (when the launch asked for it); returns the model the block should read.
__device__ inline const DModel& stage_model(const StepArgs& A, unsigned char* sm) {
  if (!A.stage_model) return A.m;
  DModel* dm = reinterpret_cast<DModel*>(sm);
  unsigned char* arena = sm + (sizeof(DModel) + 15) / 16 * 16;
  const int4* src = reinterpret_cast<const int4*>(A.m.arena);
  int4* dst = reinterpret_cast<int4*>(arena);
  int n16 = (A.m.arena_bytes + 15) / 16;
  for (int i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
  if (threadIdx.x == 0) {
    *dm = A.m;
    uintptr_t base = reinterpret_cast<uintptr_t>(A.m.arena);
    for (int k = 0; k < A.n_ptr; k++) {
      uintptr_t* f = reinterpret_cast<uintptr_t*>(reinterpret_cast<unsigned char*>(dm) + A.ptr_off[k]);
      if (*f >= base && *f < base + (uintptr_t)A.m.arena_bytes) *f = reinterpret_cast<uintptr_t>(arena) + (*f - base);
    }
    dm->arena = arena;
  }
  __syncthreads();
  return *dm;
}

__device__ inline double* tile_workspace(const StepArgs& A, unsigned char* sm, int tib) {
  int off = A.stage_model ? staged_model_bytes(A.m.arena_bytes) : 0;
  return reinterpret_cast<double*>(sm + off) + (size_t)tib * A.w.stride;
}

// forward.rs:336-389: one substep of one env, state in the tile workspace
template <int G>
__device__ void substep(const Tile<G>& T, const DModel& m, const StepArgs& A, const EnvCtx& e, int* status,
                        int* iters, int* ncon_out, int* nrows_out) {
  const WsLayout& w = A.w;
  const ScrLayout& s = A.s;
  int lane = T.lane(), nv = m.nv;
  double* ws = e.ws;
  double h = m.timestep;

  tree_down(T, m, w, e, true, e.scr + s.geoms);
  tree_up(T, m, w, e, true);
  passive_actuation(T, m, w, e);
  int ncon = collide(T, m, w, s, e, status);
  *ncon_out = ncon;

  double* smooth = ws + w.smooth;
  double* acc = ws + w.acc;
  for (int k = lane; k < nv; k += G) {
    smooth[k] = ws[w.passive + k] + ws[w.actf + k] + ws[w.applied + k] - ws[w.bias + k];
    acc[k] = smooth[k];
  }
  T.sync();
  // the tree region is dead from here on: factorisations and Newton use it
  bool damped = has_implicit_terms(m, e.prm);
  if (!factor_mass(T, m, w, e, 0.0)) {
    *status |= ST_NOT_SPD;
    return;
  }
  solve_blocks(T, ws + w.fac, nv, nv, m.nblock, m.block_adr, m.dof_block, m.maxbs, ws + w.rinv, acc);
  int nr = build_rows(T, m, w, s, e, ncon, status);
  *nrows_out = nr;
  const double* warm = A.warm_mode == WARM_COLD ? nullptr : ws + w.qacc;
  *iters = newton_solve(T, m, w, s, e, nr, acc, warm);
  if (damped) {
    if (!factor_mass(T, m, w, e, h)) {
      *status |= ST_NOT_SPD;
      return;
    }
    for (int k = lane; k < nv; k += G) acc[k] = smooth[k] + ws[w.qfrc_c + k];
    T.sync();
    solve_blocks(T, ws + w.fac, nv, nv, m.nblock, m.block_adr, m.dof_block, m.maxbs, ws + w.rinv, acc);
  }
  double* v = ws + w.vel;
  double* qvel = ws + w.qvel;
  for (int k = lane; k < nv; k += G) {
    double vk = qvel[k] + h * acc[k];
    v[k] = vk;
    ws[w.qacc + k] = (vk - qvel[k]) / h;
  }
  T.sync();
  integrate_pos(T, m, ws + w.qpos, v, h);
  for (int k = lane; k < nv; k += G) qvel[k] = v[k];
  T.sync();
}

template <int G>
__device__ void load_env(const Tile<G>& T, const DModel& m, const StepArgs& A, const EnvCtx& e) {
  const WsLayout& w = A.w;
  int lane = T.lane();
  size_t env = e.env;
  for (int k = lane; k < m.nq; k += G) e.ws[w.qpos + k] = A.st.qpos[env * m.nq + k];
  for (int k = lane; k < m.nv; k += G) {
    e.ws[w.qvel + k] = A.st.qvel[env * m.nv + k];
    e.ws[w.qacc + k] = A.st.qacc[env * m.nv + k];
    e.ws[w.applied + k] = A.st.applied[env * m.nv + k];
  }
  for (int k = lane; k < m.nu; k += G) e.ws[w.ctrl + k] = A.st.ctrl[env * m.nu + k];
  T.sync();
}

template <int G>
__device__ void store_env(const Tile<G>& T, const DModel& m, const StepArgs& A, const EnvCtx& e) {
  const WsLayout& w = A.w;
  int lane = T.lane();
  size_t env = e.env;
  for (int k = lane; k < m.nq; k += G) A.st.qpos[env * m.nq + k] = e.ws[w.qpos + k];
  for (int k = lane; k < m.nv; k += G) {
    A.st.qvel[env * m.nv + k] = e.ws[w.qvel + k];
    A.st.qacc[env * m.nv + k] = e.ws[w.qacc + k];
  }
  for (int k = lane; k < m.nu; k += G) A.st.ctrl[env * m.nu + k] = e.ws[w.ctrl + k];
}

// pops the next work item for the tile (one atomic per env)
template <int G>
__device__ inline int next_item(const Tile<G>& T, int* queue) {
  int item = 0;
  if (T.lane() == 0) item = atomicAdd(queue, 1);
  return T.bcast(item, 0);
}

template <int G>
__global__ void __launch_bounds__(256) step_kernel(const __grid_constant__ StepArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DModel& m = stage_model(A, smem);
  cg::thread_block block = cg::this_thread_block();
  Tile<G> T(cg::tiled_partition<G>(block));
  int tib = threadIdx.x / G;
  size_t gtile = (size_t)blockIdx.x * (blockDim.x / G) + tib;
  EnvCtx e;
  e.ws = tile_workspace(A, smem, tib);
  e.scr = A.scratch + gtile * (size_t)A.s.stride;
  for (;;) {
    int item = next_item(T, A.queue);
    if (item >= A.count) break;
    e.env = A.start + item;
    e.prm = A.st.params + (size_t)e.env * m.pstride;
    load_env(T, m, A, e);
    int status = 0, iters = 0, ncon = 0, nrows = 0;
    for (int sidx = 0; sidx < A.nstep; sidx++) {
      if (A.ctrl_seq) {
        for (int k = T.lane(); k < m.nu; k += G)
          e.ws[A.w.ctrl + k] = A.ctrl_seq[((size_t)item * A.nstep + sidx) * m.nu + k];
        T.sync();
      }
      substep(T, m, A, e, &status, &iters, &ncon, &nrows);
      if (A.qpos_out)
        for (int k = T.lane(); k < m.nq; k += G)
          A.qpos_out[((size_t)item * A.nstep + sidx) * m.nq + k] = e.ws[A.w.qpos + k];
      if (status & ST_NOT_SPD) break;
    }
    store_env(T, m, A, e);
    if (T.lane() == 0) {
      A.st.iters[e.env] = iters;
      A.st.ncon[e.env] = ncon;
      A.st.nrows[e.env] = nrows;
      A.st.status[e.env] = status;
    }
    T.sync();
  }
}

// Forward pass only (forward.rs:263-271) for diagnostics: writes M, bias
// and the contact list of each env to `dbg`.
template <int G>
__global__ void __launch_bounds__(256) forward_kernel(const __grid_constant__ StepArgs A, double* dbg, int dbg_stride,
                                                      int maxcon_out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DModel& m = stage_model(A, smem);
  cg::thread_block block = cg::this_thread_block();
  Tile<G> T(cg::tiled_partition<G>(block));
  int tib = threadIdx.x / G;
  size_t gtile = (size_t)blockIdx.x * (blockDim.x / G) + tib;
  EnvCtx e;
  e.ws = tile_workspace(A, smem, tib);
  e.scr = A.scratch + gtile * (size_t)A.s.stride;
  for (;;) {
    int item = next_item(T, A.queue);
    if (item >= A.count) break;
    e.env = A.start + item;
    e.prm = A.st.params + (size_t)e.env * m.pstride;
    load_env(T, m, A, e);
    int status = 0;
    tree_down(T, m, A.w, e, true, e.scr + A.s.geoms);
    tree_up(T, m, A.w, e, true);
    passive_actuation(T, m, A.w, e);
    int ncon = collide(T, m, A.w, A.s, e, &status);
    double* out = dbg + (size_t)item * dbg_stride;
    int nv = m.nv;
    for (int k = T.lane(); k < nv * nv; k += G) out[k] = e.ws[A.w.qm + k];
    for (int k = T.lane(); k < nv; k += G) out[nv * nv + k] = e.ws[A.w.bias + k];
    if (T.lane() == 0) out[nv * nv + nv] = ncon;
    const double* con = e.scr + A.s.contacts;
    for (int t = T.lane(); t < ncon * 13 && t < maxcon_out * 13; t += G) {
      int c = t / 13, f = t % 13;
      out[nv * nv + nv + 1 + t] = con[C_STRIDE * c + f];
    }
    T.sync();
  }
}

// forward.rs:275-333: invweight0 of each env's model at its reset state
template <int G>
__global__ void __launch_bounds__(256) set_const_kernel(const __grid_constant__ StepArgs A, const int* envs, int n) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DModel& m = stage_model(A, smem);
  cg::thread_block block = cg::this_thread_block();
  Tile<G> T(cg::tiled_partition<G>(block));
  int tib = threadIdx.x / G;
  size_t gtile = (size_t)blockIdx.x * (blockDim.x / G) + tib;
  const WsLayout& w = A.w;
  EnvCtx e;
  e.ws = tile_workspace(A, smem, tib);
  e.scr = A.scratch + gtile * (size_t)A.s.stride;
  int nv = m.nv;
  for (;;) {
    int item = next_item(T, A.queue);
    if (item >= n) break;
    e.env = envs ? envs[item] : A.start + item;
    double* prm = A.st.params + (size_t)e.env * m.pstride;
    e.prm = prm;
    for (int k = T.lane(); k < m.nq; k += G) e.ws[w.qpos + k] = prm[m.p_qpos_reset + k];
    T.sync();
    tree_down(T, m, w, e, false, nullptr);
    tree_up(T, m, w, e, false);
    if (nv == 0) continue;
    // M^-1 by Cholesky of the full matrix (forward.rs:286-288); the factor
    // lives in scratch because the workspace's tree region is still needed
    double* L = e.scr + A.s.chol;
    double* rinv = e.ws + w.rinv;
    for (int t = T.lane(); t < nv * nv; t += G) L[t] = e.ws[w.qm + t];
    T.sync();
    bool ok = chol_blocks(T, L, nv, nv, 1, nullptr, nullptr, nv, rinv);
    // one right-hand side per lane: unit vectors, then per body 3 axes x
    // (translation, rotation) rows; x = M^-1 row, quad = row . x
    double* xs = e.scr + A.s.jac;  // [rhs][nv]
    int nrhs = nv + 6 * m.nbody;
    double* quad = e.scr + A.s.rows;  // [nrhs]
    if (ok) {
      for (int r = T.lane(); r < nrhs; r += G) {
        double* x = xs + (size_t)r * nv;
        double* row = xs + (size_t)(nrhs + (r % G)) * nv;  // per-lane copy of the row
        for (int k = 0; k < nv; k++) row[k] = 0.0;
        if (r < nv) {
          row[r] = 1.0;
        } else {
          int q = r - nv;
          int b = q / 6, axis = (q % 6) / 2, kind = q % 2;
          if (b == 0) {
            quad[r] = 0.0;
            continue;
          }
          V3 dir{axis == 0 ? 1.0 : 0.0, axis == 1 ? 1.0 : 0.0, axis == 2 ? 1.0 : 0.0};
          V3 xip = ld3(e.ws + w.xpos + 3 * b) + mv(ld9(e.ws + w.xmat + 9 * b), ld3(prm + m.p_ipos + 3 * b));
          for (int k = m.body_lastdof[b]; k != -1; k = m.dof_parent[k]) {
            Sp c = ld6(e.ws + w.cdof + 6 * k);
            row[k] = kind == 0 ? dot(dir, point_vel(c, xip)) : dot(dir, c.ang);
          }
        }
        for (int k = 0; k < nv; k++) x[k] = row[k];
        for (int i = 0; i < nv; i++) x[i] = (x[i] - dot_ref(L + i * nv, 1, x, 1, i)) / L[i * nv + i];
        for (int i = nv - 1; i >= 0; i--) {
          x[i] /= L[i * nv + i];
          double xi = -x[i];
          for (int k = 0; k < i; k++) x[k] += xi * L[i * nv + k];
        }
        double sacc = 0.0;
        for (int k = 0; k < nv; k++) sacc += row[k] * x[k];
        quad[r] = sacc;
      }
    }
    T.sync();
    if (T.lane() == 0) {
      double* dw = prm + m.p_dof_invw;
      double* bw = prm + m.p_body_invw;
      for (int k = 0; k < nv; k++) dw[k] = ok ? quad[k] : 0.0;
      for (int b = 0; b < 2 * m.nbody; b++) bw[b] = 0.0;
      if (ok) {
        for (int j = 0; j < m.njnt; j++) {
          int da = m.jnt_dofadr[j];
          int ngrp = m.jnt_type[j] == JNT_FREE ? 2 : (m.jnt_type[j] == JNT_BALL ? 1 : 0);
          for (int gi = 0; gi < ngrp; gi++) {
            int g0 = da + 3 * gi;
            double avg = (dw[g0] + dw[g0 + 1] + dw[g0 + 2]) / 3.0;
            dw[g0] = dw[g0 + 1] = dw[g0 + 2] = avg;
          }
        }
        for (int b = 1; b < m.nbody; b++) {
          double wt[2] = {0.0, 0.0};
          for (int axis = 0; axis < 3; axis++)
            for (int kind = 0; kind < 2; kind++) wt[kind] += quad[nv + 6 * b + 2 * axis + kind] / 3.0;
          bw[2 * b] = wt[0];
          bw[2 * b + 1] = wt[1];
        }
      }
    }
    T.sync();
  }
}

// Geom and camera poses (f32 Pose = pos[3], row-major mat[9]) from qpos,
// as the reference's poses() reads them after its closing kinematics pass
// (crates/pippin-env/src/pippin_cpu.rs:189-205).
template <int G>
__global__ void __launch_bounds__(256) poses_kernel(const __grid_constant__ StepArgs A, float* geoms, float* cams) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DModel& m = stage_model(A, smem);
  cg::thread_block block = cg::this_thread_block();
  Tile<G> T(cg::tiled_partition<G>(block));
  int tib = threadIdx.x / G;
  size_t gtile = (size_t)blockIdx.x * (blockDim.x / G) + tib;
  const WsLayout& w = A.w;
  EnvCtx e;
  e.ws = tile_workspace(A, smem, tib);
  e.scr = A.scratch + gtile * (size_t)A.s.stride;
  double* gr = e.scr + A.s.geoms;
  for (;;) {
    int item = next_item(T, A.queue);
    if (item >= A.count) break;
    e.env = A.start + item;
    e.prm = A.st.params + (size_t)e.env * m.pstride;
    for (int k = T.lane(); k < m.nq; k += G) e.ws[w.qpos + k] = A.st.qpos[(size_t)e.env * m.nq + k];
    T.sync();
    tree_down(T, m, w, e, false, gr);
    for (int g = T.lane(); g < m.ngeom; g += G) {
      float* o = geoms + ((size_t)item * m.ngeom + g) * 12;
      for (int a = 0; a < 12; a++) o[a] = (float)gr[G_STRIDE * g + a];
    }
    for (int c = T.lane(); c < m.ncam; c += G) {
      int b = m.cam_body[c];
      M3 xm = ld9(e.ws + w.xmat + 9 * b);
      V3 pos = ld3(e.ws + w.xpos + 3 * b) + mv(xm, ld3(m.cam_pos + 3 * c));
      M3 mat = mm(xm, q_mat(ld4(m.cam_quat + 4 * c)));
      float* o = cams + ((size_t)item * m.ncam + c) * 12;
      for (int a = 0; a < 3; a++) o[a] = (float)comp(pos, a);
      for (int a = 0; a < 9; a++) o[3 + a] = (float)mat.m[a];
    }
    T.sync();
  }
}

// data.rs:122-131: qpos <- per-env reset state, zero qvel/ctrl/applied,
// drop the PGS warm start; qacc (the Newton warm start) is kept.
__global__ void reset_kernel(const __grid_constant__ StepArgs A, const int64_t* ids, int n) {
  const DModel& m = A.m;
  int width = m.nq + 2 * m.nv + m.nu;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)n * width;
       t += (size_t)gridDim.x * blockDim.x) {
    size_t env = ids[t / width];
    int f = (int)(t % width);
    if (f < m.nq) {
      A.st.qpos[env * m.nq + f] = A.st.params[env * m.pstride + m.p_qpos_reset + f];
    } else if ((f -= m.nq) < m.nv) {
      A.st.qvel[env * m.nv + f] = 0.0;
    } else if ((f -= m.nv) < m.nu) {
      A.st.ctrl[env * m.nu + f] = 0.0;
    } else {
      f -= m.nu;
      A.st.applied[env * m.nv + f] = 0.0;
      if (f == 0 && A.st.prev_ncon) A.st.prev_ncon[env] = 0;
    }
  }
}

// ---------------------------------------------------------------- launchers
template <int G>
static const void* kernel_ptr(int which) {
  switch (which) {
    case K_STEP: return (const void*)step_kernel<G>;
    case K_FORWARD: return (const void*)forward_kernel<G>;
    case K_SET_CONST: return (const void*)set_const_kernel<G>;
    case K_POSES: return (const void*)poses_kernel<G>;
  }
  return nullptr;
}

const void* tile_kernel(int which, int G) {
  switch (G) {
    case 8: return kernel_ptr<8>(which);
    case 16: return kernel_ptr<16>(which);
    case 32: return kernel_ptr<32>(which);
  }
  return nullptr;
}

size_t block_smem(const StepArgs& a, const LaunchCfg& c) {
  return (a.stage_model ? (size_t)staged_model_bytes(a.m.arena_bytes) : 0) +
         (size_t)c.tiles_per_block * a.w.stride * sizeof(double);
}

#define PG_LAUNCH(KERNEL, ...)                                                      \
  do {                                                                              \
    size_t smem = block_smem(a, c);                                                 \
    dim3 grid(c.blocks), block(c.tiles_per_block * c.G);                           \
    switch (c.G) {                                                                  \
      case 8: KERNEL<8><<<grid, block, smem, s>>>(__VA_ARGS__); break;              \
      case 16: KERNEL<16><<<grid, block, smem, s>>>(__VA_ARGS__); break;            \
      case 32: KERNEL<32><<<grid, block, smem, s>>>(__VA_ARGS__); break;            \
      default: return cudaErrorInvalidValue;                                        \
    }                                                                               \
    return cudaGetLastError();                                                      \
  } while (0)

cudaError_t launch_step(const StepArgs& a, const LaunchCfg& c, cudaStream_t s) { PG_LAUNCH(step_kernel, a); }

cudaError_t launch_forward(const StepArgs& a, const LaunchCfg& c, double* dbg, int dbg_stride, int maxcon_out,
                           cudaStream_t s) {
  PG_LAUNCH(forward_kernel, a, dbg, dbg_stride, maxcon_out);
}

cudaError_t launch_set_const(const StepArgs& a, const LaunchCfg& c, const int* envs, int n, cudaStream_t s) {
  PG_LAUNCH(set_const_kernel, a, envs, n);
}

cudaError_t launch_poses(const StepArgs& a, const LaunchCfg& c, float* geoms, float* cams, cudaStream_t s) {
  PG_LAUNCH(poses_kernel, a, geoms, cams);
}

cudaError_t launch_reset(const StepArgs& a, const int64_t* ids, int n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  int width = a.m.nq + 2 * a.m.nv + a.m.nu;
  size_t total = (size_t)n * width;
  int threads = 256;
  int blocks = (int)((total + threads - 1) / threads);
  if (blocks > 4096) blocks = 4096;
  reset_kernel<<<blocks, threads, 0, s>>>(a, ids, n);
  return cudaGetLastError();
}

}  // namespace pg
