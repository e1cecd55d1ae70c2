// Kernels of the batched FP64 physics backend.
//
// A substep (crates/pippin/src/forward.rs:336-389) runs as three phase
// kernels over the env range, each small enough for the instruction cache:
//   smooth_kernel   kinematics, CRBA, RNE, passive and actuator forces, the
//                   factorisation of M and a0 = M^-1 f, and the factor of
//                   M + hD used at the end (the same control flow in every
//                   env, so the tiles of a warp stay in lockstep)
//   collide_kernel  broad and narrow phase
//   newton_kernel   constraint rows, Newton, implicit-damping solve,
//                   integration (the phase whose work varies per env)
// They hand data over in a per-env work record in HBM (it stays in L2 for
// batches of a few thousand envs). Every kernel is persistent: a grid sized
// to the GPU's resident capacity whose tiles of G lanes pop env indices from
// a device counter (one atomicAdd per env; no tile waits on another, so
// there is no spin to bound). Each block first copies the model (a few KB)
// into shared memory.
#include <cuda_runtime.h>

#include <algorithm>

#include "pg_kernels.h"
#include "pg_mlp.h"
#include "pg_pgs.cuh"

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

// shared memory of a collide tile: its queue of broad-phase survivors, with
// the edge query's two survivor lists behind it when the model has general
// pairs (ints); then the polytope cache (world vertices and face normals of
// both polytopes of a general pair) and the clip buffers (doubles)
__host__ __device__ inline int collide_tile_ints(const DModel& m) {
  return COLLIDE_QUEUE + (m.gen_vmax > 0 ? 2 * GEN_SURV_CAP : 0);
}
__host__ __device__ inline int collide_cache_doubles(const DModel& m) { return m.gen_cache + m.gen_clip; }

__device__ inline double* tile_workspace(const StepArgs& A, unsigned char* sm, int stride, int tib) {
  int off = A.stage_model ? staged_model_bytes(A.m.arena_bytes) : 0;
  return reinterpret_cast<double*>(sm + off) + (size_t)tib * stride;
}

// Work items of a persistent grid: a tile's first item is its own index in
// the grid; later ones come from the phase's counter (one atomic per env),
// offset by the tile count, and only when the grid has fewer tiles than
// items. A grid with a tile per item takes no atomics and no round trip to
// the counter before its first env or after its last.
template <int G>
__device__ inline int first_item() {
  return blockIdx.x * (blockDim.x / G) + threadIdx.x / G;
}
template <int G>
__device__ inline int next_item(const Tile<G>& T, int* queue, int count) {
  int ntiles = gridDim.x * (blockDim.x / G);
  if (ntiles >= count) return count;
  int item = 0;
  if (T.lane() == 0) item = atomicAdd(queue, 1);
  return ntiles + T.bcast(item, 0);
}

template <int G>
__device__ inline void copy_in(const Tile<G>& T, double* dst, const double* src, int n) {
  for (int k = T.lane(); k < n; k += G) dst[k] = src[k];
}

// ---------------------------------------------------------------- phase 1
// forward.rs:263-271 (minus collide) and forward.rs:342-356: smooth forces,
// a0 = M^-1 f, and the factor of M + hD (forward.rs:359-366) when damped.
template <int G>
__global__ void __launch_bounds__(256) smooth_kernel(const __grid_constant__ StepArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DModel& m = stage_model(A, smem);
  cg::thread_block block = cg::this_thread_block();
  Tile<G> T(cg::tiled_partition<G>(block));
  const WsLayout& w = A.w;
  EnvCtx e;
  e.ws = tile_workspace(A, smem, w.stride, threadIdx.x / G);
  e.scr = nullptr;
  e.con = nullptr;
  int nq = m.nq, nv = m.nv, nu = m.nu;
  double h = m.timestep;
  for (int item = first_item<G>(); item < A.count; item = next_item(T, A.queue + 0, A.count)) {
    size_t env = (size_t)A.start + item;
    e.env = (int)env;
    e.prm = A.st.params + env * m.pstride;
    double* wk = A.work + env * A.k.stride;
    e.geo = wk + A.k.geoms;
    double* ws = e.ws;
    prefetch_l1(T, e.prm, sizeof(double) * m.pstride);
    load_async(T, ws + w.qpos, A.st.qpos + env * nq, nq);
    load_async(T, ws + w.qvel, A.st.qvel + env * nv, nv);
    if (A.ctrl_seq) {
      const double* c = A.ctrl_seq + ((size_t)item * A.nstep + A.sidx) * nu;
      load_async(T, ws + w.ctrl, c, nu);
      copy_in(T, A.st.ctrl + env * nu, c, nu);  // rollout leaves the last controls in place
    } else {
      load_async(T, ws + w.ctrl, A.st.ctrl + env * nu, nu);
    }
    load_wait();
    T.sync();
    tree_down(T, m, w, e, true, e.geo);
    tree_up(T, m, w, e, true, wk + A.k.qm);  // M goes straight to the work record
    passive_actuation(T, m, w, e);
    double* smooth = ws + w.smooth;
    double* acc = ws + w.acc;
    const double* applied = A.st.applied + env * nv;
    for (int k = T.lane(); k < nv; k += G) {
      double f = ws[w.passive + k] + ws[w.actf + k] + applied[k] - ws[w.bias + k];
      smooth[k] = f;
      acc[k] = f;
      wk[A.k.bias + k] = ws[w.bias + k];
    }
    copy_in(T, wk + A.k.cdof, ws + w.cdof, 6 * nv);
    T.sync();
    // the tree region is dead from here on: the factorisations use it
    int status = 0;
    bool damped = has_implicit_terms(T, m, e.prm);
    // the factor of M + hD too: for the damped solve after Newton, and always
    // for PGS (forward.rs:366-368), which factors M + hD even with D = 0
    bool both = damped || m.solver == SOLVER_PGS;
    if (both ? factor_mass2(T, m, w, e, h, wk + A.k.qm) : factor_mass(T, m, w, e, 0.0, wk + A.k.qm)) {
      solve_auto(T, ws + w.fac, nv, nv, m.nblock, m.block_adr, m.dof_block, m.maxbs, ws + w.rinv, acc);
      copy_in(T, wk + A.k.a0, acc, nv);
      copy_in(T, wk + A.k.smooth, smooth, nv);
      if (both) {
        copy_in(T, wk + A.k.lh, ws + w.fac2, nv * nv);
        copy_in(T, wk + A.k.rinvh, ws + w.rinv2, nv);
      }
    } else {
      status |= ST_NOT_SPD;
    }
    if (T.lane() == 0) {
      wk[A.k.meta + K_META_STATUS] = status;
      wk[A.k.meta + K_META_DAMPED] = damped ? 1.0 : 0.0;
    }
    T.sync();
  }
}

// ---------------------------------------------------------------- phase 2
// forward.rs:214-260: broad and narrow phase over the candidate pairs
// two blocks of 256 threads an SM (128 registers a thread): the general
// narrow phase alone would take every register and halve the resident tiles
template <int G>
__global__ void __launch_bounds__(256, 2) collide_kernel(const __grid_constant__ StepArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DModel& m = stage_model(A, smem);
  cg::thread_block block = cg::this_thread_block();
  Tile<G> T(cg::tiled_partition<G>(block));
  EnvCtx e;
  e.ws = nullptr;
  e.scr = nullptr;
  // the tile's queue of broad-phase survivors (2G ints) and edge lists, then
  // its polytope cache and clip buffers
  int tpb = blockDim.x / G;
  int* queue = reinterpret_cast<int*>(tile_workspace(A, smem, 0, 0)) + (threadIdx.x / G) * collide_tile_ints(m);
  GenScratch gs{nullptr, nullptr, nullptr};
  if (m.gen_vmax > 0) {
    double* tile = reinterpret_cast<double*>(reinterpret_cast<int*>(tile_workspace(A, smem, 0, 0)) +
                                             tpb * collide_tile_ints(m)) +
                   (threadIdx.x / G) * collide_cache_doubles(m);
    gs.cache = m.gen_cache ? tile : nullptr;
    gs.clip = m.gen_clip ? tile + m.gen_cache : nullptr;
    gs.surv = queue + COLLIDE_QUEUE;
  }
  for (int item = first_item<G>(); item < A.count; item = next_item(T, A.queue + Q_COLLIDE, A.count)) {
    size_t env = (size_t)A.start + item;
    e.env = (int)env;
    e.prm = A.st.params + env * m.pstride;
    double* wk = A.work + env * A.k.stride;
    e.geo = wk + A.k.geoms;
    e.con = wk + A.k.contacts;
    prefetch_l1(T, e.prm, sizeof(double) * m.pstride);
    prefetch_l1(T, e.geo, sizeof(double) * G_STRIDE * m.ngeom);
    int status = 0;
    int ncon = collide(T, m, A.w, A.s, e, &status, queue, gs);
    if (T.lane() == 0) {
      wk[A.k.meta + K_META_NCON] = ncon;
      wk[A.k.meta + K_META_STATUS] = (double)((int)wk[A.k.meta + K_META_STATUS] | status);
      // the Newton phase takes envs with contacts (its long solves) first,
      // so that the envs left for the end of its queue are short ones
      if (A.order) {
        int slot = ncon > 0 ? atomicAdd(A.queue + Q_FRONT, 1) : A.count - 1 - atomicAdd(A.queue + Q_BACK, 1);
        A.order[slot] = item;
      }
    }
    T.sync();
    if (A.learn.mode == LEARN_DUMP || (A.learn.mode == LEARN_PREDICT && A.warm_mode == WARM_LEARNED))
      learn_list(T, A.learn, e, ncon, wk + A.k.meta);
    T.sync();
  }
}

// ---------------------------------------------------------------- phase 3
// newton.rs:113-473 and forward.rs:359-389: rows, Newton, the damped
// solve qacc = (M + hD)^-1 (f + qfrc_constraint), integration.
// two blocks of 256 threads an SM (128 registers a thread): 28 tiles of 16
// lanes an SM, one wave for 4096 Ant envs. LEARN = false (newton_plain_kernel,
// launched when the learned start neither predicts nor collects) leaves the
// learned start's code out of the kernel.
template <int G, bool LEARN>
__device__ __forceinline__ void newton_phase(const StepArgs& A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DModel& m = stage_model(A, smem);
  cg::thread_block block = cg::this_thread_block();
  Tile<G> T(cg::tiled_partition<G>(block));
  const WsLayout& w = A.wn;
  int tib = threadIdx.x / G;
  size_t gtile = (size_t)blockIdx.x * (blockDim.x / G) + tib;
  EnvCtx e;
  e.ws = tile_workspace(A, smem, w.stride, tib);
  e.scr = A.scratch + gtile * (size_t)A.s.stride;
  int nq = m.nq, nv = m.nv;
  double h = m.timestep;
  for (int item = first_item<G>(); item < A.count; item = next_item(T, A.queue + Q_NEWTON, A.count)) {
    const int ei = A.order ? A.order[item] : item;  // the env's index in the range
    size_t env = (size_t)A.start + ei;
    e.env = (int)env;
    e.prm = A.st.params + env * m.pstride;
    double* wk = A.work + env * A.k.stride;
    e.geo = wk + A.k.geoms;
    e.con = wk + A.k.contacts;
    double* ws = e.ws;
    prefetch_l1(T, e.prm, sizeof(double) * m.pstride);
    // the state and the smooth phase's results are on their way while the
    // meta block is read (an env that stopped stepping does not use them)
    load_async(T, ws + w.qpos, A.st.qpos + env * nq, nq);
    load_async(T, ws + w.qvel, A.st.qvel + env * nv, nv);
    load_async(T, ws + w.qacc, A.st.qacc + env * nv, nv);
    e.qm = w.qm >= 0 ? ws + w.qm : wk + A.k.qm;
    e.fac = w.fac >= 0 ? ws + w.fac : e.scr + A.s.chol;
    if (w.qm >= 0) load_async(T, ws + w.qm, wk + A.k.qm, nv * nv);
    load_async(T, ws + w.cdof, wk + A.k.cdof, 6 * nv);
    load_async(T, ws + w.acc, wk + A.k.a0, nv);
    load_async(T, ws + w.smooth, wk + A.k.smooth, nv);
    int status = (int)wk[A.k.meta + K_META_STATUS];
    int ncon = (int)wk[A.k.meta + K_META_NCON];
    prefetch_l1(T, e.con, sizeof(double) * C_STRIDE * ncon);
    load_wait();
    T.sync();
    int iters = 0, nr = 0;
    if (!(status & ST_NOT_SPD)) {
      double* acc = ws + w.acc;
      double* v = ws + w.vel;
      double* vpos = v;
      double* qvel = ws + w.qvel;
      if (m.solver == SOLVER_PGS) {
        // forward.rs:366-375: velocities through M + hD, then PGS on them
        // (the factor read in place when it does not live in the workspace)
        const double* lh = w.fac >= 0 ? ws + w.fac : wk + A.k.lh;
        if (w.fac >= 0) load_async(T, ws + w.fac, wk + A.k.lh, nv * nv);
        load_async(T, ws + w.rinv, wk + A.k.rinvh, nv);
        for (int k = T.lane(); k < nv; k += G) acc[k] = ws[w.smooth + k];
        load_wait();
        T.sync();
        solve_auto(T, lh, nv, nv, m.nblock, m.block_adr, m.dof_block, m.maxbs, ws + w.rinv, acc);
        for (int k = T.lane(); k < nv; k += G) v[k] = qvel[k] + h * acc[k];
        T.sync();
        vpos = ws + w.tmp;
        iters = pgs_solve(T, m, w, A.s, e, ncon, v, vpos, lh, A.st.prev_con + env * m.maxcon * P_STRIDE,
                          A.st.prev_ncon + env, &nr, &status);
        for (int k = T.lane(); k < nv; k += G) ws[w.qacc + k] = (v[k] - qvel[k]) / h;
        T.sync();
      } else {
        nr = build_rows(T, m, w, A.s, e, ncon, &status);
        const double* warm = A.warm_mode == WARM_REF_PREV_QACC ? ws + w.qacc : nullptr;
        // the learned warm start's predictions, or the slots for its targets
        const float *lfeat = nullptr, *lforce = nullptr;
        float* ldump = nullptr;
        int lnum = 0;
        if (LEARN && (A.learn.mode == LEARN_DUMP || (A.learn.mode == LEARN_PREDICT && A.warm_mode == WARM_LEARNED))) {
          int lbase = (int)wk[A.k.meta + K_META_LBASE];
          lnum = (int)wk[A.k.meta + K_META_LNUM];
          if (lnum > 0) {
            lfeat = A.learn.feat + (size_t)lbase * LEARN_NF;
            if (A.learn.mode == LEARN_PREDICT && A.warm_mode == WARM_LEARNED) lforce = A.learn.force + (size_t)lbase * 3;
            if (A.learn.mode == LEARN_DUMP) ldump = A.learn.rows + (size_t)lbase * 4;
          }
        }
        iters = newton_solve<G, LEARN>(T, m, w, A.s, e, nr, acc, warm, lfeat, lforce, lnum, ldump);
        if (wk[A.k.meta + K_META_DAMPED] != 0.0) {
          const double* lh = w.fac >= 0 ? ws + w.fac : wk + A.k.lh;
          if (w.fac >= 0) load_async(T, ws + w.fac, wk + A.k.lh, nv * nv);
          load_async(T, ws + w.rinv, wk + A.k.rinvh, nv);
          for (int k = T.lane(); k < nv; k += G) acc[k] = ws[w.smooth + k] + ws[w.qfrc_c + k];
          load_wait();
          T.sync();
          solve_auto(T, lh, nv, nv, m.nblock, m.block_adr, m.dof_block, m.maxbs, ws + w.rinv, acc);
        }
        for (int k = T.lane(); k < nv; k += G) {
          double vk = qvel[k] + h * acc[k];
          v[k] = vk;
          ws[w.qacc + k] = (vk - qvel[k]) / h;
        }
        T.sync();
      }
      integrate_pos(T, m, ws + w.qpos, vpos, h);
      copy_in(T, A.st.qpos + env * nq, ws + w.qpos, nq);
      copy_in(T, A.st.qvel + env * nv, v, nv);
      copy_in(T, A.st.qacc + env * nv, ws + w.qacc, nv);
      if (A.qpos_out) copy_in(T, A.qpos_out + ((size_t)ei * A.nstep + A.sidx) * nq, ws + w.qpos, nq);
    } else if (A.qpos_out) {
      copy_in(T, A.qpos_out + ((size_t)ei * A.nstep + A.sidx) * nq, A.st.qpos + env * nq, nq);
    }
    if (T.lane() == 0) {
      A.st.iters[env] = iters;
      A.st.ncon[env] = ncon;
      A.st.nrows[env] = nr;
      A.st.status[env] = (A.sidx == 0 ? 0 : A.st.status[env]) | status;
    }
    T.sync();
  }
}

template <int G>
__global__ void __launch_bounds__(256, 2) newton_kernel(const __grid_constant__ StepArgs A) {
  newton_phase<G, true>(A);
}
template <int G>
__global__ void __launch_bounds__(256, 2) newton_plain_kernel(const __grid_constant__ StepArgs A) {
  newton_phase<G, false>(A);
}

// whether a substep's Newton phase needs the learned start's code
inline bool newton_learns(const StepArgs& a) {
  return a.learn.mode == LEARN_DUMP || (a.learn.mode == LEARN_PREDICT && a.warm_mode == WARM_LEARNED);
}

// ---------------------------------------------------------------- learned start
// Features of the learned warm start's slots, between the collision and
// Newton phases (the network's forward pass over them follows as its own
// launch, mlp_forward_counted). A block takes 16 slots at a time: 8 threads
// share a slot's 3 x nv contact-frame Jacobian entries (thread t takes dofs
// t, t + 8, ...) and reduce J qvel and J a0 by shuffles, then write its 24
// features (in the contact frame n, t1, t2: depth, friction, J qvel (3),
// J a0 (3), the two bodies' translational and rotational invweight sums, the
// normal (3), the env's touching-contact count, the timestep, the point
// relative to each geom's centre (3 + 3), both geom types, and 1) to the list.
__device__ inline double learn_feature(int f, const DModel& m, const double* r, const double* prm, const double* geo,
                                       const double (&jv)[3], const double (&ja)[3], double nt) {
  int g1 = (int)r[C_G1], g2 = (int)r[C_G2];
  int b1 = m.geom_body[g1], b2 = m.geom_body[g2];
  switch (f) {
    case 0: return r[C_DEPTH];
    case 1: return fmax(prm[m.p_friction + g1], prm[m.p_friction + g2]);
    case 2: case 3: case 4: return jv[f - 2];
    case 5: case 6: case 7: return ja[f - 5];
    case 8: return prm[m.p_body_invw + 2 * b1] + prm[m.p_body_invw + 2 * b2];
    case 9: return prm[m.p_body_invw + 2 * b1 + 1] + prm[m.p_body_invw + 2 * b2 + 1];
    case 10: case 11: case 12: return r[C_NORMAL + f - 10];
    case 13: return nt;
    case 14: return m.timestep;
    case 15: case 16: case 17: return r[C_POS + f - 15] - geo[G_STRIDE * g2 + G_POS + f - 15];
    case 18: case 19: case 20: return r[C_POS + f - 18] - geo[G_STRIDE * g1 + G_POS + f - 18];
    case 21: return (double)m.geom_type[g1];
    case 22: return (double)m.geom_type[g2];
    default: return 1.0;
  }
}

constexpr int LEARN_THREADS = 128;  // 16 slots of 8 threads

__global__ void __launch_bounds__(LEARN_THREADS) learn_kernel(const __grid_constant__ StepArgs A) {
  const LearnArgs& L = A.learn;
  const int64_t n = min(*L.count, L.cap);
  const DModel& m = A.m;
  const int nv = m.nv;
  const int j = threadIdx.x >> 3, t = threadIdx.x & 7;  // slot of the group, thread of the slot
  for (int64_t base = (int64_t)blockIdx.x * 16; base < n; base += (int64_t)gridDim.x * 16) {
    const int64_t slot = base + j;
    int env = -1, c = 0;
    if (slot < n) {
      env = L.items[2 * slot];
      c = L.items[2 * slot + 1];
    }
    const bool live = env >= 0;
    const double* wk = A.work + (size_t)(live ? env : 0) * A.k.stride;
    const double* r = wk + A.k.contacts + C_STRIDE * c;
    double jv[3] = {0.0, 0.0, 0.0}, ja[3] = {0.0, 0.0, 0.0};
    if (live) {
      int g1 = (int)r[C_G1], g2 = (int)r[C_G2];
      int b1 = m.geom_body[g1], b2 = m.geom_body[g2];
      V3 p = ld3(r + C_POS);
      V3 dir[3] = {ld3(r + C_NORMAL), ld3(r + C_T1), ld3(r + C_T2)};
      const double* cdof = wk + A.k.cdof;
      const double* a0 = wk + A.k.a0;
      const double* qvel = A.st.qvel + (size_t)env * nv;
      for (int k = t; k < nv; k += 8)
        for (int d = 0; d < 3; d++) {
          double jk = pair_jac(m, cdof, b1, b2, p, dir[d], k);
          jv[d] += jk * qvel[k];
          ja[d] += jk * a0[k];
        }
    }
#pragma unroll
    for (int o = 1; o < 8; o <<= 1)
      for (int d = 0; d < 3; d++) {
        jv[d] += __shfl_xor_sync(0xffffffffu, jv[d], o);
        ja[d] += __shfl_xor_sync(0xffffffffu, ja[d], o);
      }
    if (slot < n)
      for (int f = t; f < LEARN_NF; f += 8) {
        float v = 0.0f;
        if (live)
          v = (float)learn_feature(f, m, r, A.st.params + (size_t)env * m.pstride, wk + A.k.geoms, jv, ja,
                                   wk[A.k.meta + K_META_LNUM]);
        L.feat[slot * LEARN_NF + f] = v;
      }
  }
}

// row' M^-1 row for set_const's right-hand sides (one per lane, r < nrhs):
// the unit vectors, then per body 3 axes x (translation, rotation) rows of
// its Jacobian at the inertial frame. With M = L L', row' M^-1 row is
// |L^-1 row|^2: one forward substitution, the vector in registers (NB >= nv;
// larger models solve in scratch below).
template <int NB, int G>
__device__ void invweight_quads(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e,
                                const double* prm, const double* L, int nv, int nrhs, double* quad) {
  for (int r = T.lane(); r < nrhs; r += G) {
    double y[NB];
    if (r < nv) {
#pragma unroll
      for (int k = 0; k < NB; k++) y[k] = k == r ? 1.0 : 0.0;
    } else {
      int q = r - nv;
      int b = q / 6, axis = (q % 6) / 2, kind = q % 2;
      if (b == 0) {
        quad[r] = 0.0;
        continue;
      }
      V3 dir{axis == 0 ? 1.0 : 0.0, axis == 1 ? 1.0 : 0.0, axis == 2 ? 1.0 : 0.0};
      V3 xip = ld3(e.ws + w.xpos + 3 * b) + mv(q_mat(ld4(e.ws + w.xquat + 4 * b)), ld3(prm + m.p_ipos + 3 * b));
      unsigned long long chain = m.body_dofmask[b];
#pragma unroll
      for (int k = 0; k < NB; k++) {
        y[k] = 0.0;
        if (k < nv && ((chain >> k) & 1ull)) {
          Sp c = ld6(e.ws + w.cdof + 6 * k);
          y[k] = kind == 0 ? dot(dir, point_vel(c, xip)) : dot(dir, c.ang);
        }
      }
    }
    double sq = 0.0;
#pragma unroll
    for (int i = 0; i < NB; i++) {
      if (i < nv) {
        double v = y[i];
#pragma unroll
        for (int k = 0; k < i; k++) v -= L[i * nv + k] * y[k];
        y[i] = v / L[i * nv + i];
        sq += y[i] * y[i];
      }
    }
    quad[r] = sq;
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
  e.ws = tile_workspace(A, smem, w.stride, tib);
  e.scr = A.scratch + gtile * (size_t)A.s.stride;
  int nv = m.nv;
  for (int item = first_item<G>(); item < n; item = next_item(T, A.queue + 0, n)) {
    e.env = envs ? envs[item] : A.start + item;
    double* prm = A.st.params + (size_t)e.env * m.pstride;
    e.prm = prm;
    copy_in(T, e.ws + w.qpos, prm + m.p_qpos_reset, m.nq);
    T.sync();
    // M^-1 by Cholesky of the full matrix (forward.rs:286-288); M and its
    // factor live in scratch because the workspace's tree region is still
    // needed
    double* L = e.scr + A.s.chol;
    double* rinv = e.ws + w.rinv;
    tree_down(T, m, w, e, false, nullptr);
    tree_up(T, m, w, e, false, L);
    if (nv == 0) continue;
    bool ok = chol_auto(T, L, nv, nv, 1, nullptr, nullptr, nv, rinv);
    // one right-hand side per lane: unit vectors, then per body 3 axes x
    // (translation, rotation) rows; x = M^-1 row, quad = row . x
    double* xs = e.scr + A.s.jac;  // [rhs][nv]
    int nrhs = nv + 6 * m.nbody;
    double* quad = e.scr + A.s.rows;  // [nrhs]
    if (ok && nv <= 16) {
      invweight_quads<16>(T, m, w, e, prm, L, nv, nrhs, quad);
    } else if (ok) {
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
          V3 xip = ld3(e.ws + w.xpos + 3 * b) + mv(q_mat(ld4(e.ws + w.xquat + 4 * b)), ld3(prm + m.p_ipos + 3 * b));
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
  const WsLayout& w = A.w;
  EnvCtx e;
  e.ws = tile_workspace(A, smem, w.stride, threadIdx.x / G);
  e.scr = nullptr;
  for (int item = first_item<G>(); item < A.count; item = next_item(T, A.queue + 0, A.count)) {
    size_t env = (size_t)A.start + item;
    e.env = (int)env;
    e.prm = A.st.params + env * m.pstride;
    double* gr = A.work + env * A.k.stride + A.k.geoms;
    copy_in(T, e.ws + w.qpos, A.st.qpos + env * m.nq, m.nq);
    T.sync();
    tree_down(T, m, w, e, false, gr);
    for (int g = T.lane(); g < m.ngeom; g += G) {
      float* o = geoms + ((size_t)item * m.ngeom + g) * 12;
      for (int a = 0; a < 12; a++) o[a] = (float)gr[G_STRIDE * g + a];
    }
    for (int c = T.lane(); c < m.ncam; c += G) {
      int b = m.cam_body[c];
      M3 xm = q_mat(ld4(e.ws + w.xquat + 4 * b));
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
    case K_SMOOTH: return (const void*)smooth_kernel<G>;
    case K_COLLIDE: return (const void*)collide_kernel<G>;
    case K_NEWTON: return (const void*)newton_kernel<G>;
    case K_NEWTON_PLAIN: return (const void*)newton_plain_kernel<G>;
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

size_t kernel_smem(int which, const StepArgs& a, int tiles_per_block) {
  size_t staged = a.stage_model ? (size_t)staged_model_bytes(a.m.arena_bytes) : 0;
  switch (which) {
    case K_COLLIDE:
      return staged + (size_t)tiles_per_block *
                          (collide_tile_ints(a.m) * sizeof(int) + collide_cache_doubles(a.m) * sizeof(double));
    case K_NEWTON:
    case K_NEWTON_PLAIN: return staged + (size_t)tiles_per_block * a.wn.stride * sizeof(double);
    default: return staged + (size_t)tiles_per_block * a.w.stride * sizeof(double);
  }
}

#define PG_LAUNCH(WHICH, KERNEL, CFG, ...)                                          \
  do {                                                                              \
    size_t smem = kernel_smem(WHICH, a, (CFG).tiles_per_block);                     \
    dim3 grid((CFG).blocks), block((CFG).tiles_per_block * (CFG).G);               \
    switch ((CFG).G) {                                                              \
      case 8: KERNEL<8><<<grid, block, smem, s>>>(__VA_ARGS__); break;              \
      case 16: KERNEL<16><<<grid, block, smem, s>>>(__VA_ARGS__); break;            \
      case 32: KERNEL<32><<<grid, block, smem, s>>>(__VA_ARGS__); break;            \
      default: return cudaErrorInvalidValue;                                        \
    }                                                                               \
    cudaError_t _e = cudaGetLastError();                                            \
    if (_e != cudaSuccess) return _e;                                               \
  } while (0)

cudaError_t launch_smooth_collide(const StepArgs& a, const SubstepCfg& c, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(a.queue, 0, QUEUE_INTS * sizeof(int), s);
  if (e != cudaSuccess) return e;
  PG_LAUNCH(K_SMOOTH, smooth_kernel, c.smooth, a);
  PG_LAUNCH(K_COLLIDE, collide_kernel, c.collide, a);
  return cudaSuccess;
}

// The Newton phase's order (envs with contacts first) pays only when its
// grid has fewer tiles than envs, so that tiles pull further envs from the
// queue; with a tile per env every env starts at once and the order is left
// out (the collision phase then records none).
inline StepArgs ordered_for(const StepArgs& a0, const LaunchCfg& newton) {
  StepArgs a = a0;
  if ((int64_t)newton.blocks * newton.tiles_per_block >= a.count) a.order = nullptr;
  return a;
}

cudaError_t launch_substep(const StepArgs& a0, const SubstepCfg& c, cudaStream_t s) {
  const StepArgs a = ordered_for(a0, c.newton);
  cudaError_t e = launch_smooth_collide(a, c, s);
  if (e != cudaSuccess) return e;
  if (a.learn.mode == LEARN_DUMP || (a.learn.mode == LEARN_PREDICT && a.warm_mode == WARM_LEARNED)) {
    e = launch_learn(a, a.learn.mode == LEARN_PREDICT, s);
    if (e != cudaSuccess) return e;
  }
  if (newton_learns(a)) PG_LAUNCH(K_NEWTON, newton_kernel, c.newton, a);
  else PG_LAUNCH(K_NEWTON_PLAIN, newton_plain_kernel, c.newton, a);
  return cudaSuccess;
}

__global__ void apply_param_kernel(const __grid_constant__ DModel d, double* params, int64_t count, int p, int64_t id,
                                   const double* v, int w, int nq) {
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < count) apply_param(d, params + e * d.pstride, p, id, v + e * w, nq);
}

cudaError_t launch_apply_param(const DModel& d, double* params, int64_t count, int p, int64_t id, const double* v, int w,
                               int nq, cudaStream_t s) {
  if (count <= 0) return cudaSuccess;
  apply_param_kernel<<<(unsigned)((count + 127) / 128), 128, 0, s>>>(d, params, count, p, id, v, w, nq);
  return cudaGetLastError();
}

__global__ void hull_support_kernel(const __grid_constant__ DModel m, int mesh, const double* dirs, int n,
                                    int* vertex) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) vertex[i] = hull_support(m, mesh, ld3(dirs + 3 * i), 0);
}

cudaError_t launch_hull_support(const DModel& m, int mesh, const double* dirs, int n, int* vertex, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  hull_support_kernel<<<(n + 127) / 128, 128, 0, s>>>(m, mesh, dirs, n, vertex);
  return cudaGetLastError();
}

cudaError_t reset_queue(const StepArgs& a, cudaStream_t s) { return cudaMemsetAsync(a.queue, 0, QUEUE_INTS * sizeof(int), s); }

cudaError_t learn_prepare() { return mlp_prepare(); }

cudaError_t launch_learn(const StepArgs& a, bool infer, cudaStream_t s) {
  // the list's slots are counted on the device: the grids cover the
  // capacity, and blocks past this substep's slots return at once
  int64_t blocks = std::min<int64_t>((a.learn.cap + 15) / 16, 16 * 148);
  if (blocks < 1) return cudaSuccess;
  learn_kernel<<<(unsigned)blocks, LEARN_THREADS, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !infer) return e;
  return mlp_forward_counted(MlpDevice{a.learn.mlp_w, a.learn.mlp_f, a.learn.mlp_err}, a.learn.feat, a.learn.count, a.learn.cap,
                             a.learn.force, s);
}

cudaError_t launch_phase(int which, const StepArgs& a0, const LaunchCfg& c, cudaStream_t s) {
  // the collision phase always records the order; the Newton phase reads it
  // when its own grid is smaller than the range (ordered_for)
  const StepArgs a = which == K_NEWTON ? ordered_for(a0, c) : a0;
  switch (which) {
    case K_SMOOTH: PG_LAUNCH(K_SMOOTH, smooth_kernel, c, a); break;
    case K_COLLIDE: PG_LAUNCH(K_COLLIDE, collide_kernel, c, a); break;
    case K_NEWTON:
      if (newton_learns(a)) PG_LAUNCH(K_NEWTON, newton_kernel, c, a);
      else PG_LAUNCH(K_NEWTON_PLAIN, newton_plain_kernel, c, a);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaSuccess;
}

cudaError_t launch_set_const(const StepArgs& a, const LaunchCfg& c, const int* envs, int n, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(a.queue, 0, QUEUE_INTS * sizeof(int), s);
  if (e != cudaSuccess) return e;
  PG_LAUNCH(K_SET_CONST, set_const_kernel, c, a, envs, n);
  return cudaSuccess;
}

cudaError_t launch_poses(const StepArgs& a, const LaunchCfg& c, float* geoms, float* cams, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(a.queue, 0, QUEUE_INTS * sizeof(int), s);
  if (e != cudaSuccess) return e;
  PG_LAUNCH(K_POSES, poses_kernel, c, a, geoms, cams);
  return cudaSuccess;
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
