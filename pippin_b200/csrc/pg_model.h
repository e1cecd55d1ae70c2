// Device-resident model, per-env parameter blocks, per-env state and the
// per-tile workspace layout of the batched substep.
//
// HBM layout (all FP64 unless noted):
//   model arena       one copy of the model constants; each block stages it
//                     into its shared memory when it fits (model_bytes)
//   env parameters    [env][pstride]: the per-env copy of every parameter
//                     the reference can change per environment
//                     (crates/pippin/src/params.rs:10-39) plus derived
//                     invweight0 (forward.rs:275-333)
//   env state         qpos[env][nq], qvel[env][nv], ctrl[env][nu],
//                     qacc[env][nv] (Newton warm start), qfrc_applied[env][nv]
//   tile scratch      [tile][sstride]: geom poses, contacts, constraint rows
//                     and island buffers of the env a tile is working on
//   shared memory     per block: staged model, then [tile][wstride]
//                     workspaces (state, M, cdof, and one region used first
//                     by the tree walks, then by the factorisations/Newton)
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/pippin_b200.h"

namespace pg {

enum { JNT_FREE = 0, JNT_BALL = 1, JNT_SLIDE = 2, JNT_HINGE = 3 };
enum { GEOM_PLANE = 0, GEOM_SPHERE = 1, GEOM_CAPSULE = 2, GEOM_BOX = 3, GEOM_CYLINDER = 4, GEOM_MESH = 5 };
enum { SOLVER_NEWTON = 0, SOLVER_PGS = 1 };
enum { WARM_REF_PREV_QACC = 0, WARM_COLD = 1, WARM_LEARNED = 2 };

// per-env status bits
enum { ST_OK = 0, ST_CAP_EXCEEDED = 1, ST_NOT_SPD = 2, ST_UNSUPPORTED_PAIR = 4 };

// contact record in tile scratch (doubles)
enum { C_POS = 0, C_NORMAL = 3, C_TANGENT = 6, C_DEPTH = 9, C_G1 = 10, C_G2 = 11, C_FEATURE = 12, C_T1 = 13,
       C_T2 = 16, C_ROW = 19, C_STRIDE = 20 };
// constraint row record in tile scratch (doubles)
enum { R_AREF = 0, R_D = 1, R_JAR = 2, R_JP = 3, R_POS = 4, R_DIAG = 5, R_FLAGS = 6, R_ACT = 7, R_STRIDE = 8 };
// geom record in tile scratch (doubles): world pose and world bounding box
enum { G_POS = 0, G_MAT = 3, G_AABB = 12, G_STRIDE = 18 };

constexpr int NV_MAX = 64;  // dof-chain masks are 64-bit
constexpr int HULL_FACE_MAX = 32;     // longest face loop a lane clips in its own buffers
constexpr int HULL_FACE_LIMIT = 256;  // longest hull face loop accepted (past HULL_FACE_MAX: clipped in shared memory)
constexpr int HULL_SCAN_BELOW = 64;   // hulls with fewer vertices scan for support points (fasthull.rs:23)
constexpr int HULL_SEEDS = 26;        // seed directions of the support walk: (x, y, z) in {-1, 0, 1}^3, not 0
constexpr int GEN_SURV_CAP = 64;      // edges per polytope the edge query lists after pruning
constexpr int GEN_CACHE_LIMIT = 1152; // largest polytope cache of a collide tile (doubles); above: no cache
constexpr int CYL_SIDES = 16;  // a cylinder in the general narrow phase: a prism of this many sides
constexpr int COLLIDE_QUEUE = 64;  // broad-phase survivor slots per collide tile (2 x the widest tile)

struct DModel {
  // ---- dims
  int nq, nv, nu, nbody, njnt, ngeom, ncam, neq, npair, nblock, nlevel, nmesh;
  int maxcon, maxrows, maxbs;
  int gen_vmax, gen_fmax;  // most vertices / faces of a polytope in a general pair (0: no such pair)
  int gen_lmax;            // longest face loop of a polytope in a general pair
  int gen_cache;           // doubles of polytope cache per collide tile (0: vertices formed at each use)
  int gen_clip;            // doubles of shared clip buffers per collide tile (0: the lane's own buffers)
  // ---- options (model.rs:60-100)
  double timestep, gravity[3];
  int integrator, solver, iterations;
  double tolerance, margin, solref[2], solimp[5], impratio, hertz, dampratio, slop;

  // ---- bodies
  const int* body_parent;
  const int* body_jntadr;
  const int* body_jntnum;
  const int* body_dofadr;
  const int* body_dofnum;
  const int* body_lastdof;
  const unsigned long long* body_dofmask;  // bit k: dof k on the body's chain to the world
  const double* body_pos;                  // [nb][3]
  const double* body_quat;                 // [nb][4]
  const int* level_adr;                    // [nlevel+1] into level_body (bodies by depth)
  const int* level_body;
  const int* child_adr;                    // [nb+1] into child_list (children, decreasing id)
  const int* child_list;
  // ---- joints
  const int* jnt_type;
  const int* jnt_qposadr;
  const int* jnt_dofadr;
  const int* jnt_limited;
  const double* jnt_pos;  // [nj][3]
  const double* jnt_axis;
  const double* jnt_range;  // [nj][2]
  const double* jnt_stiffness;
  const double* jnt_springref;
  // ---- dofs
  const int* dof_body;
  const int* dof_parent;
  const double* dof_armature;
  const int* dof_block;       // block id of each dof
  const int* block_adr;       // [nblock][2] = [start, end)
  const int* dofact_adr;      // [nv+1] actuator contributions per dof, in actuator order
  const int* dofact_u;
  const double* dofact_coef;
  // ---- geoms
  const int* geom_type;
  const int* geom_body;
  const int* geom_dataid;
  const double* geom_pos;   // [ng][3]
  const double* geom_quat;  // [ng][4]
  const int* pair_g;        // [npair][2] candidate pairs (static filter; masks per env)
  // ---- cameras
  const int* cam_body;
  const double* cam_pos;
  const double* cam_quat;
  // ---- actuators
  const double* act_gear;
  const int* act_ctrllimited;
  const double* act_ctrlrange;  // [nu][2]
  const int* act_forcelimited;
  const double* act_forcerange;
  const int* act_moment_adr;
  const int* act_moment_num;
  const int* moment_jnt;
  const double* moment_coef;
  // ---- joint equality
  const int* eq_j1;
  const int* eq_j2;
  const double* eq_poly;    // [neq][5]
  const double* eq_solref;  // [neq][2]
  const double* eq_solimp;  // [neq][5]
  // ---- reference configuration
  const double* qpos0;
  // ---- convex hulls (for mesh geoms)
  const int* hull_vadr;
  const int* hull_vnum;
  const double* hull_vert;  // [*][3]
  const int* hull_fadr;      // per mesh: first polygon face, count
  const int* hull_fnum;
  const double* hull_face;   // [*][4]: outward unit normal, offset (n.x <= d)
  const int* hull_fvadr;     // per face: its vertex loop (counter-clockwise from outside)
  const int* hull_fvnum;
  const int* hull_fv;
  const int* hull_eadr;      // per mesh: first edge, count
  const int* hull_enum;
  const int* hull_edge;      // [*][2] vertex pairs
  const int* hull_eface;     // [*][2] the two faces of each edge (mesh-local face index)
  const int* hull_nbadr;     // per hull vertex (global index): its neighbours in hull_nb, count
  const int* hull_nbnum;
  const int* hull_nb;        // neighbour vertices (mesh-local index), from the edges
  const int* hull_seed;      // [nmesh][HULL_SEEDS] vertex extreme along each seed direction

  // ---- per-env parameter block offsets (doubles) and stride
  int p_friction, p_size, p_contype, p_conaff, p_mass, p_inertia, p_ipos, p_damping, p_gain, p_bias, p_qpos_reset,
      p_body_invw, p_dof_invw, p_rgba;
  int pstride;

  // ---- the arena all pointers above point into
  const unsigned char* arena;
  int arena_bytes;
};

// One env's new values of one parameter into its parameter block
// (params.rs:121-176); pg_set_param runs it on the device, one env a thread.
__host__ __device__ inline void apply_param(const DModel& d, double* prm, int p, int64_t id, const double* v, int nq) {
  switch (p) {
    case PG_PARAM_GEOM_FRICTION: prm[d.p_friction + id] = ::fmax(v[0], 0.0); break;
    case PG_PARAM_GEOM_SIZE: for (int k = 0; k < 3; k++) prm[d.p_size + 3 * id + k] = v[k]; break;
    case PG_PARAM_GEOM_RGBA: for (int k = 0; k < 4; k++) prm[d.p_rgba + 4 * id + k] = (double)(float)v[k]; break;
    case PG_PARAM_GEOM_CONTYPE:
    case PG_PARAM_GEOM_CONAFFINITY: {
      double bits = ::floor(::fmin(::fmax(v[0], 0.0), 4294967295.0));
      prm[(p == PG_PARAM_GEOM_CONTYPE ? d.p_contype : d.p_conaff) + id] = bits;
      break;
    }
    case PG_PARAM_BODY_MASS: {
      double old = prm[d.p_mass + id];
      double scale = old > 0.0 ? v[0] / old : 1.0;
      prm[d.p_mass + id] = v[0];
      for (int k = 0; k < 9; k++) prm[d.p_inertia + 9 * id + k] *= scale;
      break;
    }
    case PG_PARAM_DOF_DAMPING: prm[d.p_damping + id] = ::fmax(v[0], 0.0); break;
    case PG_PARAM_ACTUATOR_GAIN: prm[d.p_gain + id] = v[0]; break;
    case PG_PARAM_ACTUATOR_BIAS: for (int k = 0; k < 3; k++) prm[d.p_bias + 3 * id + k] = v[k]; break;
    case PG_PARAM_BODY_INERTIA:
      for (int k = 0; k < 9; k++) prm[d.p_inertia + 9 * id + k] = 0.0;
      for (int k = 0; k < 3; k++) prm[d.p_inertia + 9 * id + 4 * k] = v[k];
      break;
    case PG_PARAM_BODY_IPOS: for (int k = 0; k < 3; k++) prm[d.p_ipos + 3 * id + k] = v[k]; break;
    case PG_PARAM_QPOS0: for (int k = 0; k < nq; k++) prm[d.p_qpos_reset + k] = v[k]; break;
  }
}

// Per-tile shared-memory workspace (offsets in doubles). The `tree` region
// (poses, inertias, velocities, forces) is dead once the contacts are built
// and is reused by the factorisations and Newton (`fac` .. `warm`).
struct WsLayout {
  // live for the whole substep
  int qpos, qvel, ctrl, qacc, applied, qm, cdof, smooth, qfrc_c, acc, rinv, actforce, actclamped, misc;
  // tree walks, passive/actuator forces
  int xpos, xquat, xmat, cinert, cvel, cacc, cfrc, bias, passive, actf;
  // factorisations and Newton (alias the tree region); fac2 / rinv2: the
  // smooth phase's second factor (M + hD) beside the first (M)
  int fac, a0, grad, p, tmp, tmp2, mp, vel, warm, fac2, rinv2;
  // register Newton (nv <= 16, one dof tree): constraint rows [16][nv],
  // Hessian factor (packed), published vector [16] and row coefficients [32]
  // (placed over buffers that path leaves unused; -1 when it does not apply)
  int sj, sl, sx, sc;
  int stride;
};

// Per-tile global scratch layout (offsets in doubles).
struct ScrLayout {
  int geoms;     // ngeom * G_STRIDE
  int contacts;  // maxcon * C_STRIDE
  int jac;       // maxrows * nv
  int rows;      // maxrows * R_STRIDE
  int chol;      // nv * nv   (set_const factor)
  int sub_m;     // nv * nv   (island gather)
  int sub_j;     // maxrows * nv
  int sub_rows;  // maxrows * R_STRIDE
  int isl_dof;   // nv ints stored as doubles
  int isl_row;   // maxrows
  int isl_of_row;
  int mj;        // maxrows * nv   (PGS: M^-1 J' rows)
  int stride;
};

// Per-env work record in HBM, handed from one phase kernel to the next
// (offsets in doubles): what smooth dynamics leaves for the collision and
// Newton phases, the geoms and contacts of the narrow phase, and a small
// meta block (contact count, status bits, whether implicit damping applies).
enum { K_META_NCON = 0, K_META_STATUS = 1, K_META_DAMPED = 2, K_META_LBASE = 3, K_META_LNUM = 4, K_META_SIZE = 6 };

// Learned warm start: features of the touching contacts of all envs in one
// compact list (slots taken with a device counter), the network's frame
// forces for them, and, when collecting training data, the converged forces
// of their four pyramid rows.
enum { LEARN_OFF = 0, LEARN_PREDICT = 1, LEARN_DUMP = 2 };
constexpr int LEARN_NF = 24;  // features per contact
struct LearnArgs {
  int mode;
  int cap;          // slots in the list
  int* count;       // slots taken this substep (reset with the work counters)
  int* items;       // [cap][2] (env, contact) of each slot, from the collision phase
  float* feat;      // [cap][24]
  float* force;     // [cap][3]  predicted frame forces
  float* rows;      // [cap][4]  converged pyramid row forces (LEARN_DUMP)
  const uint16_t* mlp_w;  // the network (pg_mlp.h MlpDevice)
  const float* mlp_f;
  int* mlp_err;           // set when a wait of the forward pass on the tensor cores ran out
};
struct WorkLayout {
  int qm, cdof, a0, smooth, bias, lh, rinvh, geoms, contacts, meta;
  int stride;
};

struct EnvState {
  double* qpos;
  double* qvel;
  double* ctrl;
  double* qacc;
  double* applied;
  double* params;  // [env][pstride]
  int32_t* iters;
  int32_t* ncon;
  int32_t* nrows;
  int32_t* status;
  // PGS warm start carried between steps (solver.rs:254-289)
  double* prev_con;  // [env][maxcon][P_STRIDE]
  int32_t* prev_ncon;
};
// previous-step contact (PGS warm start): position, friction frame, geoms,
// impulses (normal, tangent 1, tangent 2)
enum { P_POS = 0, P_T1 = 3, P_T2 = 6, P_G1 = 9, P_G2 = 10, P_LAMBDA = 11, P_STRIDE = 14 };
// PGS row record in tile scratch (doubles; solver.rs:18-36)
enum { PR_KIND = 0, PR_SEP = 1, PR_MU = 2, PR_NORMAL = 3, PR_CONTACT = 4, PR_INVA = 5, PR_LAMBDA = 6, PR_STRIDE = 8 };
enum { PK_NORMAL = 0, PK_FRICTION = 1, PK_BILATERAL = 2 };

constexpr int MAX_PTR_FIELDS = 80;

// the work counters of a substep: one per phase kernel, the learned start's
// contact count, and the two ends of the Newton-phase order
enum { Q_SMOOTH = 0, Q_COLLIDE = 1, Q_NEWTON = 2, Q_LEARN = 3, Q_FRONT = 4, Q_BACK = 5, QUEUE_INTS = 8 };

struct StepArgs {
  DModel m;
  WsLayout w;   // smooth-dynamics phase (also set_const, poses)
  WsLayout wn;  // Newton phase
  ScrLayout s;
  WorkLayout k;
  EnvState st;
  double* scratch;   // [tiles][s.stride] (the Newton phase's rows and islands)
  double* work;      // [env][k.stride]
  int* queue;        // QUEUE_INTS work counters (reset before each substep): Q_* below
  int* order;        // [count] Newton-phase order (envs with contacts first), or nullptr: env order
  int start, count, nstep;
  int sidx;          // substep index within the call
  int warm_mode;
  LearnArgs learn;
  const double* ctrl_seq;  // optional (count, nstep, nu): per-substep controls
  double* qpos_out;        // optional (count, nstep, nq): qpos after each substep
  // model staging: byte offsets of the pointer fields of DModel, and
  // whether the arena is copied into shared memory
  int stage_model;
  int n_ptr;
  int ptr_off[MAX_PTR_FIELDS];
};

// shared bytes a block reserves for the staged model (DModel copy + arena)
#ifdef __CUDACC__
__host__ __device__
#endif
inline int staged_model_bytes(int arena_bytes) {
  return ((int)sizeof(DModel) + 15) / 16 * 16 + (arena_bytes + 15) / 16 * 16;
}

}  // namespace pg
