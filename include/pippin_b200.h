/* pippin_b200: batched FP64 rigid-body physics on one NVIDIA B200.
 *
 * C-ABI of the backend that plugs in behind pippin-env's `Physics` trait
 * (crates/pippin-env/src/lib.rs:109-155). Plain pointers and sizes only; the
 * caller owns every buffer and the library copies in and out (as the
 * reference backends do, crates/pippin-env/src/pippin_cpu.rs:159-205).
 * One handle holds a batch of environments on one GPU. Calls on a handle must
 * be serialised by the caller (the trait object is Send, not Sync).
 *
 * Every function returns 0 (PG_OK) on success or a PG_ERR_* code; the message
 * of the last failure on the calling thread is pg_last_error(). Buffer-size
 * mismatches return PG_ERR_LENGTH where the reference's check_len panics
 * (crates/pippin-env/src/lib.rs:241-243); a Rust shim turns that into the
 * same panic.
 *
 * Model blob (input of pg_create; written by pippin_b200/mjcf.py):
 *   bytes 0..7   magic "PGBLOB01"
 *   bytes 8..11  uint32 version (1)
 *   bytes 12..15 uint32 number of arrays N
 *   then N directory entries of 64 bytes:
 *     char     name[40]   NUL-padded array name
 *     uint32   dtype      1 = float64, 2 = int64, 3 = uint8
 *     uint32   reserved
 *     uint64   count      elements
 *     uint64   offset     byte offset from the blob start, multiple of 8
 *   then the array data (little-endian). The arrays are the fields of the
 *   reference's compiled Model (crates/pippin/src/model.rs:103-249), named as
 *   there; see pippin_b200/mjcf.py:to_blob for the list.
 */
#ifndef PIPPIN_B200_H
#define PIPPIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pg_handle pg_handle;

/* status codes */
enum {
  PG_OK = 0,
  PG_ERR_INVALID = 1,     /* bad argument or model (message in pg_last_error) */
  PG_ERR_LENGTH = 2,      /* buffer length does not match envs x width */
  PG_ERR_CUDA = 3,        /* CUDA runtime error */
  PG_ERR_UNSUPPORTED = 4, /* feature not available for this model */
  PG_ERR_NOMEM = 5
};

/* State fields (crates/pippin-env/src/lib.rs:20-26, plus the Newton warm
 * start and applied forces of crates/pippin/src/batch.rs:98-104). */
enum { PG_FIELD_QPOS = 0, PG_FIELD_QVEL = 1, PG_FIELD_CTRL = 2, PG_FIELD_QACC = 3, PG_FIELD_QFRC_APPLIED = 4 };

/* Per-env parameters, in the order of crates/pippin/src/params.rs:10-39. */
enum {
  PG_PARAM_GEOM_FRICTION = 0,
  PG_PARAM_GEOM_SIZE = 1,
  PG_PARAM_GEOM_RGBA = 2,
  PG_PARAM_GEOM_CONTYPE = 3,
  PG_PARAM_GEOM_CONAFFINITY = 4,
  PG_PARAM_BODY_MASS = 5,
  PG_PARAM_DOF_DAMPING = 6,
  PG_PARAM_ACTUATOR_GAIN = 7,
  PG_PARAM_ACTUATOR_BIAS = 8,
  PG_PARAM_BODY_INERTIA = 9,
  PG_PARAM_BODY_IPOS = 10,
  PG_PARAM_QPOS0 = 11
};

enum { PG_SOLVER_NEWTON = 0, PG_SOLVER_PGS = 1 };
/* Newton start: the reference's cost-gated previous qacc
 * (crates/pippin/src/newton.rs:238-245), cold (a0), or the learned
 * per-contact prediction behind the same cost gate. */
enum { PG_WARM_REF_PREV_QACC = 0, PG_WARM_COLD = 1, PG_WARM_LEARNED = 2 };

/* geom shapes (crates/pippin-env/src/lib.rs:39-55) */
enum { PG_SHAPE_PLANE = 0, PG_SHAPE_SPHERE = 1, PG_SHAPE_CAPSULE = 2, PG_SHAPE_BOX = 3, PG_SHAPE_CYLINDER = 4,
       PG_SHAPE_MESH = 5 };

/* per-env status bits reported by pg_stats */
enum { PG_STATUS_CAP_EXCEEDED = 1, PG_STATUS_NOT_SPD = 2, PG_STATUS_UNSUPPORTED_PAIR = 4 };

/* crates/pippin-env/src/lib.rs:28-36 (plus body and joint counts) */
typedef struct pg_model_dims {
  int64_t nq, nv, nu, ngeom, ncam, nbody, njnt;
} pg_model_dims;

/* crates/pippin-env/src/lib.rs:102-107: world pose, row-major rotation */
typedef struct pg_pose {
  float pos[3];
  float mat[9];
} pg_pose;

/* crates/pippin-env/src/lib.rs:171-176 */
typedef struct pg_geom_appearance {
  float rgba[4];
  float scale[3];
  float pad;
} pg_geom_appearance;

/* crates/pippin-env/src/lib.rs:58-68 (name via pg_name_of) */
typedef struct pg_geom_visual {
  int32_t shape;  /* PG_SHAPE_* */
  int32_t mesh;   /* mesh index for PG_SHAPE_MESH, else -1 */
  float size[3];
  float rgba[4];
  int32_t body;
  int32_t group;
} pg_geom_visual;

/* name tables for pg_name_of */
enum { PG_NAMES_BODY = 0, PG_NAMES_GEOM = 1, PG_NAMES_CAMERA = 2, PG_NAMES_MESH = 3, PG_NAMES_JOINT = 4,
       PG_NAMES_ACTUATOR = 5 };

/* Construct a batch of n_envs copies of the model on CUDA device `device`
 * (replaces PippinCpu::new, crates/pippin-env/src/pippin_cpu.rs:22-29). */
int pg_create(const void* model_blob, size_t bytes, int64_t n_envs, int device, pg_handle** out);
int pg_destroy(pg_handle* h);

/* Physics::name / num_envs / dims (crates/pippin-env/src/lib.rs:110-112) */
const char* pg_name(const pg_handle* h);
int64_t pg_num_envs(const pg_handle* h);
int pg_dims(const pg_handle* h, pg_model_dims* out);

/* Physics::step(envs, nstep) (lib.rs:115-116; pippin_cpu.rs:98-112): advance
 * envs [start, end) by nstep substeps each. Stream-ordered: returns after
 * launch; the next call that reads state waits for it. */
int pg_step(pg_handle* h, int64_t start, int64_t end, int64_t nstep);

/* Physics::set(Ctrl) followed by Physics::step, with the controls already in
 * device memory (an on-GPU policy's output): ctrl_dev is (end-start, nu)
 * FP64 on the handle's device, read in stream order on pg_stream. */
int pg_step_device(pg_handle* h, int64_t start, int64_t end, int64_t nstep, const double* ctrl_dev);

/* pg_step without allocating: no counterpart in the reference. For callers
 * that cannot have a call allocate device memory (another component owns the
 * GPU's memory, a latency-critical loop must stay out of the allocator, or
 * memory is already exhausted). Scratch comes from a fixed 16 MiB array in
 * the library's device image, one per GPU that loads the library, held until
 * exit; as many envs step at once as fit in it, the rest follow in the same
 * launch. A model whose per-block scratch exceeds the array is rejected with
 * PG_ERR_UNSUPPORTED. Every call looks the array's device address up again
 * (so a context the host program resets and makes again is followed); the
 * first call on a device also loads the library's device image there, so make
 * it before any stream capture. All calls share the array and keep its last
 * contents: calls that overlap on the GPU race. Stream-ordered like pg_step. */
int pg_step_static(pg_handle* h, int64_t start, int64_t end, int64_t nstep);

/* Batch::rollout (crates/pippin/src/batch.rs:46-59): ctrl is
 * (end-start, nstep, nu), qpos_out (end-start, nstep, nq) or NULL. Host
 * buffers; returns when qpos_out is filled. */
int pg_rollout(pg_handle* h, int64_t start, int64_t end, int64_t nstep, const double* ctrl, double* qpos_out);

/* Physics::reset(envs) (lib.rs:117-118; pippin_cpu.rs:114-120) */
int pg_reset(pg_handle* h, const int64_t* envs, int64_t n);

/* Physics::get / set (lib.rs:120-123; pippin_cpu.rs:159-187), row-major
 * (end-start, width); `len` is the buffer's element count. */
int pg_get(pg_handle* h, int field, int64_t start, int64_t end, double* out, size_t len);
int pg_set(pg_handle* h, int field, int64_t start, int64_t end, const double* src, size_t len);

/* Physics::poses (lib.rs:125-127; pippin_cpu.rs:189-205): geoms is
 * (end-start) x ngeom poses, cams (end-start) x ncam. */
int pg_poses(pg_handle* h, int64_t start, int64_t end, pg_pose* geoms, size_t ngeoms_len, pg_pose* cams,
             size_t ncams_len);

/* Physics::poses into device memory, for a renderer on the same GPU (the
 * zero-copy frame path of crates/pippin-env/src/pipeline.rs:28-40; the values
 * are pg_poses's, crates/pippin-env/src/pippin_cpu.rs:189-205). geoms_dev
 * holds (end-start) x ngeom poses, cams_dev (end-start) x ncam (either may be
 * NULL when its count is 0), both on the handle's device. Enqueued on
 * pg_stream after the steps before it; returns without waiting. */
int pg_poses_device(pg_handle* h, int64_t start, int64_t end, pg_pose* geoms_dev, pg_pose* cams_dev);

/* Physics::set_param / get_param (lib.rs:129-141; pippin_cpu.rs:122-143;
 * params.rs:111-177). values are (end-start, width). All-or-nothing:
 * nothing changes when any value is rejected. */
int pg_param_width(const pg_handle* h, int param);
int pg_set_param(pg_handle* h, int param, int64_t id, int64_t start, int64_t end, const double* values, size_t len);
int pg_get_param(pg_handle* h, int param, int64_t id, int64_t start, int64_t end, double* out, size_t len);

/* Physics::appearance (lib.rs:145-158; pippin_cpu.rs:145-157) */
int pg_appearance(pg_handle* h, int64_t start, int64_t end, pg_geom_appearance* out, size_t len);

/* Physics::scene (lib.rs:113; pippin_cpu.rs:63-96): static export */
int pg_scene_counts(const pg_handle* h, int64_t* nbody, int64_t* ngeom, int64_t* nmesh, int64_t* ncam);
int pg_scene_geoms(const pg_handle* h, pg_geom_visual* out, size_t len);
int pg_scene_mesh(const pg_handle* h, int64_t mesh, float* vertices, size_t nvert_len, uint32_t* triangles,
                  size_t ntri_len, int64_t* nvert, int64_t* ntri);
int pg_camera_fovy(const pg_handle* h, int64_t cam, float* fovy);
int pg_name_of(const pg_handle* h, int table, int64_t id, char* buf, size_t len);

/* Solver options for every env (model.rs:60-100 `kind`, `iterations`,
 * `tolerance`) and the Newton start. Negative values keep the current. */
int pg_set_solver(pg_handle* h, int kind, int max_iter, double tolerance, int warm_mode);

/* Per-env diagnostics of the last step (data.rs:52-55 newton iterations,
 * contact and row counts, PG_STATUS_* bits). Any pointer may be NULL. */
int pg_stats(pg_handle* h, int64_t start, int64_t end, int32_t* iters, int32_t* ncon, int32_t* nrows,
             int32_t* status);

/* Learned Newton warm start. No counterpart in the reference, which starts
 * Newton from the previous step's acceleration when that lowers the cost
 * (newton.rs:238-245). With a network loaded and warm mode PG_WARM_LEARNED,
 * each substep lists the touching contacts (24 features each), predicts
 * their frame forces on the tensor cores, and offers a0 + M^-1 J' f as the
 * starting point behind the same cost gate; the solution and its tolerance
 * are unchanged. Applies to the Newton solver on every model (the register
 * path and the tile paths with islands).
 * pg_set_warm_mlp: weights as in include/pippin_b200_mlp.h (36662 floats). */
int pg_set_warm_mlp(pg_handle* h, const float* weights, size_t len);

/* Training pairs for the warm start: one substep of envs [start, end) (with
 * the current controls, like pg_step), returning for each touching contact
 * solved by Newton its 24 features (X) and the converged
 * forces of its four pyramid rows (rows; the frame forces are
 * f_n = r0 + r1 + r2 + r3, f_t1 = mu (r0 - r1), f_t2 = mu (r2 - r3), mu =
 * feature 1). X holds pg_warm_capacity * 24 floats, rows pg_warm_capacity * 4.
 * *n gets the number of pairs written. */
int pg_warm_samples(pg_handle* h, int64_t start, int64_t end, float* X, size_t xlen, float* rows, size_t rlen,
                    int64_t* n);
int64_t pg_warm_capacity(const pg_handle* h);

/* Forward pass of one env without integration (forward.rs:263-271), for
 * per-stage parity checks: qm (nv*nv), qfrc_bias (nv), contacts as 13
 * doubles each (pos[3] normal[3] tangent[3] depth geom1 geom2 feature). */
int pg_debug_forward(pg_handle* h, int64_t env, double* qm, double* qfrc_bias, double* contacts, int64_t maxcon,
                     int64_t* ncon);

/* invweight0 of one env's model (forward.rs:275-333): body (nbody*2), dof (nv) */
int pg_invweight(pg_handle* h, int64_t env, double* body, double* dof);

/* Launch shape: lanes per env (8, 16, 32) and envs per block; 0 = keep.
 * pg_autotune times the candidate shapes on the current state (which it
 * saves and restores) and keeps the fastest. */
int pg_set_launch(pg_handle* h, int lanes_per_env, int envs_per_block);
int pg_get_launch(const pg_handle* h, int* lanes_per_env, int* envs_per_block, int* blocks);
int pg_autotune(pg_handle* h, int64_t nstep);

/* Wait for all work on the handle's stream. */
int pg_synchronize(pg_handle* h);

/* Device pointer of a state field, row-major (num_envs, width) FP64, for
 * zero-copy consumers on the same device (ordered on pg_stream). */
int pg_field_device_ptr(pg_handle* h, int field, double** dev_ptr);
/* The handle's CUDA stream (a cudaStream_t). */
void* pg_stream(pg_handle* h);

/* Message of the last failed call on this thread ("" if none). */
const char* pg_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PIPPIN_B200_H */
