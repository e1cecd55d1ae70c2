// Oracle (test infrastructure only): model, per-env data and engine entry
// points of the CPU restatement. Only tests/, bench.py's CPU-baseline leg and
// the smoke check load it; the product never does.
//
// Restates crates/pippin/src/{model.rs, data.rs, forward.rs, newton.rs,
// solver.rs, collision.rs, params.rs}. The model is read from the same model
// blob the CUDA backend consumes (written by pippin_b200/mjcf.py), so loader
// differences cannot show up as kernel error.
#pragma once
#include <array>
#include <memory>
#include <string>
#include <vector>

#include "om_math.h"

namespace om {

// model.rs:6-11 (blob codes 0..3)
enum JointType { JNT_FREE = 0, JNT_BALL = 1, JNT_SLIDE = 2, JNT_HINGE = 3 };
// model.rs:31-39 (blob codes 0..5)
enum GeomType { GEOM_PLANE = 0, GEOM_SPHERE = 1, GEOM_CAPSULE = 2, GEOM_BOX = 3, GEOM_CYLINDER = 4, GEOM_MESH = 5 };
enum Integrator { INT_EULER = 0, INT_IMPLICITFAST = 1 };
enum SolverKind { SOLVER_NEWTON = 0, SOLVER_PGS = 1 };

// model.rs:60-100
struct SolverOptions {
  int kind = SOLVER_NEWTON;
  int iterations = 30;
  Real tolerance = 1e-8;
  Real contact_margin = 1e-3;
  Real solref[2] = {0.02, 1.0};
  Real solimp[5] = {0.9, 0.95, 0.001, 0.5, 2.0};
  Real impratio = 1.0;
  Real contact_hertz = 0.0;
  Real contact_damping_ratio = 1.0;
  Real contact_slop = 5e-4;
};

struct Hull {  // convex hull of a mesh geom (vertices in the geom frame)
  std::vector<Vec3> vert;
  std::vector<std::array<int, 3>> tri;
  // polygon faces (outward normal, offset, counter-clockwise vertex loop)
  // and unique edges, for the general convex narrow phase
  std::vector<Vec3> face_n;
  std::vector<Real> face_d;
  std::vector<std::vector<int>> face_loop;
  std::vector<std::array<int, 2>> edge;
};

// model.rs:103-249 (fields the step path reads; names and layouts match)
struct Model {
  Real timestep = 0.002;
  Vec3 gravity{{0, 0, -9.81}};
  int integrator = INT_EULER;
  SolverOptions solver;
  int nq = 0, nv = 0, nu = 0;

  std::vector<int> body_parent, body_jntadr, body_jntnum, body_dofadr, body_dofnum, body_lastdof, body_weldid;
  std::vector<Vec3> body_pos, body_ipos;
  std::vector<Quat> body_quat;
  std::vector<Real> body_mass;
  std::vector<Mat3> body_inertia;

  std::vector<int> jnt_type, jnt_body, jnt_qposadr, jnt_dofadr, jnt_limited;
  std::vector<Vec3> jnt_pos, jnt_axis;
  std::vector<std::array<Real, 2>> jnt_range;
  std::vector<Real> jnt_stiffness, jnt_springref;

  std::vector<int> dof_body, dof_jnt, dof_parent;
  std::vector<Real> dof_damping, dof_armature;

  std::vector<int> geom_type, geom_body, geom_dataid, geom_group;
  std::vector<Vec3> geom_pos, geom_size;
  std::vector<Quat> geom_quat;
  std::vector<Real> geom_friction, geom_rbound;
  std::vector<uint32_t> geom_contype, geom_conaffinity;
  std::vector<std::array<Real, 4>> geom_rgba;
  std::vector<std::array<Vec3, 2>> geom_aabb;  // (center, half) in the geom frame

  std::vector<int> cam_body;
  std::vector<Vec3> cam_pos;
  std::vector<Quat> cam_quat;
  std::vector<Real> cam_fovy;

  std::vector<int> actuator_joint, actuator_ctrllimited, actuator_forcelimited;
  std::vector<Real> actuator_gear, actuator_gain;
  std::vector<std::array<Real, 3>> actuator_bias;
  std::vector<std::array<Real, 2>> actuator_ctrlrange, actuator_forcerange;
  std::vector<std::vector<std::pair<int, Real>>> actuator_moment;

  std::vector<int> eq_joint1, eq_joint2;  // eq_joint2 = -1: fixed to a constant
  std::vector<std::array<Real, 5>> eq_polycoef, eq_solimp;
  std::vector<std::array<Real, 2>> eq_solref;

  std::vector<std::pair<int, int>> dof_blocks;  // [start, end)
  std::vector<Hull> mesh_hull;

  std::vector<std::array<Real, 2>> body_invweight;
  std::vector<Real> dof_invweight;
  std::vector<Real> qpos0, qpos_reset;

  // Geom pairs passing every static filter except the contype/conaffinity
  // masks (model.rs:430-451 minus the mask test), in (g1, g2) lexicographic
  // order; `collision_pairs` is this list filtered by the current masks,
  // which reproduces rebuild_collision_pairs (model.rs:398-407).
  std::vector<std::pair<int, int>> pair_candidates;
  std::vector<std::pair<int, int>> collision_pairs;

  int nbody() const { return (int)body_parent.size(); }
  int njnt() const { return (int)jnt_type.size(); }
  int ngeom() const { return (int)geom_type.size(); }

  void rebuild_collision_pairs();
  Real rbound(int g) const;
  std::array<Vec3, 2> local_aabb(int g) const;
};

// Parse a model blob (format documented in include/pippin_b200.h), then run
// set_const. Returns nullptr and fills `err` on malformed input.
std::shared_ptr<Model> load_blob(const void* blob, size_t bytes, std::string* err);

// collision.rs:9-19
struct Contact {
  Vec3 pos, normal, tangent;
  Real depth;
  int geom[2];
  uint32_t feature;
};
struct Hit {  // collision.rs:31-37
  Vec3 pos, normal;
  Real depth;
  Vec3 tangent;
};
// collision.rs:47-55
void contact_frame(const Contact& c, Vec3* t1, Vec3* t2);

// newton.rs:36-44
struct NRow {
  Real aref, d;
  bool bilateral;
  bool active(Real r) const { return bilateral || r < 0.0; }
};

// solver.rs:17-33
enum RowKindTag { ROW_NORMAL = 0, ROW_FRICTION = 1, ROW_BILATERAL = 2 };
struct PgsRow {
  int kind;
  Real sep;     // Normal / Bilateral
  int normal;   // Friction: index of its normal row
  Real mu;      // Friction
  Real inv_a;
  int contact;  // -1 for limits / equality rows
};

// data.rs:8-131 (per-env state and scratch)
struct Data {
  Real time = 0.0;
  std::vector<Real> qpos, qvel, ctrl, qfrc_applied;
  std::vector<Vec3> xpos, xipos, xanchor, xaxis, geom_xpos;
  std::vector<Quat> xquat;
  std::vector<Mat3> xmat, geom_xmat;
  std::vector<Spatial> cdof, cdof_dot, cvel;
  std::vector<SpInertia> cinert, crb;
  std::vector<Real> qm, qm_chol, qfrc_bias, qfrc_passive, qfrc_actuator, qfrc_constraint, qacc, actuator_force;
  std::vector<char> actuator_clamped;
  std::vector<Contact> contacts;

  // scratch (data.rs:58-80)
  std::vector<Real> jac, minv_jt, lambda, v, v_pos, smooth, tmp_nv, diag, pos;
  std::vector<NRow> nrows;
  std::vector<PgsRow> rows;
  std::vector<Contact> prev_contacts;
  std::vector<std::array<Real, 3>> prev_lambda;
  std::vector<Spatial> cacc, cfrc;
  int newton_iters = 0;
  int nrows_last = 0;   // constraint rows of the last step (diagnostic)
  int status = 0;       // 0 ok; 2 = mass matrix not positive definite
};

void data_init(const Model& m, Data& d);        // data.rs:83-119
void data_reset(const Model& m, Data& d);       // data.rs:122-131

// forward.rs
void kinematics(const Model& m, Data& d);
void crba(const Model& m, Data& d);
void velocity(const Model& m, Data& d);
void rne(const Model& m, Data& d);
void passive(const Model& m, Data& d);
void actuation(const Model& m, Data& d);
void collide(const Model& m, Data& d);
void forward(const Model& m, Data& d);
void set_const(Model& m);
void step(const Model& m, Data& d);
void integrate_pos(const Model& m, Real* qpos, const Real* qvel, Real h);
void mass_solve(const Model& m, const Real* l, Real* x);

// collision.rs:59-96 and the general convex path (collision.rs:102-147)
struct GeomPose {
  int typ;
  Vec3 pos;
  Mat3 mat;
  Vec3 size;
  const Hull* hull;
};
void collide_pair(const GeomPose& a, const GeomPose& b, Real margin, std::vector<Hit>& out);
// narrow-phase helpers shared by the primitive and general paths
struct DistPt {
  Real d;
  Vec3 p;
};
Vec3 closest_on_segment(Vec3 a, Vec3 b, Vec3 p);
void closest_segments(Vec3 p0, Vec3 p1, Vec3 q0, Vec3 q1, Vec3* x, Vec3* y);
std::vector<Vec3> clip(const std::vector<Vec3>& poly, Vec3 pn, Real off);
void reduce_to_four(std::vector<DistPt>& pts);
void stable_sort_dist(std::vector<DistPt>& v);
bool needs_general(int a, int b);
void collide_general(const GeomPose& a, const GeomPose& b, Real margin, std::vector<Hit>& out);
int hull_support_walk(const std::vector<Vec3>& pts, const std::vector<std::array<int, 2>>& edges, Vec3 dir);

// newton.rs:378-473, solver.rs:63-251
void newton_solve(const Model& m, Data& d, Real* a);
void pgs_solve(const Model& m, Data& d, Real* v, std::vector<Real>& v_pos);
Real impedance(const Real solimp[5], Real pos);  // newton.rs:52-66

// params.rs
enum Param {
  P_GEOM_FRICTION = 0, P_GEOM_SIZE, P_GEOM_RGBA, P_GEOM_CONTYPE, P_GEOM_CONAFFINITY, P_BODY_MASS,
  P_DOF_DAMPING, P_ACTUATOR_GAIN, P_ACTUATOR_BIAS, P_BODY_INERTIA, P_BODY_IPOS, P_QPOS0, P_COUNT
};
int param_width(const Model& m, int p);
int param_count(const Model& m, int p);
bool set_param(Model& m, int p, int id, const Real* v, int n, std::string* err);
void get_param(const Model& m, int p, int id, Real* out);

// Per-stage FP64 operation counter (adds, multiplies, divides, sqrt as
// written in the reference loops), accumulated per thread.
enum Stage { ST_KIN = 0, ST_CRBA, ST_RNE, ST_PASSACT, ST_COLLIDE, ST_FACTOR, ST_ROWS, ST_NEWTON, ST_PGS, ST_INTEGRATE, ST_COUNT };
// Built twice: counting (OM_COUNT_FLOPS=1) for the algorithmic-FLOP figures,
// and without counters for the timed CPU baseline.
extern thread_local double g_flops[ST_COUNT];
#ifndef OM_COUNT_FLOPS
#define OM_COUNT_FLOPS 1
#endif
#if OM_COUNT_FLOPS
#define OM_FLOPS(stage, n) (::om::g_flops[(stage)] += (double)(n))
#else
#define OM_FLOPS(stage, n) ((void)0)
#endif

}  // namespace om
