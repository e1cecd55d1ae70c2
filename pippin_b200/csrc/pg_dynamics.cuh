// Smooth dynamics of one environment on a tile of G lanes. Restates
// crates/pippin/src/forward.rs:14-211 as two tree walks:
//   down the tree, level by level (the bodies of one depth in parallel):
//     kinematics (:14-90) -> cdof, pose, cinert; velocity (:115-144) -> cvel;
//     RNE forward pass (:147-164) -> cacc, cfrc. cdof_dot is consumed as it
//     is formed (its only use is the body's own acceleration sum).
//   up the tree: composite inertia crb (CRBA, :93-101) in place of cinert,
//     and the RNE force sum (:165-168), children added in decreasing body
//     order as the reference's reverse loops do.
// then M (:102-111) and qfrc_bias (:169-171) with one lane per dof.
#pragma once
#include "pg_math.cuh"
#include "pg_model.h"
#include "pg_tile.cuh"

namespace pg {

struct EnvCtx {
  double* ws;         // tile workspace (shared memory)
  const double* prm;  // this env's parameter block
  double* scr;        // tile scratch (global): constraint rows, island buffers
  double* geo;        // this env's geom records (G_STRIDE each)
  double* con;        // this env's contacts (C_STRIDE each)
  int env;
  const double* qm;   // Newton phase: M (nv x nv), in the workspace or the work record
  double* fac;        // Newton phase: an nv x nv matrix to factor in (workspace or scratch)
};

// forward.rs:14-90 + 115-164 for one body, given its parent's results
__device__ inline void tree_down_body(const DModel& m, const WsLayout& w, const EnvCtx& e, int b, bool dynamics) {
  double* ws = e.ws;
  const double* q = ws + w.qpos;
  int p = m.body_parent[b];
  M3 xmp = q_mat(ld4(ws + w.xquat + 4 * p));  // the parent's stored rotation, exactly
  V3 pos = ld3(ws + w.xpos + 3 * p) + mv(xmp, ld3(m.body_pos + 3 * b));
  Q4 quat = q_mul(ld4(ws + w.xquat + 4 * p), ld4(m.body_quat + 4 * b));
  double* cdof = ws + w.cdof;
  int j0 = m.body_jntadr[b], j1 = j0 + m.body_jntnum[b];
  for (int j = j0; j < j1; j++) {
    int qa = m.jnt_qposadr[j], da = m.jnt_dofadr[j];
    int type = m.jnt_type[j];
    if (type == JNT_FREE) {
      pos = V3{q[qa], q[qa + 1], q[qa + 2]};
      quat = q_normalized(Q4{q[qa + 3], q[qa + 4], q[qa + 5], q[qa + 6]});
      M3 r = q_mat(quat);
      for (int k = 0; k < 3; k++) {
        V3 ek{k == 0 ? 1.0 : 0.0, k == 1 ? 1.0 : 0.0, k == 2 ? 1.0 : 0.0};
        st6(cdof + 6 * (da + k), Sp{V3{0, 0, 0}, ek});
        V3 a = col(r, k);
        st6(cdof + 6 * (da + 3 + k), Sp{a, cross(pos, a)});
      }
    } else if (type == JNT_BALL) {
      V3 jp = ld3(m.jnt_pos + 3 * j);
      V3 anchor = pos + q_rot(quat, jp);
      Q4 ql = q_normalized(Q4{q[qa], q[qa + 1], q[qa + 2], q[qa + 3]});
      quat = q_mul(quat, ql);
      pos = anchor - q_rot(quat, jp);
      M3 r = q_mat(quat);
      for (int k = 0; k < 3; k++) {
        V3 a = col(r, k);
        st6(cdof + 6 * (da + k), Sp{a, cross(anchor, a)});
      }
    } else if (type == JNT_HINGE) {
      V3 jp = ld3(m.jnt_pos + 3 * j), ja = ld3(m.jnt_axis + 3 * j);
      V3 anchor = pos + q_rot(quat, jp);
      V3 axis = q_rot(quat, ja);
      quat = q_mul(quat, q_axis_angle(ja, q[qa] - m.qpos0[qa]));
      pos = anchor - q_rot(quat, jp);
      st6(cdof + 6 * da, Sp{axis, cross(anchor, axis)});
    } else {  // slide
      V3 axis = q_rot(quat, ld3(m.jnt_axis + 3 * j));
      pos = pos + axis * (q[qa] - m.qpos0[qa]);
      st6(cdof + 6 * da, Sp{V3{0, 0, 0}, axis});
    }
  }
  quat = q_normalized(quat);
  M3 xm = q_mat(quat);
  st3(ws + w.xpos + 3 * b, pos);
  st4(ws + w.xquat + 4 * b, quat);
  const double* prm = e.prm;
  V3 xipos = pos + mv(xm, ld3(prm + m.p_ipos + 3 * b));
  SpI I = spi_from_com(prm[m.p_mass + b], xipos, mrot(ld9(prm + m.p_inertia + 9 * b), xm));
  st13(ws + w.cinert + 13 * b, I);
  if (!dynamics) return;
  // velocity (forward.rs:115-144) and RNE forward (forward.rs:153-164)
  const double* qvel = ws + w.qvel;
  Sp v = ld6(ws + w.cvel + 6 * p);
  Sp a = ld6(ws + w.cacc + 6 * p);
  for (int j = j0; j < j1; j++) {
    int da = m.jnt_dofadr[j], type = m.jnt_type[j];
    if (type == JNT_FREE || type == JNT_BALL) {
      int lin = type == JNT_FREE ? 3 : 0;
      int rot = type == JNT_FREE ? da + 3 : da;
      for (int k = 0; k < lin; k++) v = sp_add(v, sp_scale(ld6(cdof + 6 * (da + k)), qvel[da + k]));
      // all rotational dofs share one velocity (forward.rs:130-133)
      Sp cdd[3];
      for (int k = 0; k < 3; k++) cdd[k] = cross_motion(v, ld6(cdof + 6 * (rot + k)));
      for (int k = 0; k < 3; k++) a = sp_add(a, sp_scale(cdd[k], qvel[rot + k]));
      for (int k = 0; k < 3; k++) v = sp_add(v, sp_scale(ld6(cdof + 6 * (rot + k)), qvel[rot + k]));
    } else {
      Sp c = ld6(cdof + 6 * da);
      a = sp_add(a, sp_scale(cross_motion(v, c), qvel[da]));
      v = sp_add(v, sp_scale(c, qvel[da]));
    }
  }
  st6(ws + w.cvel + 6 * b, v);
  st6(ws + w.cacc + 6 * b, a);
  Sp hm = spi_mul(I, v);
  st6(ws + w.cfrc + 6 * b, sp_add(spi_mul(I, a), cross_force(v, hm)));
}

// Geom poses and world bounding boxes into tile scratch (forward.rs:84-89,
// 217-232): [pos 3, mat 9, aabb center 3, aabb half 3] per geom.
__device__ inline void geom_local_aabb(const DModel& m, const double* prm, int g, V3* c, V3* h) {
  V3 s = ld3(prm + m.p_size + 3 * g);
  *c = V3{0, 0, 0};
  switch (m.geom_type[g]) {
    case GEOM_PLANE: *h = V3{INFINITY, INFINITY, INFINITY}; break;
    case GEOM_SPHERE: *h = V3{s.x, s.x, s.x}; break;
    case GEOM_CAPSULE: *h = V3{s.x, s.x, s.x + s.y}; break;
    case GEOM_BOX: *h = s; break;
    case GEOM_CYLINDER: *h = V3{s.x, s.x, s.y}; break;
    default: {  // mesh: bounds of the hull vertices (model.rs:372-378)
      int id = m.geom_dataid[g];
      V3 lo{INFINITY, INFINITY, INFINITY}, hi{-INFINITY, -INFINITY, -INFINITY};
      for (int k = 0; k < m.hull_vnum[id]; k++) {
        V3 v = ld3(m.hull_vert + 3 * (m.hull_vadr[id] + k));
        lo = V3{fmin(lo.x, v.x), fmin(lo.y, v.y), fmin(lo.z, v.z)};
        hi = vmax(hi, v);
      }
      *c = (lo + hi) * 0.5;
      *h = (hi - lo) * 0.5;
    }
  }
}

template <int G>
__device__ void geom_poses(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e, double* gout) {
  const double* ws = e.ws;
  for (int g = T.lane(); g < m.ngeom; g += G) {
    int b = m.geom_body[g];
    M3 xm = q_mat(ld4(ws + w.xquat + 4 * b));
    V3 gp = ld3(ws + w.xpos + 3 * b) + mv(xm, ld3(m.geom_pos + 3 * g));
    M3 gm = mm(xm, q_mat(ld4(m.geom_quat + 4 * g)));
    double* o = gout + G_STRIDE * g;
    st3(o + G_POS, gp);
    st9(o + G_MAT, gm);
    V3 c, h;
    geom_local_aabb(m, e.prm, g, &c, &h);
    if (!isfinite(h.x)) {
      st3(o + G_AABB, V3{0, 0, 0});
      st3(o + G_AABB + 3, h);
    } else {
      st3(o + G_AABB, gp + mv(gm, c));
      st3(o + G_AABB + 3, V3{fabs(gm.m[0]) * h.x + fabs(gm.m[1]) * h.y + fabs(gm.m[2]) * h.z,
                             fabs(gm.m[3]) * h.x + fabs(gm.m[4]) * h.y + fabs(gm.m[5]) * h.z,
                             fabs(gm.m[6]) * h.x + fabs(gm.m[7]) * h.y + fabs(gm.m[8]) * h.z});
    }
  }
}

// Down the tree (positions, and with `dynamics` velocities and RNE forward
// terms), then geom poses into `gout`.
template <int G>
__device__ void tree_down(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e, bool dynamics,
                          double* gout) {
  double* ws = e.ws;
  int lane = T.lane();
  if (lane == 0) {
    st3(ws + w.xpos, V3{0, 0, 0});
    st4(ws + w.xquat, q_identity());
    if (dynamics) {
      st6(ws + w.cvel, sp_zero());
      st6(ws + w.cacc, Sp{V3{0, 0, 0}, -V3{m.gravity[0], m.gravity[1], m.gravity[2]}});
    }
  }
  T.sync();
  for (int L = 1; L < m.nlevel; L++) {
    for (int i = m.level_adr[L] + lane; i < m.level_adr[L + 1]; i += G) tree_down_body(m, w, e, m.level_body[i], dynamics);
    T.sync();
  }
  if (gout) {
    geom_poses(T, m, w, e, gout);
    T.sync();
  }
}

// Up the tree: crb (in place of cinert) and, with `dynamics`, the cfrc sums;
// then M = cdof' crb cdof along ancestor chains (+ armature) into qm (nv x nv,
// shared or global) and qfrc_bias = cdof' cfrc.
template <int G>
__device__ void tree_up(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e, bool dynamics,
                        double* qm) {
  double* ws = e.ws;
  int lane = T.lane(), nv = m.nv;
  double* crb = ws + w.cinert;
  double* cfrc = ws + w.cfrc;
  for (int L = m.nlevel - 2; L >= 1; L--) {
    for (int i = m.level_adr[L] + lane; i < m.level_adr[L + 1]; i += G) {
      int b = m.level_body[i];
      int c0 = m.child_adr[b], c1 = m.child_adr[b + 1];
      if (c0 == c1) continue;
      SpI acc = ld13(crb + 13 * b);
      for (int c = c0; c < c1; c++) {
        SpI k = ld13(crb + 13 * m.child_list[c]);
        acc.mass = acc.mass + k.mass;
        acc.mc = acc.mc + k.mc;
        for (int t = 0; t < 9; t++) acc.io.m[t] = acc.io.m[t] + k.io.m[t];
      }
      st13(crb + 13 * b, acc);
      if (dynamics) {
        Sp f = ld6(cfrc + 6 * b);
        for (int c = c0; c < c1; c++) f = sp_add(f, ld6(cfrc + 6 * m.child_list[c]));
        st6(cfrc + 6 * b, f);
      }
    }
    T.sync();
  }
  const double* cdof = ws + w.cdof;
  for (int k = lane; k < nv * nv; k += G) qm[k] = 0.0;
  T.sync();
  for (int i = lane; i < nv; i += G) {
    int bi = m.dof_body[i];
    Sp ci = ld6(cdof + 6 * i);
    Sp f = spi_mul(ld13(crb + 13 * bi), ci);
    for (int j = i; j != -1; j = m.dof_parent[j]) {
      double v = sp_dot(ld6(cdof + 6 * j), f);
      qm[i * nv + j] = v;
      qm[j * nv + i] = v;
    }
    qm[i * nv + i] += m.dof_armature[i];
    if (dynamics) ws[w.bias + i] = sp_dot(ci, ld6(cfrc + 6 * bi));
  }
  T.sync();
}

// forward.rs:173-211
template <int G>
__device__ void passive_actuation(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e) {
  double* ws = e.ws;
  int lane = T.lane();
  const double* qpos = ws + w.qpos;
  const double* qvel = ws + w.qvel;
  const double* prm = e.prm;
  double* pas = ws + w.passive;
  for (int k = lane; k < m.nv; k += G) pas[k] = -prm[m.p_damping + k] * qvel[k];
  T.sync();
  for (int j = lane; j < m.njnt; j += G) {
    double kp = m.jnt_stiffness[j];
    int t = m.jnt_type[j];
    if (kp != 0.0 && (t == JNT_HINGE || t == JNT_SLIDE))
      pas[m.jnt_dofadr[j]] -= kp * (qpos[m.jnt_qposadr[j]] - m.jnt_springref[j]);
  }
  double* force = ws + w.actforce;
  double* clamped = ws + w.actclamped;
  const double* ctrl = ws + w.ctrl;
  for (int u = lane; u < m.nu; u += G) {
    double gear = m.act_gear[u];
    int a0 = m.act_moment_adr[u], an = m.act_moment_num[u];
    double ls = 0.0, vs = 0.0;
    for (int k = 0; k < an; k++) ls += m.moment_coef[a0 + k] * qpos[m.jnt_qposadr[m.moment_jnt[a0 + k]]];
    for (int k = 0; k < an; k++) vs += m.moment_coef[a0 + k] * qvel[m.jnt_dofadr[m.moment_jnt[a0 + k]]];
    double length = gear * ls, vel = gear * vs;
    double c = ctrl[u];
    if (m.act_ctrllimited[u]) c = clampd(c, m.act_ctrlrange[2 * u], m.act_ctrlrange[2 * u + 1]);
    const double* bb = prm + m.p_bias + 3 * u;
    double f = prm[m.p_gain + u] * c + bb[0] + bb[1] * length + bb[2] * vel;
    bool cl = false;
    if (m.act_forcelimited[u]) {
      double lo = m.act_forcerange[2 * u], hi = m.act_forcerange[2 * u + 1];
      cl = f < lo || f > hi;
      f = clampd(f, lo, hi);
    }
    force[u] = f;
    clamped[u] = cl ? 1.0 : 0.0;
  }
  T.sync();
  double* actf = ws + w.actf;
  for (int k = lane; k < m.nv; k += G) {
    double s = 0.0;
    for (int i = m.dofact_adr[k]; i < m.dofact_adr[k + 1]; i++) {
      int u = m.dofact_u[i];
      s += m.act_gear[u] * m.dofact_coef[i] * force[u];
    }
    actf[k] = s;
  }
  T.sync();
}

}  // namespace pg
