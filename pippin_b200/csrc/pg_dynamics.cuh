// Smooth dynamics of one environment on a tile of G lanes: forward
// kinematics and cdof, CRBA, velocities + RNE bias forces, passive and
// actuator forces. Restates crates/pippin/src/forward.rs:14-211. Tree walks
// go level by level (bodies of one depth in parallel); sums over children
// run in decreasing body order, which is the order of the reference's
// reverse body loops, so composite inertias and forces add up identically.
#pragma once
#include "pg_math.cuh"
#include "pg_model.h"
#include "pg_tile.cuh"

namespace pg {

struct EnvCtx {
  double* ws;         // tile workspace (shared memory)
  const double* prm;  // this env's parameter block
  double* scr;        // tile scratch (global)
  int env;
};

// forward.rs:14-90 for one body, given its parent's pose
__device__ inline void fk_body(const DModel& m, const WsLayout& w, const EnvCtx& e, int b) {
  double* ws = e.ws;
  const double* q = ws + w.qpos;
  int p = m.body_parent[b];
  M3 xmp = ld9(ws + w.xmat + 9 * p);
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
      V3 jp = ld3(m.jnt_pos + 3 * j), ja = ld3(m.jnt_axis + 3 * j);
      V3 axis = q_rot(quat, ja);
      (void)jp;
      pos = pos + axis * (q[qa] - m.qpos0[qa]);
      st6(cdof + 6 * da, Sp{V3{0, 0, 0}, axis});
    }
  }
  quat = q_normalized(quat);
  M3 xm = q_mat(quat);
  st3(ws + w.xpos + 3 * b, pos);
  st4(ws + w.xquat + 4 * b, quat);
  st9(ws + w.xmat + 9 * b, xm);
  const double* prm = e.prm;
  V3 xipos = pos + mv(xm, ld3(prm + m.p_ipos + 3 * b));
  st3(ws + w.xipos + 3 * b, xipos);
  SpI ci = spi_from_com(prm[m.p_mass + b], xipos, mrot(ld9(prm + m.p_inertia + 9 * b), xm));
  st13(ws + w.cinert + 13 * b, ci);
}

template <int G>
__device__ void kinematics(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e) {
  double* ws = e.ws;
  int lane = T.lane();
  if (lane == 0) {
    st3(ws + w.xpos, V3{0, 0, 0});
    st4(ws + w.xquat, q_identity());
    st9(ws + w.xmat, m3_identity());
    st3(ws + w.xipos, V3{0, 0, 0});
  }
  T.sync();
  for (int L = 1; L < m.nlevel; L++) {
    for (int i = m.level_adr[L] + lane; i < m.level_adr[L + 1]; i += G) fk_body(m, w, e, m.level_body[i]);
    T.sync();
  }
  for (int g = lane; g < m.ngeom; g += G) {
    int b = m.geom_body[g];
    M3 xm = ld9(ws + w.xmat + 9 * b);
    st3(ws + w.gxpos + 3 * g, ld3(ws + w.xpos + 3 * b) + mv(xm, ld3(m.geom_pos + 3 * g)));
    st9(ws + w.gxmat + 9 * g, mm(xm, q_mat(ld4(m.geom_quat + 4 * g))));
  }
  T.sync();
}

// forward.rs:93-112
template <int G>
__device__ void crba(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e) {
  double* ws = e.ws;
  int lane = T.lane(), nv = m.nv;
  double* crb = ws + w.crb;
  const double* cin = ws + w.cinert;
  for (int L = m.nlevel - 1; L >= 1; L--) {
    for (int i = m.level_adr[L] + lane; i < m.level_adr[L + 1]; i += G) {
      int b = m.level_body[i];
      SpI acc = ld13(cin + 13 * b);
      for (int c = m.child_adr[b]; c < m.child_adr[b + 1]; c++) {
        SpI k = ld13(crb + 13 * m.child_list[c]);
        acc.mass = acc.mass + k.mass;
        acc.mc = acc.mc + k.mc;
        for (int t = 0; t < 9; t++) acc.io.m[t] = acc.io.m[t] + k.io.m[t];
      }
      st13(crb + 13 * b, acc);
    }
    T.sync();
  }
  double* qm = ws + w.qm;
  for (int k = lane; k < nv * nv; k += G) qm[k] = 0.0;
  T.sync();
  const double* cdof = ws + w.cdof;
  for (int i = lane; i < nv; i += G) {
    Sp f = spi_mul(ld13(crb + 13 * m.dof_body[i]), ld6(cdof + 6 * i));
    int j = i;
    while (j != -1) {
      double v = sp_dot(ld6(cdof + 6 * j), f);
      qm[i * nv + j] = v;
      qm[j * nv + i] = v;
      j = m.dof_parent[j];
    }
    qm[i * nv + i] += m.dof_armature[i];
  }
  T.sync();
}

// forward.rs:115-171 (velocity and RNE share one pass down the tree)
template <int G>
__device__ void velocity_rne(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e) {
  double* ws = e.ws;
  int lane = T.lane();
  const double* qvel = ws + w.qvel;
  const double* cdof = ws + w.cdof;
  double* cdd = ws + w.cdof_dot;
  double* cvel = ws + w.cvel;
  double* cacc = ws + w.cacc;
  double* cfrc = ws + w.cfrc;
  if (lane == 0) {
    st6(cvel, sp_zero());
    st6(cacc, Sp{V3{0, 0, 0}, -V3{m.gravity[0], m.gravity[1], m.gravity[2]}});
    st6(cfrc, sp_zero());
  }
  T.sync();
  for (int L = 1; L < m.nlevel; L++) {
    for (int i = m.level_adr[L] + lane; i < m.level_adr[L + 1]; i += G) {
      int b = m.level_body[i];
      int p = m.body_parent[b];
      Sp v = ld6(cvel + 6 * p);
      for (int j = m.body_jntadr[b]; j < m.body_jntadr[b] + m.body_jntnum[b]; j++) {
        int da = m.jnt_dofadr[j], type = m.jnt_type[j];
        if (type == JNT_FREE || type == JNT_BALL) {
          int lin = type == JNT_FREE ? 3 : 0;
          int rot = type == JNT_FREE ? da + 3 : da;
          for (int k = 0; k < lin; k++) {
            st6(cdd + 6 * (da + k), sp_zero());
            v = sp_add(v, sp_scale(ld6(cdof + 6 * (da + k)), qvel[da + k]));
          }
          // all rotational dofs share one velocity (forward.rs:130-133)
          for (int k = 0; k < 3; k++) st6(cdd + 6 * (rot + k), cross_motion(v, ld6(cdof + 6 * (rot + k))));
          for (int k = 0; k < 3; k++) v = sp_add(v, sp_scale(ld6(cdof + 6 * (rot + k)), qvel[rot + k]));
        } else {
          st6(cdd + 6 * da, cross_motion(v, ld6(cdof + 6 * da)));
          v = sp_add(v, sp_scale(ld6(cdof + 6 * da), qvel[da]));
        }
      }
      st6(cvel + 6 * b, v);
      Sp a = ld6(cacc + 6 * p);
      for (int k = m.body_dofadr[b]; k < m.body_dofadr[b] + m.body_dofnum[b]; k++)
        a = sp_add(a, sp_scale(ld6(cdd + 6 * k), qvel[k]));
      st6(cacc + 6 * b, a);
      SpI I = ld13(ws + w.cinert + 13 * b);
      Sp h = spi_mul(I, v);
      st6(cfrc + 6 * b, sp_add(spi_mul(I, a), cross_force(v, h)));
    }
    T.sync();
  }
  for (int L = m.nlevel - 2; L >= 1; L--) {
    for (int i = m.level_adr[L] + lane; i < m.level_adr[L + 1]; i += G) {
      int b = m.level_body[i];
      Sp f = ld6(cfrc + 6 * b);
      for (int c = m.child_adr[b]; c < m.child_adr[b + 1]; c++) f = sp_add(f, ld6(cfrc + 6 * m.child_list[c]));
      st6(cfrc + 6 * b, f);
    }
    T.sync();
  }
  double* bias = ws + w.bias;
  for (int k = lane; k < m.nv; k += G) bias[k] = sp_dot(ld6(cdof + 6 * k), ld6(cfrc + 6 * m.dof_body[k]));
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
