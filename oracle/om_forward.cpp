// Oracle (test infrastructure only): smooth dynamics and time stepping.
// Restates crates/pippin/src/forward.rs line by line (operation order kept).
// OM_FLOPS lines count the FP64 operations of each routine as written.
#include <algorithm>

#include "om_model.h"

namespace om {

// flop counts of the small kernels (adds, subs, muls, divs as written)
enum : int {
  F_DOT3 = 5, F_CROSS = 9, F_MV = 15, F_MM = 45, F_QMAT = 31, F_QMUL = 28, F_SPI_COM = 66, F_ROT = 90,
  F_SPI_MUL = 42, F_SPDOT = 11, F_CRM = 30, F_PV = 12
};

// forward.rs:14-90
void kinematics(const Model& m, Data& d) {
  d.xpos[0] = v3zero();
  d.xquat[0] = qidentity();
  d.xmat[0] = m3identity();
  d.xipos[0] = v3zero();
  const Real* q = d.qpos.data();
  for (int b = 1; b < m.nbody(); b++) {
    int p = m.body_parent[b];
    Vec3 pos = d.xpos[p] + mul_vec(d.xmat[p], m.body_pos[b]);
    Quat quat = qmul(d.xquat[p], m.body_quat[b]);
    OM_FLOPS(ST_KIN, 3 + F_MV + F_QMUL);
    for (int j = m.body_jntadr[b]; j < m.body_jntadr[b] + m.body_jntnum[b]; j++) {
      int qa = m.jnt_qposadr[j], da = m.jnt_dofadr[j];
      switch (m.jnt_type[j]) {
        case JNT_FREE: {
          pos = v3(q[qa], q[qa + 1], q[qa + 2]);
          quat = qnormalized(Quat{{q[qa + 3], q[qa + 4], q[qa + 5], q[qa + 6]}});
          d.xanchor[j] = pos;
          d.xaxis[j] = v3(0, 0, 1);
          Mat3 r = qto_mat(quat);
          for (int k = 0; k < 3; k++) {
            Vec3 e = v3zero();
            e[k] = 1.0;
            d.cdof[da + k] = sp(v3zero(), e);
            Vec3 a = col(r, k);
            d.cdof[da + 3 + k] = sp(a, cross(pos, a));
          }
          OM_FLOPS(ST_KIN, 12 + F_QMAT + 3 * F_CROSS);
          break;
        }
        case JNT_BALL: {
          Vec3 anchor = pos + qrotate(quat, m.jnt_pos[j]);
          Quat ql = qnormalized(Quat{{q[qa], q[qa + 1], q[qa + 2], q[qa + 3]}});
          quat = qmul(quat, ql);
          pos = anchor - qrotate(quat, m.jnt_pos[j]);
          d.xanchor[j] = anchor;
          d.xaxis[j] = v3(0, 0, 1);
          Mat3 r = qto_mat(quat);
          for (int k = 0; k < 3; k++) {
            Vec3 a = col(r, k);
            d.cdof[da + k] = sp(a, cross(anchor, a));
          }
          OM_FLOPS(ST_KIN, 3 * F_QMAT + 2 * F_MV + 6 + 12 + F_QMUL + 3 * F_CROSS);
          break;
        }
        case JNT_HINGE: {
          Vec3 anchor = pos + qrotate(quat, m.jnt_pos[j]);
          Vec3 axis = qrotate(quat, m.jnt_axis[j]);
          quat = qmul(quat, qaxis_angle(m.jnt_axis[j], q[qa] - m.qpos0[qa]));
          pos = anchor - qrotate(quat, m.jnt_pos[j]);
          d.xanchor[j] = anchor;
          d.xaxis[j] = axis;
          d.cdof[da] = sp(axis, cross(anchor, axis));
          OM_FLOPS(ST_KIN, 3 * F_QMAT + 3 * F_MV + 6 + F_QMUL + 14 + F_CROSS);
          break;
        }
        case JNT_SLIDE: {
          Vec3 anchor = pos + qrotate(quat, m.jnt_pos[j]);
          Vec3 axis = qrotate(quat, m.jnt_axis[j]);
          pos += axis * (q[qa] - m.qpos0[qa]);
          d.xanchor[j] = anchor;
          d.xaxis[j] = axis;
          d.cdof[da] = sp(v3zero(), axis);
          OM_FLOPS(ST_KIN, 2 * F_QMAT + 2 * F_MV + 3 + 7);
          break;
        }
      }
    }
    quat = qnormalized(quat);
    d.xpos[b] = pos;
    d.xquat[b] = quat;
    d.xmat[b] = qto_mat(quat);
    d.xipos[b] = pos + mul_vec(d.xmat[b], m.body_ipos[b]);
    d.cinert[b] = spi_from_com(m.body_mass[b], d.xipos[b], mrotate(m.body_inertia[b], d.xmat[b]));
    OM_FLOPS(ST_KIN, 12 + F_QMAT + 3 + F_MV + F_ROT + F_SPI_COM);
  }
  for (int g = 0; g < m.ngeom(); g++) {
    int b = m.geom_body[g];
    d.geom_xpos[g] = d.xpos[b] + mul_vec(d.xmat[b], m.geom_pos[g]);
    d.geom_xmat[g] = mul_mat(d.xmat[b], qto_mat(m.geom_quat[g]));
    OM_FLOPS(ST_KIN, 3 + F_MV + F_MM + F_QMAT);
  }
}

// forward.rs:93-112
void crba(const Model& m, Data& d) {
  int nv = m.nv;
  d.crb = d.cinert;
  for (int b = m.nbody() - 1; b >= 1; b--) {
    int p = m.body_parent[b];
    d.crb[p] = spi_add(d.crb[p], d.crb[b]);
    OM_FLOPS(ST_CRBA, 13);
  }
  std::fill(d.qm.begin(), d.qm.end(), 0.0);
  for (int i = 0; i < nv; i++) {
    Spatial f = spi_mul(d.crb[m.dof_body[i]], d.cdof[i]);
    OM_FLOPS(ST_CRBA, F_SPI_MUL);
    int j = i;
    while (j != -1) {
      Real v = spdot(d.cdof[j], f);
      d.qm[(size_t)i * nv + j] = v;
      d.qm[(size_t)j * nv + i] = v;
      j = m.dof_parent[j];
      OM_FLOPS(ST_CRBA, F_SPDOT);
    }
    d.qm[(size_t)i * nv + i] += m.dof_armature[i];
    OM_FLOPS(ST_CRBA, 1);
  }
}

// forward.rs:115-144
void velocity(const Model& m, Data& d) {
  d.cvel[0] = spzero();
  for (int b = 1; b < m.nbody(); b++) {
    Spatial v = d.cvel[m.body_parent[b]];
    for (int j = m.body_jntadr[b]; j < m.body_jntadr[b] + m.body_jntnum[b]; j++) {
      int da = m.jnt_dofadr[j];
      int t = m.jnt_type[j];
      if (t == JNT_FREE || t == JNT_BALL) {
        int lin = t == JNT_FREE ? 3 : 0;
        int rot = t == JNT_FREE ? da + 3 : da;
        for (int k = 0; k < lin; k++) {
          d.cdof_dot[da + k] = spzero();
          v = spadd(v, spscale(d.cdof[da + k], d.qvel[da + k]));
        }
        // all rotational dofs share the same velocity (forward.rs:130-133)
        for (int k = 0; k < 3; k++) d.cdof_dot[rot + k] = cross_motion(v, d.cdof[rot + k]);
        for (int k = 0; k < 3; k++) v = spadd(v, spscale(d.cdof[rot + k], d.qvel[rot + k]));
        OM_FLOPS(ST_RNE, lin * 12 + 3 * F_CRM + 36);
      } else {
        d.cdof_dot[da] = cross_motion(v, d.cdof[da]);
        v = spadd(v, spscale(d.cdof[da], d.qvel[da]));
        OM_FLOPS(ST_RNE, F_CRM + 12);
      }
    }
    d.cvel[b] = v;
  }
}

// forward.rs:147-171
void rne(const Model& m, Data& d) {
  int nb = m.nbody();
  d.cacc.assign(nb, spzero());
  d.cfrc.assign(nb, spzero());
  d.cacc[0] = sp(v3zero(), -m.gravity);
  d.cfrc[0] = spzero();
  for (int b = 1; b < nb; b++) {
    Spatial a = d.cacc[m.body_parent[b]];
    for (int k = m.body_dofadr[b]; k < m.body_dofadr[b] + m.body_dofnum[b]; k++) {
      a = spadd(a, spscale(d.cdof_dot[k], d.qvel[k]));
      OM_FLOPS(ST_RNE, 12);
    }
    d.cacc[b] = a;
    Spatial h = spi_mul(d.cinert[b], d.cvel[b]);
    d.cfrc[b] = spadd(spi_mul(d.cinert[b], a), cross_force(d.cvel[b], h));
    OM_FLOPS(ST_RNE, 2 * F_SPI_MUL + F_CRM + 6);
  }
  for (int b = nb - 1; b >= 1; b--) {
    int p = m.body_parent[b];
    Spatial f = d.cfrc[b];
    d.cfrc[p] = spadd(d.cfrc[p], f);
    OM_FLOPS(ST_RNE, 6);
  }
  for (int k = 0; k < m.nv; k++) {
    d.qfrc_bias[k] = spdot(d.cdof[k], d.cfrc[m.dof_body[k]]);
    OM_FLOPS(ST_RNE, F_SPDOT);
  }
}

// forward.rs:173-183
void passive(const Model& m, Data& d) {
  for (int k = 0; k < m.nv; k++) d.qfrc_passive[k] = -m.dof_damping[k] * d.qvel[k];
  OM_FLOPS(ST_PASSACT, m.nv);
  for (int j = 0; j < m.njnt(); j++) {
    Real kp = m.jnt_stiffness[j];
    if (kp != 0.0 && (m.jnt_type[j] == JNT_HINGE || m.jnt_type[j] == JNT_SLIDE)) {
      d.qfrc_passive[m.jnt_dofadr[j]] -= kp * (d.qpos[m.jnt_qposadr[j]] - m.jnt_springref[j]);
      OM_FLOPS(ST_PASSACT, 3);
    }
  }
}

// forward.rs:185-211
void actuation(const Model& m, Data& d) {
  std::fill(d.qfrc_actuator.begin(), d.qfrc_actuator.end(), 0.0);
  for (int u = 0; u < m.nu; u++) {
    Real gear = m.actuator_gear[u];
    const auto& moment = m.actuator_moment[u];
    Real ls = 0.0, vs = 0.0;
    for (auto& jc : moment) ls += jc.second * d.qpos[m.jnt_qposadr[jc.first]];
    for (auto& jc : moment) vs += jc.second * d.qvel[m.jnt_dofadr[jc.first]];
    Real length = gear * ls, vel = gear * vs;
    Real ctrl = d.ctrl[u];
    if (m.actuator_ctrllimited[u]) ctrl = clampr(ctrl, m.actuator_ctrlrange[u][0], m.actuator_ctrlrange[u][1]);
    const auto& bb = m.actuator_bias[u];
    Real f = m.actuator_gain[u] * ctrl + bb[0] + bb[1] * length + bb[2] * vel;
    bool clamped = false;
    if (m.actuator_forcelimited[u]) {
      Real lo = m.actuator_forcerange[u][0], hi = m.actuator_forcerange[u][1];
      clamped = f < lo || f > hi;
      f = clampr(f, lo, hi);
    }
    d.actuator_force[u] = f;
    d.actuator_clamped[u] = clamped;
    for (auto& jc : moment) d.qfrc_actuator[m.jnt_dofadr[jc.first]] += gear * jc.second * f;
    OM_FLOPS(ST_PASSACT, 4 * moment.size() + 2 + 6 + 3 * moment.size());
  }
}

// forward.rs:214-260
void collide(const Model& m, Data& d) {
  d.contacts.clear();
  Real margin = m.solver.contact_margin;
  int ng = m.ngeom();
  std::vector<std::array<Vec3, 2>> aabb(ng);
  for (int g = 0; g < ng; g++) {
    Vec3 c = m.geom_aabb[g][0], h = m.geom_aabb[g][1];
    const Mat3& r = d.geom_xmat[g];
    if (!std::isfinite(h[0])) {
      aabb[g] = {v3zero(), h};
      continue;
    }
    Vec3 center = d.geom_xpos[g] + mul_vec(r, c);
    Vec3 half = v3(std::fabs(r[0]) * h[0] + std::fabs(r[1]) * h[1] + std::fabs(r[2]) * h[2],
                   std::fabs(r[3]) * h[0] + std::fabs(r[4]) * h[1] + std::fabs(r[5]) * h[2],
                   std::fabs(r[6]) * h[0] + std::fabs(r[7]) * h[1] + std::fabs(r[8]) * h[2]);
    aabb[g] = {center, half};
    OM_FLOPS(ST_COLLIDE, 18 + 15);
  }
  std::vector<Hit> hits;
  for (auto& pr : m.collision_pairs) {
    int g1 = pr.first, g2 = pr.second;
    Vec3 c1 = aabb[g1][0], h1 = aabb[g1][1], c2 = aabb[g2][0], h2 = aabb[g2][1];
    bool sep = false;
    for (int k = 0; k < 3; k++)
      if (std::fabs(c1[k] - c2[k]) > h1[k] + h2[k] + margin) {
        sep = true;
        break;
      }
    OM_FLOPS(ST_COLLIDE, 12);
    if (sep) continue;
    auto pose = [&](int g) {
      return GeomPose{m.geom_type[g], d.geom_xpos[g], d.geom_xmat[g], m.geom_size[g],
                      m.geom_type[g] == GEOM_MESH ? &m.mesh_hull[m.geom_dataid[g]] : nullptr};
    };
    hits.clear();
    if (needs_general(m.geom_type[g1], m.geom_type[g2]))
      collide_general(pose(g1), pose(g2), margin, hits);
    else
      collide_pair(pose(g1), pose(g2), margin, hits);
    for (size_t i = 0; i < hits.size(); i++) {
      Contact c;
      c.pos = hits[i].pos;
      c.normal = hits[i].normal;
      c.tangent = hits[i].tangent;
      c.depth = hits[i].depth;
      c.geom[0] = g1;
      c.geom[1] = g2;
      c.feature = (uint32_t)i;
      d.contacts.push_back(c);
    }
  }
}

// forward.rs:263-271
void forward(const Model& m, Data& d) {
  kinematics(m, d);
  crba(m, d);
  velocity(m, d);
  rne(m, d);
  passive(m, d);
  actuation(m, d);
  collide(m, d);
}

// forward.rs:275-333: MuJoCo's invweight0 at the reference configuration
void set_const(Model& m) {
  Data d;
  data_init(m, d);
  kinematics(m, d);
  crba(m, d);
  int nv = m.nv;
  m.dof_invweight.assign(nv, 0.0);
  m.body_invweight.assign(m.nbody(), {0.0, 0.0});
  if (nv == 0) return;
  std::vector<Real> l = d.qm;
  if (!cholesky(l.data(), nv)) return;
  std::vector<Real> x(nv), e(nv), row(nv);
  auto quad = [&](const std::vector<Real>& r) {
    x = r;
    cholesky_solve(l.data(), nv, x.data());
    Real s = 0.0;
    for (int k = 0; k < nv; k++) s += r[k] * x[k];
    return s;
  };
  for (int k = 0; k < nv; k++) {
    std::fill(e.begin(), e.end(), 0.0);
    e[k] = 1.0;
    m.dof_invweight[k] = quad(e);
  }
  for (int j = 0; j < m.njnt(); j++) {
    int da = m.jnt_dofadr[j];
    int ng = 0, groups[2];
    if (m.jnt_type[j] == JNT_FREE) {
      groups[0] = 0;
      groups[1] = 3;
      ng = 2;
    } else if (m.jnt_type[j] == JNT_BALL) {
      groups[0] = 0;
      ng = 1;
    }
    for (int gi = 0; gi < ng; gi++) {
      int g = groups[gi];
      Real avg = (m.dof_invweight[da + g] + m.dof_invweight[da + g + 1] + m.dof_invweight[da + g + 2]) / 3.0;
      for (int i = 0; i < 3; i++) m.dof_invweight[da + g + i] = avg;
    }
  }
  for (int b = 1; b < m.nbody(); b++) {
    Real w[2] = {0.0, 0.0};
    for (int axis = 0; axis < 3; axis++) {
      Vec3 dir = v3zero();
      dir[axis] = 1.0;
      for (int kind = 0; kind < 2; kind++) {
        std::fill(row.begin(), row.end(), 0.0);
        int k = m.body_lastdof[b];
        while (k != -1) {
          const Spatial& c = d.cdof[k];
          row[k] = kind == 0 ? dot(dir, point_velocity(c, d.xipos[b])) : dot(dir, c.ang);
          k = m.dof_parent[k];
        }
        w[kind] += quad(row) / 3.0;
      }
    }
    m.body_invweight[b] = {w[0], w[1]};
  }
}

// forward.rs:407-431
static bool is_ancestor(const Model& m, int a, int b) {
  int k = m.dof_parent[b];
  while (k != -1) {
    if (k == a) return true;
    k = m.dof_parent[k];
  }
  return false;
}

static void add_implicit_terms(const Model& m, const std::vector<char>& clamped, Real h, Real* mat) {
  int nv = m.nv;
  for (int k = 0; k < nv; k++) mat[(size_t)k * nv + k] += h * m.dof_damping[k];
  OM_FLOPS(ST_FACTOR, 2 * nv);
  if (m.integrator == INT_IMPLICITFAST) {
    for (int u = 0; u < m.nu; u++) {
      Real kv = -m.actuator_bias[u][2] * m.actuator_gear[u] * m.actuator_gear[u];
      if (kv == 0.0 || clamped[u]) continue;
      for (auto& A : m.actuator_moment[u])
        for (auto& B : m.actuator_moment[u]) {
          int a = m.jnt_dofadr[A.first], b = m.jnt_dofadr[B.first];
          if (a == b || is_ancestor(m, a, b) || is_ancestor(m, b, a)) {
            mat[(size_t)a * nv + b] += h * kv * A.second * B.second;
            OM_FLOPS(ST_FACTOR, 4);
          }
        }
    }
  }
}

// forward.rs:454-456
static bool has_implicit_terms(const Model& m) {
  for (Real b : m.dof_damping)
    if (b != 0.0) return true;
  if (m.integrator == INT_IMPLICITFAST)
    for (auto& b : m.actuator_bias)
      if (b[2] != 0.0) return true;
  return false;
}

[[maybe_unused]] static Real chol_flops(int n) { return (Real)n * n * n / 3.0 + (Real)n * n; }
[[maybe_unused]] static Real solve_flops(int n) { return 2.0 * n * n; }

// forward.rs:392-401; a non-positive-definite mass matrix sets status 2
// (the reference panics there)
static bool factor_mass(const Model& m, Data& d, Real h) {
  int nv = m.nv;
  d.qm_chol = d.qm;
  add_implicit_terms(m, d.actuator_clamped, h, d.qm_chol.data());
  for (auto& r : m.dof_blocks) {
    OM_FLOPS(ST_FACTOR, chol_flops(r.second - r.first));
    if (!cholesky_block(d.qm_chol.data(), nv, r.first, r.second)) {
      d.status = 2;
      return false;
    }
  }
  return true;
}

// forward.rs:434-438
void mass_solve(const Model& m, const Real* l, Real* x) {
  for (auto& r : m.dof_blocks) {
    cholesky_solve_block(l, m.nv, r.first, r.second, x);
    OM_FLOPS(ST_FACTOR, solve_flops(r.second - r.first));
  }
}

// forward.rs:336-389
void step(const Model& m, Data& d) {
  forward(m, d);
  int nv = m.nv;
  Real h = m.timestep;
  bool damped = has_implicit_terms(m);
  d.smooth.resize(nv);
  for (int k = 0; k < nv; k++) d.smooth[k] = d.qfrc_passive[k] + d.qfrc_actuator[k] + d.qfrc_applied[k] - d.qfrc_bias[k];
  OM_FLOPS(ST_PASSACT, 3 * nv);
  std::vector<Real>& acc = d.tmp_nv;
  acc = d.smooth;
  std::vector<Real>& v = d.v;
  std::vector<Real>& v_pos = d.v_pos;
  v.clear();
  if (m.solver.kind == SOLVER_NEWTON) {
    if (!factor_mass(m, d, 0.0)) return;
    mass_solve(m, d.qm_chol.data(), acc.data());
    newton_solve(m, d, acc.data());
    if (damped) {
      if (!factor_mass(m, d, h)) return;
      for (int k = 0; k < nv; k++) acc[k] = d.smooth[k] + d.qfrc_constraint[k];
      OM_FLOPS(ST_FACTOR, nv);
      mass_solve(m, d.qm_chol.data(), acc.data());
    }
    v.resize(nv);
    for (int k = 0; k < nv; k++) v[k] = d.qvel[k] + h * acc[k];
    v_pos = v;
  } else {
    if (!factor_mass(m, d, h)) return;
    mass_solve(m, d.qm_chol.data(), acc.data());
    v.resize(nv);
    for (int k = 0; k < nv; k++) v[k] = d.qvel[k] + h * acc[k];
    pgs_solve(m, d, v.data(), v_pos);
  }
  OM_FLOPS(ST_INTEGRATE, 2 * nv);
  for (int k = 0; k < nv; k++) d.qacc[k] = (v[k] - d.qvel[k]) / h;
  OM_FLOPS(ST_INTEGRATE, 2 * nv);
  integrate_pos(m, d.qpos.data(), v_pos.data(), h);
  d.qvel = v;
  d.time += h;
}

// forward.rs:459-480
void integrate_pos(const Model& m, Real* qpos, const Real* qvel, Real h) {
  for (int j = 0; j < m.njnt(); j++) {
    int qa = m.jnt_qposadr[j], da = m.jnt_dofadr[j];
    switch (m.jnt_type[j]) {
      case JNT_FREE: {
        for (int k = 0; k < 3; k++) qpos[qa + k] += h * qvel[da + k];
        Quat q{{qpos[qa + 3], qpos[qa + 4], qpos[qa + 5], qpos[qa + 6]}};
        Vec3 w = v3(qvel[da + 3], qvel[da + 4], qvel[da + 5]);
        Quat r = qintegrate_local(q, w, h);
        for (int k = 0; k < 4; k++) qpos[qa + 3 + k] = r[k];
        OM_FLOPS(ST_INTEGRATE, 6 + 6 + 2 + 6 + F_QMUL + 12);
        break;
      }
      case JNT_BALL: {
        Quat q{{qpos[qa], qpos[qa + 1], qpos[qa + 2], qpos[qa + 3]}};
        Vec3 w = v3(qvel[da], qvel[da + 1], qvel[da + 2]);
        Quat r = qintegrate_local(q, w, h);
        for (int k = 0; k < 4; k++) qpos[qa + k] = r[k];
        OM_FLOPS(ST_INTEGRATE, 6 + 2 + 6 + F_QMUL + 12);
        break;
      }
      default:
        qpos[qa] += h * qvel[da];
        OM_FLOPS(ST_INTEGRATE, 2);
    }
  }
}

}  // namespace om
