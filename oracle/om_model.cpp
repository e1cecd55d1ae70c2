// Oracle (test infrastructure only): model blob reader, data init/reset and
// per-env parameters. Restates crates/pippin/src/model.rs:279-451,
// crates/pippin/src/data.rs:83-131 and crates/pippin/src/params.rs:61-177.
#include <cstring>
#include <map>

#include "om_model.h"

namespace om {

thread_local double g_flops[ST_COUNT];

namespace {

struct Entry {
  uint32_t dtype;
  uint64_t count;
  const uint8_t* data;
};

struct Blob {
  std::map<std::string, Entry> arrays;
  std::string err;

  bool parse(const void* p, size_t bytes) {
    const uint8_t* b = (const uint8_t*)p;
    if (bytes < 16 || std::memcmp(b, "PGBLOB01", 8) != 0) {
      err = "bad model blob magic";
      return false;
    }
    uint32_t version, n;
    std::memcpy(&version, b + 8, 4);
    std::memcpy(&n, b + 12, 4);
    if (version != 1) {
      err = "unsupported model blob version";
      return false;
    }
    if (16 + (uint64_t)n * 64 > bytes) {
      err = "truncated model blob directory";
      return false;
    }
    for (uint32_t i = 0; i < n; i++) {
      const uint8_t* e = b + 16 + 64 * (size_t)i;
      char name[41];
      std::memcpy(name, e, 40);
      name[40] = 0;
      Entry en;
      std::memcpy(&en.dtype, e + 40, 4);
      uint64_t off;
      std::memcpy(&en.count, e + 48, 8);
      std::memcpy(&off, e + 56, 8);
      uint64_t esize = en.dtype == 3 ? 1 : 8;
      if (en.dtype < 1 || en.dtype > 3 || off % 8 != 0 || off + en.count * esize > bytes) {
        err = std::string("bad model blob entry ") + name;
        return false;
      }
      en.data = b + off;
      arrays[name] = en;
    }
    return true;
  }
  const Entry* find(const char* name, uint32_t dtype) {
    auto it = arrays.find(name);
    if (it == arrays.end()) return nullptr;
    if (it->second.dtype != dtype) return nullptr;
    return &it->second;
  }
  bool f64(const char* name, std::vector<Real>& out, long expect = -1) {
    const Entry* e = find(name, 1);
    if (!e || (expect >= 0 && (long)e->count != expect)) {
      if (err.empty()) err = std::string("model blob: missing or mis-sized f64 array ") + name;
      return false;
    }
    out.resize(e->count);
    std::memcpy(out.data(), e->data, 8 * e->count);
    return true;
  }
  bool i64(const char* name, std::vector<int64_t>& out, long expect = -1) {
    const Entry* e = find(name, 2);
    if (!e || (expect >= 0 && (long)e->count != expect)) {
      if (err.empty()) err = std::string("model blob: missing or mis-sized i64 array ") + name;
      return false;
    }
    out.resize(e->count);
    std::memcpy(out.data(), e->data, 8 * e->count);
    return true;
  }
};

template <class T>
void to_int(const std::vector<int64_t>& src, std::vector<T>& dst) {
  dst.resize(src.size());
  for (size_t i = 0; i < src.size(); i++) dst[i] = (T)src[i];
}
void to_vec3(const std::vector<Real>& s, std::vector<Vec3>& d) {
  d.resize(s.size() / 3);
  for (size_t i = 0; i < d.size(); i++) d[i] = v3(s[3 * i], s[3 * i + 1], s[3 * i + 2]);
}
void to_quat(const std::vector<Real>& s, std::vector<Quat>& d) {
  d.resize(s.size() / 4);
  for (size_t i = 0; i < d.size(); i++) d[i] = Quat{{s[4 * i], s[4 * i + 1], s[4 * i + 2], s[4 * i + 3]}};
}
template <size_t N>
void to_arr(const std::vector<Real>& s, std::vector<std::array<Real, N>>& d) {
  d.resize(s.size() / N);
  for (size_t i = 0; i < d.size(); i++)
    for (size_t k = 0; k < N; k++) d[i][k] = s[N * i + k];
}

}  // namespace

std::shared_ptr<Model> load_blob(const void* p, size_t bytes, std::string* err) {
  Blob b;
  auto fail = [&]() -> std::shared_ptr<Model> {
    if (err) *err = b.err.empty() ? "model blob is inconsistent" : b.err;
    return nullptr;
  };
  if (!b.parse(p, bytes)) return fail();
  auto mp = std::make_shared<Model>();
  Model& m = *mp;
  std::vector<Real> f;
  std::vector<int64_t> ii;

  if (!b.f64("timestep", f, 1)) return fail();
  m.timestep = f[0];
  if (!b.f64("gravity", f, 3)) return fail();
  m.gravity = v3(f[0], f[1], f[2]);
  if (!b.i64("integrator", ii, 1)) return fail();
  m.integrator = (int)ii[0];
  if (!b.i64("opt_solver", ii, 1)) return fail();
  m.solver.kind = (int)ii[0];
  if (!b.i64("opt_iterations", ii, 1)) return fail();
  m.solver.iterations = (int)ii[0];
  if (!b.f64("opt_tolerance", f, 1)) return fail();
  m.solver.tolerance = f[0];
  if (!b.f64("opt_margin", f, 1)) return fail();
  m.solver.contact_margin = f[0];
  if (!b.f64("opt_solref", f, 2)) return fail();
  m.solver.solref[0] = f[0];
  m.solver.solref[1] = f[1];
  if (!b.f64("opt_solimp", f, 5)) return fail();
  for (int k = 0; k < 5; k++) m.solver.solimp[k] = f[k];
  if (!b.f64("opt_impratio", f, 1)) return fail();
  m.solver.impratio = f[0];
  if (!b.f64("opt_hertz", f, 1)) return fail();
  m.solver.contact_hertz = f[0];
  if (!b.f64("opt_dampratio", f, 1)) return fail();
  m.solver.contact_damping_ratio = f[0];
  if (!b.f64("opt_slop", f, 1)) return fail();
  m.solver.contact_slop = f[0];

  std::vector<int64_t> dims;
  if (!b.i64("dims", dims, 9)) return fail();
  m.nq = (int)dims[0];
  m.nv = (int)dims[1];
  m.nu = (int)dims[2];
  long nb = dims[3], nj = dims[4], ng = dims[5], nc = dims[6], ne = dims[7], nmesh = dims[8];

  if (!b.i64("body_parent", ii, nb)) return fail();
  to_int(ii, m.body_parent);
  if (!b.i64("body_jntadr", ii, nb)) return fail();
  to_int(ii, m.body_jntadr);
  if (!b.i64("body_jntnum", ii, nb)) return fail();
  to_int(ii, m.body_jntnum);
  if (!b.i64("body_dofadr", ii, nb)) return fail();
  to_int(ii, m.body_dofadr);
  if (!b.i64("body_dofnum", ii, nb)) return fail();
  to_int(ii, m.body_dofnum);
  if (!b.i64("body_lastdof", ii, nb)) return fail();
  to_int(ii, m.body_lastdof);
  if (!b.i64("body_weldid", ii, nb)) return fail();
  to_int(ii, m.body_weldid);
  if (!b.f64("body_pos", f, 3 * nb)) return fail();
  to_vec3(f, m.body_pos);
  if (!b.f64("body_quat", f, 4 * nb)) return fail();
  to_quat(f, m.body_quat);
  if (!b.f64("body_mass", m.body_mass, nb)) return fail();
  if (!b.f64("body_ipos", f, 3 * nb)) return fail();
  to_vec3(f, m.body_ipos);
  if (!b.f64("body_inertia", f, 9 * nb)) return fail();
  m.body_inertia.resize(nb);
  for (long i = 0; i < nb; i++)
    for (int k = 0; k < 9; k++) m.body_inertia[i][k] = f[9 * i + k];

  if (!b.i64("jnt_type", ii, nj)) return fail();
  to_int(ii, m.jnt_type);
  if (!b.i64("jnt_body", ii, nj)) return fail();
  to_int(ii, m.jnt_body);
  if (!b.i64("jnt_qposadr", ii, nj)) return fail();
  to_int(ii, m.jnt_qposadr);
  if (!b.i64("jnt_dofadr", ii, nj)) return fail();
  to_int(ii, m.jnt_dofadr);
  if (!b.i64("jnt_limited", ii, nj)) return fail();
  to_int(ii, m.jnt_limited);
  if (!b.f64("jnt_pos", f, 3 * nj)) return fail();
  to_vec3(f, m.jnt_pos);
  if (!b.f64("jnt_axis", f, 3 * nj)) return fail();
  to_vec3(f, m.jnt_axis);
  if (!b.f64("jnt_range", f, 2 * nj)) return fail();
  to_arr(f, m.jnt_range);
  if (!b.f64("jnt_stiffness", m.jnt_stiffness, nj)) return fail();
  if (!b.f64("jnt_springref", m.jnt_springref, nj)) return fail();

  long nv = m.nv;
  if (!b.i64("dof_body", ii, nv)) return fail();
  to_int(ii, m.dof_body);
  if (!b.i64("dof_jnt", ii, nv)) return fail();
  to_int(ii, m.dof_jnt);
  if (!b.i64("dof_parent", ii, nv)) return fail();
  to_int(ii, m.dof_parent);
  if (!b.f64("dof_damping", m.dof_damping, nv)) return fail();
  if (!b.f64("dof_armature", m.dof_armature, nv)) return fail();

  if (!b.i64("geom_type", ii, ng)) return fail();
  to_int(ii, m.geom_type);
  if (!b.i64("geom_body", ii, ng)) return fail();
  to_int(ii, m.geom_body);
  if (!b.i64("geom_dataid", ii, ng)) return fail();
  to_int(ii, m.geom_dataid);
  if (!b.i64("geom_group", ii, ng)) return fail();
  to_int(ii, m.geom_group);
  if (!b.i64("geom_contype", ii, ng)) return fail();
  to_int(ii, m.geom_contype);
  if (!b.i64("geom_conaffinity", ii, ng)) return fail();
  to_int(ii, m.geom_conaffinity);
  if (!b.f64("geom_pos", f, 3 * ng)) return fail();
  to_vec3(f, m.geom_pos);
  if (!b.f64("geom_quat", f, 4 * ng)) return fail();
  to_quat(f, m.geom_quat);
  if (!b.f64("geom_size", f, 3 * ng)) return fail();
  to_vec3(f, m.geom_size);
  if (!b.f64("geom_friction", m.geom_friction, ng)) return fail();
  if (!b.f64("geom_rgba", f, 4 * ng)) return fail();
  to_arr(f, m.geom_rgba);

  if (!b.i64("cam_body", ii, nc)) return fail();
  to_int(ii, m.cam_body);
  if (!b.f64("cam_pos", f, 3 * nc)) return fail();
  to_vec3(f, m.cam_pos);
  if (!b.f64("cam_quat", f, 4 * nc)) return fail();
  to_quat(f, m.cam_quat);
  if (!b.f64("cam_fovy", m.cam_fovy, nc)) return fail();

  long nu = m.nu;
  if (!b.i64("actuator_joint", ii, nu)) return fail();
  to_int(ii, m.actuator_joint);
  if (!b.i64("actuator_ctrllimited", ii, nu)) return fail();
  to_int(ii, m.actuator_ctrllimited);
  if (!b.i64("actuator_forcelimited", ii, nu)) return fail();
  to_int(ii, m.actuator_forcelimited);
  if (!b.f64("actuator_gear", m.actuator_gear, nu)) return fail();
  if (!b.f64("actuator_gain", m.actuator_gain, nu)) return fail();
  if (!b.f64("actuator_bias", f, 3 * nu)) return fail();
  to_arr(f, m.actuator_bias);
  if (!b.f64("actuator_ctrlrange", f, 2 * nu)) return fail();
  to_arr(f, m.actuator_ctrlrange);
  if (!b.f64("actuator_forcerange", f, 2 * nu)) return fail();
  to_arr(f, m.actuator_forcerange);
  std::vector<int64_t> madr, mnum, mjnt;
  std::vector<Real> mcoef;
  if (!b.i64("actuator_moment_adr", madr, nu) || !b.i64("actuator_moment_num", mnum, nu) ||
      !b.i64("moment_jnt", mjnt) || !b.f64("moment_coef", mcoef, (long)mjnt.size()))
    return fail();
  m.actuator_moment.resize(nu);
  for (long u = 0; u < nu; u++)
    for (long k = 0; k < mnum[u]; k++) m.actuator_moment[u].push_back({(int)mjnt[madr[u] + k], mcoef[madr[u] + k]});

  if (!b.i64("eq_joint1", ii, ne)) return fail();
  to_int(ii, m.eq_joint1);
  if (!b.i64("eq_joint2", ii, ne)) return fail();
  to_int(ii, m.eq_joint2);
  if (!b.f64("eq_polycoef", f, 5 * ne)) return fail();
  to_arr(f, m.eq_polycoef);
  if (!b.f64("eq_solref", f, 2 * ne)) return fail();
  to_arr(f, m.eq_solref);
  if (!b.f64("eq_solimp", f, 5 * ne)) return fail();
  to_arr(f, m.eq_solimp);

  if (!b.i64("dof_blocks", ii)) return fail();
  for (size_t k = 0; k + 1 < ii.size(); k += 2) m.dof_blocks.push_back({(int)ii[k], (int)ii[k + 1]});
  if (!b.i64("pair_candidates", ii)) return fail();
  for (size_t k = 0; k + 1 < ii.size(); k += 2) m.pair_candidates.push_back({(int)ii[k], (int)ii[k + 1]});

  if (!b.f64("qpos0", m.qpos0, m.nq)) return fail();
  if (!b.f64("qpos_reset", m.qpos_reset, m.nq)) return fail();

  std::vector<int64_t> hva, hvn, hta, htn, htri;
  std::vector<Real> hv;
  if (!b.i64("hull_vert_adr", hva, nmesh) || !b.i64("hull_vert_num", hvn, nmesh) || !b.f64("hull_vert", hv) ||
      !b.i64("hull_tri_adr", hta, nmesh) || !b.i64("hull_tri_num", htn, nmesh) || !b.i64("hull_tri", htri))
    return fail();
  m.mesh_hull.resize(nmesh);
  for (long i = 0; i < nmesh; i++) {
    for (long k = 0; k < hvn[i]; k++) {
      long a = 3 * (hva[i] + k);
      m.mesh_hull[i].vert.push_back(v3(hv[a], hv[a + 1], hv[a + 2]));
    }
    for (long k = 0; k < htn[i]; k++) {
      long a = 3 * (hta[i] + k);
      m.mesh_hull[i].tri.push_back({(int)htri[a], (int)htri[a + 1], (int)htri[a + 2]});
    }
  }
  std::vector<int64_t> hfa, hfn, hfva, hfvn, hfv, hea, hen, he;
  std::vector<Real> hfp;
  if (!b.i64("hull_face_adr", hfa, nmesh) || !b.i64("hull_face_num", hfn, nmesh) || !b.f64("hull_face_plane", hfp) ||
      !b.i64("hull_face_vert_adr", hfva) || !b.i64("hull_face_vert_num", hfvn) || !b.i64("hull_face_vert", hfv) ||
      !b.i64("hull_edge_adr", hea, nmesh) || !b.i64("hull_edge_num", hen, nmesh) || !b.i64("hull_edge", he))
    return fail();
  for (long i = 0; i < nmesh; i++) {
    Hull& h = m.mesh_hull[i];
    long nv = (long)h.vert.size();
    for (long f = hfa[i]; f < hfa[i] + hfn[i]; f++) {
      if (f < 0 || 4 * f + 3 >= (long)hfp.size() || f >= (long)hfva.size() || f >= (long)hfvn.size()) return fail();
      h.face_n.push_back(v3(hfp[4 * f], hfp[4 * f + 1], hfp[4 * f + 2]));
      h.face_d.push_back(hfp[4 * f + 3]);
      std::vector<int> loop;
      for (long k = 0; k < hfvn[f]; k++) {
        long at = hfva[f] + k;
        if (at < 0 || at >= (long)hfv.size() || hfv[at] < 0 || hfv[at] >= nv) return fail();
        loop.push_back((int)hfv[at]);
      }
      h.face_loop.push_back(loop);
    }
    for (long e = hea[i]; e < hea[i] + hen[i]; e++) {
      if (e < 0 || 2 * e + 1 >= (long)he.size() || he[2 * e] < 0 || he[2 * e] >= nv || he[2 * e + 1] < 0 ||
          he[2 * e + 1] >= nv)
        return fail();
      h.edge.push_back({(int)he[2 * e], (int)he[2 * e + 1]});
    }
  }

  // derived geometry (model.rs:279-316)
  m.geom_rbound.resize(ng);
  m.geom_aabb.resize(ng);
  for (long g = 0; g < ng; g++) {
    m.geom_rbound[g] = m.rbound((int)g);
    m.geom_aabb[g] = m.local_aabb((int)g);
  }
  if (m.solver.contact_hertz <= 0.0) m.solver.contact_hertz = 0.25 / m.timestep;
  m.rebuild_collision_pairs();
  set_const(m);
  return mp;
}

// model.rs:398-407 (with the mask test of model.rs:438-442 applied to the
// pre-filtered candidate list)
void Model::rebuild_collision_pairs() {
  collision_pairs.clear();
  for (auto& pr : pair_candidates) {
    int g1 = pr.first, g2 = pr.second;
    bool masks = (geom_contype[g1] & geom_conaffinity[g2]) != 0 || (geom_contype[g2] & geom_conaffinity[g1]) != 0;
    if (masks) collision_pairs.push_back(pr);
  }
}

// model.rs:384-396
Real Model::rbound(int g) const {
  Vec3 s = geom_size[g];
  switch (geom_type[g]) {
    case GEOM_PLANE: return INFINITY;
    case GEOM_SPHERE: return s[0];
    case GEOM_CAPSULE: return s[0] + s[1];
    case GEOM_BOX: return norm(s);
    case GEOM_CYLINDER: return std::sqrt(s[0] * s[0] + s[1] * s[1]);
    default: {
      Real r = 0.0;
      for (auto& v : mesh_hull[geom_dataid[g]].vert) r = rmax(r, norm(v));
      return r;
    }
  }
}

// model.rs:365-382
std::array<Vec3, 2> Model::local_aabb(int g) const {
  Vec3 s = geom_size[g];
  Real inf = INFINITY;
  switch (geom_type[g]) {
    case GEOM_PLANE: return {v3zero(), v3(inf, inf, inf)};
    case GEOM_SPHERE: return {v3zero(), v3(s[0], s[0], s[0])};
    case GEOM_CAPSULE: return {v3zero(), v3(s[0], s[0], s[0] + s[1])};
    case GEOM_BOX: return {v3zero(), s};
    case GEOM_CYLINDER: return {v3zero(), v3(s[0], s[0], s[1])};
    default: {
      Vec3 lo = v3(inf, inf, inf), hi = v3(-inf, -inf, -inf);
      for (auto& v : mesh_hull[geom_dataid[g]].vert) {
        lo = vmin(lo, v);
        hi = vmax(hi, v);
      }
      return {(lo + hi) * 0.5, (hi - lo) * 0.5};
    }
  }
}

// data.rs:83-119
void data_init(const Model& m, Data& d) {
  int nb = m.nbody(), ng = m.ngeom(), nj = m.njnt(), nv = m.nv;
  d.time = 0.0;
  d.qpos = m.qpos_reset;
  d.qvel.assign(nv, 0.0);
  d.ctrl.assign(m.nu, 0.0);
  d.qfrc_applied.assign(nv, 0.0);
  d.xpos.assign(nb, v3zero());
  d.xquat.assign(nb, qidentity());
  d.xmat.assign(nb, m3identity());
  d.xipos.assign(nb, v3zero());
  d.xanchor.assign(nj, v3zero());
  d.xaxis.assign(nj, v3zero());
  d.geom_xpos.assign(ng, v3zero());
  d.geom_xmat.assign(ng, m3identity());
  d.cdof.assign(nv, spzero());
  d.cdof_dot.assign(nv, spzero());
  d.cinert.assign(nb, spi_zero());
  d.crb.assign(nb, spi_zero());
  d.cvel.assign(nb, spzero());
  d.qm.assign((size_t)nv * nv, 0.0);
  d.qm_chol.assign((size_t)nv * nv, 0.0);
  d.qfrc_bias.assign(nv, 0.0);
  d.qfrc_passive.assign(nv, 0.0);
  d.qfrc_actuator.assign(nv, 0.0);
  d.qfrc_constraint.assign(nv, 0.0);
  d.qacc.assign(nv, 0.0);
  d.actuator_force.assign(m.nu, 0.0);
  d.actuator_clamped.assign(m.nu, 0);
  d.contacts.clear();
  d.prev_contacts.clear();
  d.prev_lambda.clear();
  d.newton_iters = 0;
  d.status = 0;
}

// data.rs:122-131: qacc (the Newton warm start) is kept
void data_reset(const Model& m, Data& d) {
  d.time = 0.0;
  d.qpos = m.qpos_reset;
  std::fill(d.qvel.begin(), d.qvel.end(), 0.0);
  std::fill(d.ctrl.begin(), d.ctrl.end(), 0.0);
  std::fill(d.qfrc_applied.begin(), d.qfrc_applied.end(), 0.0);
  d.contacts.clear();
  d.prev_contacts.clear();
  d.prev_lambda.clear();
}

// ---------------------------------------------------------------- params.rs
int param_width(const Model& m, int p) {
  switch (p) {
    case P_GEOM_SIZE: case P_ACTUATOR_BIAS: case P_BODY_INERTIA: case P_BODY_IPOS: return 3;
    case P_GEOM_RGBA: return 4;
    case P_QPOS0: return m.nq;
    default: return 1;
  }
}
int param_count(const Model& m, int p) {
  switch (p) {
    case P_GEOM_FRICTION: case P_GEOM_SIZE: case P_GEOM_RGBA: case P_GEOM_CONTYPE: case P_GEOM_CONAFFINITY:
      return m.ngeom();
    case P_BODY_MASS: case P_BODY_INERTIA: case P_BODY_IPOS: return m.nbody();
    case P_QPOS0: return 1;
    case P_DOF_DAMPING: return m.nv;
    case P_ACTUATOR_GAIN: case P_ACTUATOR_BIAS: return m.nu;
    default: return 0;
  }
}

// params.rs:92-108
void get_param(const Model& m, int p, int id, Real* o) {
  switch (p) {
    case P_GEOM_FRICTION: o[0] = m.geom_friction[id]; break;
    case P_GEOM_SIZE: for (int k = 0; k < 3; k++) o[k] = m.geom_size[id][k]; break;
    case P_GEOM_RGBA: for (int k = 0; k < 4; k++) o[k] = (Real)(float)m.geom_rgba[id][k]; break;
    case P_GEOM_CONTYPE: o[0] = (Real)m.geom_contype[id]; break;
    case P_GEOM_CONAFFINITY: o[0] = (Real)m.geom_conaffinity[id]; break;
    case P_BODY_MASS: o[0] = m.body_mass[id]; break;
    case P_DOF_DAMPING: o[0] = m.dof_damping[id]; break;
    case P_ACTUATOR_GAIN: o[0] = m.actuator_gain[id]; break;
    case P_ACTUATOR_BIAS: for (int k = 0; k < 3; k++) o[k] = m.actuator_bias[id][k]; break;
    case P_BODY_INERTIA: for (int k = 0; k < 3; k++) o[k] = m.body_inertia[id][4 * k]; break;
    case P_BODY_IPOS: for (int k = 0; k < 3; k++) o[k] = m.body_ipos[id][k]; break;
    case P_QPOS0: for (int k = 0; k < m.nq; k++) o[k] = m.qpos_reset[k]; break;
  }
}

// params.rs:111-177: validate, then update and refresh derived quantities
bool set_param(Model& m, int p, int id, const Real* v, int n, std::string* err) {
  static const char* names[] = {"GeomFriction", "GeomSize", "GeomRgba", "GeomContype", "GeomConaffinity", "BodyMass",
                                "DofDamping", "ActuatorGain", "ActuatorBias", "BodyInertia", "BodyIpos", "Qpos0"};
  if (p < 0 || p >= P_COUNT) {
    *err = "unknown parameter";
    return false;
  }
  if (id < 0 || id >= param_count(m, p)) {
    *err = std::string(names[p]) + ": id " + std::to_string(id) + " out of range (have " +
           std::to_string(param_count(m, p)) + ")";
    return false;
  }
  if (n != param_width(m, p)) {
    *err = std::string(names[p]) + ": expected " + std::to_string(param_width(m, p)) + " values, got " +
           std::to_string(n);
    return false;
  }
  for (int k = 0; k < n; k++)
    if (!std::isfinite(v[k])) {
      *err = std::string(names[p]) + ": values must be finite";
      return false;
    }
  switch (p) {
    case P_GEOM_FRICTION: m.geom_friction[id] = rmax(v[0], 0.0); break;
    case P_GEOM_SIZE:
      if (m.geom_type[id] == GEOM_MESH || m.geom_type[id] == GEOM_PLANE) {
        *err = "geom_size applies to sphere, capsule, box, and cylinder geoms";
        return false;
      }
      for (int k = 0; k < 3; k++)
        if (v[k] < 0.0) {
          *err = "geom_size must be non-negative";
          return false;
        }
      m.geom_size[id] = v3(v[0], v[1], v[2]);
      m.geom_rbound[id] = m.rbound(id);
      m.geom_aabb[id] = m.local_aabb(id);
      break;
    case P_GEOM_RGBA: for (int k = 0; k < 4; k++) m.geom_rgba[id][k] = (Real)(float)v[k]; break;
    case P_GEOM_CONTYPE: case P_GEOM_CONAFFINITY: {
      uint32_t bits = (uint32_t)rmin(rmax(v[0], 0.0), 4294967295.0);  // Rust `as u32` saturates
      if (p == P_GEOM_CONTYPE) m.geom_contype[id] = bits;
      else m.geom_conaffinity[id] = bits;
      m.rebuild_collision_pairs();
      break;
    }
    case P_BODY_MASS: {
      if (id == 0) {
        *err = "the world body has no mass";
        return false;
      }
      if (v[0] <= 0.0 && m.body_jntnum[id] > 0) {
        *err = "moving bodies need positive mass";
        return false;
      }
      Real scale = m.body_mass[id] > 0.0 ? v[0] / m.body_mass[id] : 1.0;
      m.body_mass[id] = v[0];
      m.body_inertia[id] = mscale(m.body_inertia[id], scale);
      set_const(m);
      break;
    }
    case P_DOF_DAMPING: m.dof_damping[id] = rmax(v[0], 0.0); break;
    case P_ACTUATOR_GAIN: m.actuator_gain[id] = v[0]; break;
    case P_ACTUATOR_BIAS: for (int k = 0; k < 3; k++) m.actuator_bias[id][k] = v[k]; break;
    case P_BODY_INERTIA:
      if (id == 0 || v[0] < 0.0 || v[1] < 0.0 || v[2] < 0.0) {
        *err = "body_inertia needs a non-world body and non-negative moments";
        return false;
      }
      m.body_inertia[id] = m3diag(v3(v[0], v[1], v[2]));
      set_const(m);
      break;
    case P_BODY_IPOS:
      if (id == 0) {
        *err = "the world body has no center of mass";
        return false;
      }
      m.body_ipos[id] = v3(v[0], v[1], v[2]);
      set_const(m);
      break;
    case P_QPOS0: for (int k = 0; k < m.nq; k++) m.qpos_reset[k] = v[k]; break;
  }
  return true;
}

}  // namespace om
