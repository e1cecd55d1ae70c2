// Host side of the C-ABI (include/pippin_b200.h): model blob parsing, the
// derived device model (tree levels, children lists, dof-chain masks, work
// caps), per-env parameter blocks and state in HBM, launch configuration,
// CUDA-graph replay of the step, and the Physics-trait entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/pippin_b200.h"
#include "pg_kernels.h"
#include "pg_mlp.h"
#include "pg_model.h"

using namespace pg;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return PG_ERR_CUDA;
}
#define CK(call)                                  \
  do {                                            \
    cudaError_t _e = (call);                      \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

// ---------------------------------------------------------------- blob
struct BlobArr {
  uint32_t dtype = 0;
  uint64_t count = 0;
  const uint8_t* data = nullptr;
};

struct Blob {
  std::map<std::string, BlobArr> a;
  bool parse(const void* p, size_t bytes, std::string* err) {
    const uint8_t* b = (const uint8_t*)p;
    if (!p || bytes < 16 || std::memcmp(b, "PGBLOB01", 8) != 0) {
      *err = "model blob: bad magic";
      return false;
    }
    uint32_t ver, n;
    std::memcpy(&ver, b + 8, 4);
    std::memcpy(&n, b + 12, 4);
    if (ver != 1) {
      *err = "model blob: unsupported version";
      return false;
    }
    if (16 + 64ull * n > bytes) {
      *err = "model blob: truncated directory";
      return false;
    }
    for (uint32_t i = 0; i < n; i++) {
      const uint8_t* e = b + 16 + 64ull * i;
      char name[41];
      std::memcpy(name, e, 40);
      name[40] = 0;
      BlobArr x;
      uint64_t off;
      std::memcpy(&x.dtype, e + 40, 4);
      std::memcpy(&x.count, e + 48, 8);
      std::memcpy(&off, e + 56, 8);
      uint64_t es = x.dtype == 3 ? 1 : 8;
      if (x.dtype < 1 || x.dtype > 3 || off % 8 || x.count > bytes || off + x.count * es > bytes) {
        *err = std::string("model blob: bad entry ") + name;
        return false;
      }
      x.data = b + off;
      a[name] = x;
    }
    return true;
  }
  template <class T>
  bool get(const char* name, uint32_t dtype, std::vector<T>& out, long expect, std::string* err) {
    auto it = a.find(name);
    if (it == a.end() || it->second.dtype != dtype || (expect >= 0 && (long)it->second.count != expect)) {
      *err = std::string("model blob: missing or mis-sized array ") + name;
      return false;
    }
    out.resize(it->second.count);
    if (dtype == 1) {
      std::vector<double> tmp(it->second.count);
      std::memcpy(tmp.data(), it->second.data, 8 * tmp.size());
      for (size_t k = 0; k < tmp.size(); k++) out[k] = (T)tmp[k];
    } else if (dtype == 2) {
      std::vector<int64_t> tmp(it->second.count);
      std::memcpy(tmp.data(), it->second.data, 8 * tmp.size());
      for (size_t k = 0; k < tmp.size(); k++) out[k] = (T)tmp[k];
    } else {
      for (size_t k = 0; k < it->second.count; k++) out[k] = (T)it->second.data[k];
    }
    return true;
  }
  std::vector<std::string> names(const char* name) {
    std::vector<std::string> out;
    auto it = a.find(name);
    if (it == a.end()) return out;
    std::string cur;
    for (uint64_t k = 0; k < it->second.count; k++) {
      char c = (char)it->second.data[k];
      if (c == 0) {
        out.push_back(cur);
        cur.clear();
      } else {
        cur.push_back(c);
      }
    }
    return out;
  }
};

// ---------------------------------------------------------------- host model
struct HostModel {
  int nq = 0, nv = 0, nu = 0, nbody = 0, njnt = 0, ngeom = 0, ncam = 0, neq = 0, nmesh = 0;
  double timestep = 0, gravity[3] = {0, 0, 0};
  int integrator = 0, solver = 0, iterations = 0;
  double tolerance = 0, margin = 0, solref[2] = {0, 0}, solimp[5] = {0, 0, 0, 0, 0}, impratio = 0, hertz = 0,
         dampratio = 0, slop = 0;
  std::vector<int> body_parent, body_jntadr, body_jntnum, body_dofadr, body_dofnum, body_lastdof, body_weldid;
  std::vector<double> body_pos, body_quat, body_mass, body_ipos, body_inertia;
  std::vector<int> jnt_type, jnt_body, jnt_qposadr, jnt_dofadr, jnt_limited;
  std::vector<double> jnt_pos, jnt_axis, jnt_range, jnt_stiffness, jnt_springref;
  std::vector<int> dof_body, dof_jnt, dof_parent;
  std::vector<double> dof_damping, dof_armature;
  std::vector<int> geom_type, geom_body, geom_dataid, geom_group, geom_contype, geom_conaffinity;
  std::vector<double> geom_pos, geom_quat, geom_size, geom_friction, geom_rgba;
  std::vector<int> cam_body;
  std::vector<double> cam_pos, cam_quat, cam_fovy;
  std::vector<int> act_joint, act_ctrllimited, act_forcelimited, act_moment_adr, act_moment_num, moment_jnt;
  std::vector<double> act_gear, act_gain, act_bias, act_ctrlrange, act_forcerange, moment_coef;
  std::vector<int> eq_j1, eq_j2;
  std::vector<double> eq_poly, eq_solref, eq_solimp;
  std::vector<int> dof_blocks, pairs;
  std::vector<double> qpos0, qpos_reset;
  std::vector<int> hull_vadr, hull_vnum, hull_tadr, hull_tnum, hull_tri;
  std::vector<double> hull_vert;
  // polygon faces (plane, vertex loop) and edges of each hull
  std::vector<int> hull_fadr, hull_fnum, hull_fvadr, hull_fvnum, hull_fv, hull_eadr, hull_enum, hull_edge;
  std::vector<double> hull_fplane;
  std::vector<int> mesh_vadr, mesh_vnum, mesh_tadr, mesh_tnum, mesh_tri;
  std::vector<double> mesh_vert;
  std::vector<std::string> names[6];  // body, geom, camera, mesh, joint, actuator
};

bool load_model(const void* blob, size_t bytes, HostModel& m, std::string* err) {
  Blob b;
  if (!b.parse(blob, bytes, err)) return false;
  std::vector<double> f;
  std::vector<int> i;
#define F1(name, dst)                                  \
  if (!b.get(name, 1, f, 1, err)) return false;        \
  dst = f[0];
#define I1(name, dst)                                  \
  if (!b.get(name, 2, i, 1, err)) return false;        \
  dst = i[0];
  F1("timestep", m.timestep);
  if (!b.get("gravity", 1, f, 3, err)) return false;
  for (int k = 0; k < 3; k++) m.gravity[k] = f[k];
  I1("integrator", m.integrator);
  I1("opt_solver", m.solver);
  I1("opt_iterations", m.iterations);
  F1("opt_tolerance", m.tolerance);
  F1("opt_margin", m.margin);
  if (!b.get("opt_solref", 1, f, 2, err)) return false;
  m.solref[0] = f[0];
  m.solref[1] = f[1];
  if (!b.get("opt_solimp", 1, f, 5, err)) return false;
  for (int k = 0; k < 5; k++) m.solimp[k] = f[k];
  F1("opt_impratio", m.impratio);
  F1("opt_hertz", m.hertz);
  F1("opt_dampratio", m.dampratio);
  F1("opt_slop", m.slop);
#undef F1
#undef I1
  std::vector<long> dims;
  if (!b.get("dims", 2, dims, 9, err)) return false;
  m.nq = (int)dims[0];
  m.nv = (int)dims[1];
  m.nu = (int)dims[2];
  m.nbody = (int)dims[3];
  m.njnt = (int)dims[4];
  m.ngeom = (int)dims[5];
  m.ncam = (int)dims[6];
  m.neq = (int)dims[7];
  m.nmesh = (int)dims[8];
  long nb = m.nbody, nj = m.njnt, nv = m.nv, ng = m.ngeom, nc = m.ncam, nu = m.nu, ne = m.neq, nm = m.nmesh;
  bool ok = b.get("body_parent", 2, m.body_parent, nb, err) && b.get("body_jntadr", 2, m.body_jntadr, nb, err) &&
            b.get("body_jntnum", 2, m.body_jntnum, nb, err) && b.get("body_dofadr", 2, m.body_dofadr, nb, err) &&
            b.get("body_dofnum", 2, m.body_dofnum, nb, err) && b.get("body_lastdof", 2, m.body_lastdof, nb, err) &&
            b.get("body_weldid", 2, m.body_weldid, nb, err) && b.get("body_pos", 1, m.body_pos, 3 * nb, err) &&
            b.get("body_quat", 1, m.body_quat, 4 * nb, err) && b.get("body_mass", 1, m.body_mass, nb, err) &&
            b.get("body_ipos", 1, m.body_ipos, 3 * nb, err) && b.get("body_inertia", 1, m.body_inertia, 9 * nb, err) &&
            b.get("jnt_type", 2, m.jnt_type, nj, err) && b.get("jnt_body", 2, m.jnt_body, nj, err) &&
            b.get("jnt_qposadr", 2, m.jnt_qposadr, nj, err) && b.get("jnt_dofadr", 2, m.jnt_dofadr, nj, err) &&
            b.get("jnt_limited", 2, m.jnt_limited, nj, err) && b.get("jnt_pos", 1, m.jnt_pos, 3 * nj, err) &&
            b.get("jnt_axis", 1, m.jnt_axis, 3 * nj, err) && b.get("jnt_range", 1, m.jnt_range, 2 * nj, err) &&
            b.get("jnt_stiffness", 1, m.jnt_stiffness, nj, err) && b.get("jnt_springref", 1, m.jnt_springref, nj, err) &&
            b.get("dof_body", 2, m.dof_body, nv, err) && b.get("dof_jnt", 2, m.dof_jnt, nv, err) &&
            b.get("dof_parent", 2, m.dof_parent, nv, err) && b.get("dof_damping", 1, m.dof_damping, nv, err) &&
            b.get("dof_armature", 1, m.dof_armature, nv, err) && b.get("geom_type", 2, m.geom_type, ng, err) &&
            b.get("geom_body", 2, m.geom_body, ng, err) && b.get("geom_dataid", 2, m.geom_dataid, ng, err) &&
            b.get("geom_group", 2, m.geom_group, ng, err) && b.get("geom_contype", 2, m.geom_contype, ng, err) &&
            b.get("geom_conaffinity", 2, m.geom_conaffinity, ng, err) && b.get("geom_pos", 1, m.geom_pos, 3 * ng, err) &&
            b.get("geom_quat", 1, m.geom_quat, 4 * ng, err) && b.get("geom_size", 1, m.geom_size, 3 * ng, err) &&
            b.get("geom_friction", 1, m.geom_friction, ng, err) && b.get("geom_rgba", 1, m.geom_rgba, 4 * ng, err) &&
            b.get("cam_body", 2, m.cam_body, nc, err) && b.get("cam_pos", 1, m.cam_pos, 3 * nc, err) &&
            b.get("cam_quat", 1, m.cam_quat, 4 * nc, err) && b.get("cam_fovy", 1, m.cam_fovy, nc, err) &&
            b.get("actuator_joint", 2, m.act_joint, nu, err) &&
            b.get("actuator_ctrllimited", 2, m.act_ctrllimited, nu, err) &&
            b.get("actuator_forcelimited", 2, m.act_forcelimited, nu, err) &&
            b.get("actuator_gear", 1, m.act_gear, nu, err) && b.get("actuator_gain", 1, m.act_gain, nu, err) &&
            b.get("actuator_bias", 1, m.act_bias, 3 * nu, err) &&
            b.get("actuator_ctrlrange", 1, m.act_ctrlrange, 2 * nu, err) &&
            b.get("actuator_forcerange", 1, m.act_forcerange, 2 * nu, err) &&
            b.get("actuator_moment_adr", 2, m.act_moment_adr, nu, err) &&
            b.get("actuator_moment_num", 2, m.act_moment_num, nu, err) && b.get("moment_jnt", 2, m.moment_jnt, -1, err) &&
            b.get("moment_coef", 1, m.moment_coef, (long)m.moment_jnt.size(), err) &&
            b.get("eq_joint1", 2, m.eq_j1, ne, err) && b.get("eq_joint2", 2, m.eq_j2, ne, err) &&
            b.get("eq_polycoef", 1, m.eq_poly, 5 * ne, err) && b.get("eq_solref", 1, m.eq_solref, 2 * ne, err) &&
            b.get("eq_solimp", 1, m.eq_solimp, 5 * ne, err) && b.get("dof_blocks", 2, m.dof_blocks, -1, err) &&
            b.get("pair_candidates", 2, m.pairs, -1, err) && b.get("qpos0", 1, m.qpos0, m.nq, err) &&
            b.get("qpos_reset", 1, m.qpos_reset, m.nq, err) && b.get("hull_vert_adr", 2, m.hull_vadr, nm, err) &&
            b.get("hull_vert_num", 2, m.hull_vnum, nm, err) && b.get("hull_vert", 1, m.hull_vert, -1, err) &&
            b.get("hull_tri_adr", 2, m.hull_tadr, nm, err) && b.get("hull_tri_num", 2, m.hull_tnum, nm, err) &&
            b.get("hull_tri", 2, m.hull_tri, -1, err) && b.get("mesh_vert_adr", 2, m.mesh_vadr, nm, err) &&
            b.get("mesh_vert_num", 2, m.mesh_vnum, nm, err) && b.get("mesh_vert", 1, m.mesh_vert, -1, err) &&
            b.get("mesh_tri_adr", 2, m.mesh_tadr, nm, err) && b.get("mesh_tri_num", 2, m.mesh_tnum, nm, err) &&
            b.get("mesh_tri", 2, m.mesh_tri, -1, err) && b.get("hull_face_adr", 2, m.hull_fadr, nm, err) &&
            b.get("hull_face_num", 2, m.hull_fnum, nm, err) && b.get("hull_face_plane", 1, m.hull_fplane, -1, err) &&
            b.get("hull_face_vert_adr", 2, m.hull_fvadr, -1, err) &&
            b.get("hull_face_vert_num", 2, m.hull_fvnum, -1, err) && b.get("hull_face_vert", 2, m.hull_fv, -1, err) &&
            b.get("hull_edge_adr", 2, m.hull_eadr, nm, err) && b.get("hull_edge_num", 2, m.hull_enum, nm, err) &&
            b.get("hull_edge", 2, m.hull_edge, -1, err);
  if (!ok) return false;
  const char* tables[6] = {"names_body", "names_geom", "names_cam", "names_mesh", "names_jnt", "names_actuator"};
  for (int t = 0; t < 6; t++) m.names[t] = b.names(tables[t]);
  // structural checks the kernels rely on
  if (m.nv > NV_MAX) {
    *err = "model has more than 64 degrees of freedom (dof-chain masks are 64-bit)";
    return false;
  }
  if (m.dof_blocks.size() / 2 > 64) {
    *err = "model has more than 64 independent trees";
    return false;
  }
  for (int b2 = 1; b2 < m.nbody; b2++)
    if (m.body_parent[b2] < 0 || m.body_parent[b2] >= b2) {
      *err = "model blob: bodies must follow their parents";
      return false;
    }
  for (int g = 0; g < m.ngeom; g++)
    if (m.geom_body[g] < 0 || m.geom_body[g] >= m.nbody) {
      *err = "model blob: geom_body out of range";
      return false;
    }
  for (size_t k = 0; k < m.pairs.size(); k++)
    if (m.pairs[k] < 0 || m.pairs[k] >= m.ngeom) {
      *err = "model blob: pair_candidates out of range";
      return false;
    }
  // every index a kernel follows must stay in range, and every parent chain
  // must end: a corrupt blob is rejected here instead of reaching the GPU
  auto bad = [&](const char* what) {
    *err = std::string("model blob: ") + what + " out of range";
    return false;
  };
  for (int k = 0; k < m.nv; k++) {
    if (m.dof_parent[k] < -1 || m.dof_parent[k] >= k) return bad("dof_parent");
    if (m.dof_body[k] < 1 || m.dof_body[k] >= m.nbody) return bad("dof_body");
  }
  for (int b = 0; b < m.nbody; b++) {
    if (m.body_lastdof[b] < -1 || m.body_lastdof[b] >= m.nv) return bad("body_lastdof");
    if (m.body_jntadr[b] < 0 || m.body_jntnum[b] < 0 || m.body_jntadr[b] + m.body_jntnum[b] > m.njnt)
      return bad("body joints");
    if (m.body_dofadr[b] < 0 || m.body_dofnum[b] < 0 || m.body_dofadr[b] + m.body_dofnum[b] > m.nv)
      return bad("body dofs");
  }
  for (int j = 0; j < m.njnt; j++) {
    int t = m.jnt_type[j];
    int nqj = t == JNT_FREE ? 7 : (t == JNT_BALL ? 4 : 1), nvj = t == JNT_FREE ? 6 : (t == JNT_BALL ? 3 : 1);
    if (t < 0 || t > 3) return bad("jnt_type");
    if (m.jnt_qposadr[j] < 0 || m.jnt_qposadr[j] + nqj > m.nq) return bad("jnt_qposadr");
    if (m.jnt_dofadr[j] < 0 || m.jnt_dofadr[j] + nvj > m.nv) return bad("jnt_dofadr");
  }
  for (int g = 0; g < m.ngeom; g++) {
    if (m.geom_type[g] < 0 || m.geom_type[g] > 5) return bad("geom_type");
    if (m.geom_type[g] == GEOM_MESH && (m.geom_dataid[g] < 0 || m.geom_dataid[g] >= m.nmesh)) return bad("geom_dataid");
  }
  long nhv = (long)m.hull_vert.size() / 3, nht = (long)m.hull_tri.size() / 3;
  for (int i = 0; i < m.nmesh; i++) {
    if (m.hull_vadr[i] < 0 || m.hull_vnum[i] < 1 || m.hull_vadr[i] + m.hull_vnum[i] > nhv) return bad("hull vertices");
    if (m.hull_tadr[i] < 0 || m.hull_tnum[i] < 0 || m.hull_tadr[i] + m.hull_tnum[i] > nht) return bad("hull triangles");
    for (int t = 0; t < 3 * m.hull_tnum[i]; t++) {
      int v = m.hull_tri[3 * m.hull_tadr[i] + t];
      if (v < 0 || v >= m.hull_vnum[i]) return bad("hull triangle vertex");
    }
    // polygon faces: every loop within the hull's vertices and at most
    // HULL_FACE_LIMIT long (the clip buffers are sized from the longest);
    // edges likewise
    long nf = (long)m.hull_fvadr.size(), nfv = (long)m.hull_fv.size(), ne = (long)m.hull_edge.size() / 2;
    if ((long)m.hull_fvnum.size() != nf || (long)m.hull_fplane.size() != 4 * nf) return bad("hull faces");
    if (m.hull_fadr[i] < 0 || m.hull_fnum[i] < 4 || (long)m.hull_fadr[i] + m.hull_fnum[i] > nf) return bad("hull faces");
    for (int f = m.hull_fadr[i]; f < m.hull_fadr[i] + m.hull_fnum[i]; f++) {
      if (m.hull_fvnum[f] < 3 || m.hull_fvnum[f] > HULL_FACE_LIMIT || m.hull_fvadr[f] < 0 ||
          (long)m.hull_fvadr[f] + m.hull_fvnum[f] > nfv)
        return bad("hull face loop (3 to 256 vertices)");
      for (int k = 0; k < m.hull_fvnum[f]; k++) {
        int v = m.hull_fv[m.hull_fvadr[f] + k];
        if (v < 0 || v >= m.hull_vnum[i]) return bad("hull face vertex");
      }
    }
    if (m.hull_eadr[i] < 0 || m.hull_enum[i] < 6 || (long)m.hull_eadr[i] + m.hull_enum[i] > ne) return bad("hull edges");
    for (int e = m.hull_eadr[i]; e < m.hull_eadr[i] + m.hull_enum[i]; e++)
      for (int k = 0; k < 2; k++)
        if (m.hull_edge[2 * e + k] < 0 || m.hull_edge[2 * e + k] >= m.hull_vnum[i]) return bad("hull edge vertex");
    long nmv = (long)m.mesh_vert.size() / 3, nmt = (long)m.mesh_tri.size() / 3;
    if (m.mesh_vadr[i] < 0 || m.mesh_vnum[i] < 0 || m.mesh_vadr[i] + m.mesh_vnum[i] > nmv) return bad("mesh vertices");
    if (m.mesh_tadr[i] < 0 || m.mesh_tnum[i] < 0 || m.mesh_tadr[i] + m.mesh_tnum[i] > nmt) return bad("mesh triangles");
  }
  for (int c = 0; c < m.ncam; c++)
    if (m.cam_body[c] < 0 || m.cam_body[c] >= m.nbody) return bad("cam_body");
  for (int u = 0; u < m.nu; u++) {
    if (m.act_moment_adr[u] < 0 || m.act_moment_num[u] < 1 ||
        m.act_moment_adr[u] + m.act_moment_num[u] > (int)m.moment_jnt.size())
      return bad("actuator_moment");
  }
  for (int j : m.moment_jnt)
    if (j < 0 || j >= m.njnt || (m.jnt_type[j] != JNT_HINGE && m.jnt_type[j] != JNT_SLIDE)) return bad("moment_jnt");
  for (int e = 0; e < m.neq; e++) {
    if (m.eq_j1[e] < 0 || m.eq_j1[e] >= m.njnt) return bad("eq_joint1");
    if (m.eq_j2[e] < -1 || m.eq_j2[e] >= m.njnt) return bad("eq_joint2");
  }
  if (m.dof_blocks.size() % 2 || m.pairs.size() % 2) return bad("dof_blocks/pairs layout");
  {
    int expect = 0;
    for (size_t k = 0; k + 1 < m.dof_blocks.size(); k += 2) {
      if (m.dof_blocks[k] != expect || m.dof_blocks[k + 1] <= m.dof_blocks[k]) return bad("dof_blocks");
      expect = m.dof_blocks[k + 1];
    }
    if (expect != m.nv) return bad("dof_blocks");
  }
  if (!(m.timestep > 0.0) || !std::isfinite(m.timestep)) return bad("timestep");
  if (m.hertz <= 0.0) m.hertz = 0.25 / m.timestep;
  return true;
}

// Largest contact count a pair can produce (collision.rs routines).
int max_hits(int a, int b) {
  if (a > b) std::swap(a, b);
  if (a == GEOM_PLANE) {
    if (b == GEOM_SPHERE) return 1;
    if (b == GEOM_CAPSULE) return 2;
    return 4;  // box, cylinder, mesh
  }
  if (a == GEOM_SPHERE && b <= GEOM_BOX) return 1;
  if (a == GEOM_CAPSULE && (b == GEOM_CAPSULE || b == GEOM_BOX)) return 3;
  return 4;
}

// ---------------------------------------------------------------- device model
struct DevArena {
  std::vector<uint8_t> host;
  size_t add(const void* p, size_t bytes) {
    size_t off = (host.size() + 15) & ~size_t(15);
    host.resize(off + std::max<size_t>(bytes, 8));
    if (bytes) std::memcpy(host.data() + off, p, bytes);
    return off;
  }
};

struct Handle {
  HostModel hm;
  DModel dm{};
  WsLayout w{}, wn{};
  ScrLayout s{};
  WorkLayout k{};
  int64_t n = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  void* d_model = nullptr;
  double *qpos = nullptr, *qvel = nullptr, *ctrl = nullptr, *qacc = nullptr, *applied = nullptr, *params = nullptr;
  int32_t *iters = nullptr, *ncon = nullptr, *nrows = nullptr, *status = nullptr;
  double* scratch = nullptr;
  size_t scratch_tiles = 0;
  double* work = nullptr;  // [env][k.stride]
  double* prev_con = nullptr;   // [env][maxcon][P_STRIDE] PGS warm start (allocated with PGS)
  int32_t* prev_ncon = nullptr;  // [env]
  int* queue = nullptr;
  int* order = nullptr;  // [n] Newton-phase order of a substep's envs
  // learned warm start: contact list, network, and whether one is loaded
  LearnArgs learn{};
  bool mlp_loaded = false;
  std::vector<double> base_params;
  int warm_mode = WARM_REF_PREV_QACC;
  SubstepCfg cfg{{16, 4, 0}, {32, 4, 0}, {16, 4, 0}};
  int sm_count = 0;
  size_t smem_optin = 0;
  // growable device buffers
  struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
  };
  Buf b_ctrl, b_qout, b_poses_g, b_poses_c, b_dbg, b_vals, b_ids;
  // graph cache for pg_step
  std::map<std::tuple<int64_t, int64_t, int64_t>, cudaGraphExec_t> graphs;
  uint64_t version = 1, graph_version = 0;
  std::string name = "pippin-cuda";
};

}  // namespace

struct pg_handle : Handle {};

namespace {

int grow(Handle* h, Handle::Buf& b, size_t bytes) {
  if (b.bytes >= bytes) return PG_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  size_t want = std::max<size_t>(bytes, 256);
  cudaError_t e = cudaMalloc(&b.p, want);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  b.bytes = want;
  (void)h;
  return PG_OK;
}

void clear_graphs(Handle* h) {
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
}

// largest arena staged into shared memory (bigger models read it from L1/L2)
constexpr int STAGE_LIMIT = 48 * 1024;
std::vector<int> dmodel_pointer_fields();

StepArgs make_args(Handle* h) {
  StepArgs a{};
  a.m = h->dm;
  a.w = h->w;
  a.wn = h->wn;
  a.s = h->s;
  a.k = h->k;
  a.work = h->work;
  a.st.qpos = h->qpos;
  a.st.qvel = h->qvel;
  a.st.ctrl = h->ctrl;
  a.st.qacc = h->qacc;
  a.st.applied = h->applied;
  a.st.params = h->params;
  a.st.iters = h->iters;
  a.st.ncon = h->ncon;
  a.st.nrows = h->nrows;
  a.st.status = h->status;
  a.st.prev_con = h->prev_con;
  a.st.prev_ncon = h->prev_ncon;
  a.scratch = h->scratch;
  a.queue = h->queue;
  a.order = h->order;
  a.warm_mode = h->warm_mode;
  a.learn = h->learn;
  a.learn.count = h->queue + Q_LEARN;
  a.stage_model = h->dm.arena_bytes <= STAGE_LIMIT ? 1 : 0;
  std::vector<int> po = dmodel_pointer_fields();
  a.n_ptr = (int)std::min<size_t>(po.size(), MAX_PTR_FIELDS);
  for (int k = 0; k < a.n_ptr; k++) a.ptr_off[k] = po[k];
  return a;
}

// Workspace layouts of the smooth-dynamics phase (w) and the Newton phase
// (wn), the Newton phase's tile scratch (s) and the per-env work record (k).
void layouts(const HostModel& m, int maxcon, int maxrows, WsLayout* w, WsLayout* wn, ScrLayout* s, WorkLayout* k) {
  int off = 0;
  auto take = [&](int n) {
    int o = off;
    off += (n + 1) & ~1;  // keep 16-byte alignment
    return o;
  };
  int nb = m.nbody, nv = m.nv, ng = m.ngeom, nu = m.nu;
  *w = WsLayout{};
  std::fill_n(reinterpret_cast<int*>(w), sizeof(WsLayout) / sizeof(int), -1);
  // smooth phase: live throughout
  w->qpos = take(m.nq);
  w->qvel = take(nv);
  w->ctrl = take(nu);
  w->cdof = take(6 * nv);
  w->smooth = take(nv);
  w->acc = take(nv);
  w->rinv = take(nv);
  w->actforce = take(nu);
  w->actclamped = take(nu);
  w->misc = take(8);
  int region = off;
  // tree walks and passive/actuator forces ...
  w->xpos = take(3 * nb);
  w->xquat = take(4 * nb);
  w->cinert = take(13 * nb);
  w->cvel = take(6 * nb);
  w->cacc = take(6 * nb);
  w->cfrc = take(6 * nb);
  w->bias = take(nv);
  w->passive = take(nv);
  w->actf = take(nv);
  int tree_end = off;
  // ... then the factorisations in the same region
  off = region;
  w->fac = take(nv * nv);
  w->fac2 = take(nv * nv);
  w->rinv2 = take(nv);
  w->stride = std::max(off, tree_end);

  // Newton phase
  off = 0;
  *wn = WsLayout{};
  std::fill_n(reinterpret_cast<int*>(wn), sizeof(WsLayout) / sizeof(int), -1);
  wn->qpos = take(m.nq);
  wn->qvel = take(nv);
  wn->qacc = take(nv);
  // M and the big factor stay in shared memory for models the one-lane-per-row
  // path takes; larger ones read M from the work record and factor in the
  // tile's global scratch (its set_const slot), so that their workspace stays
  // small enough for several tiles an SM
  bool small_mats = nv <= 16;
  wn->qm = small_mats ? take(nv * nv) : -1;
  wn->smooth = take(nv);
  wn->acc = take(nv);
  wn->qfrc_c = take(nv);
  // cdof, rinv and warm side by side: the register Newton keeps its packed
  // factor there (cdof is dead once the rows are built, rinv and
  // warm are not used on that path)
  wn->cdof = take(6 * nv);
  wn->rinv = take(nv);
  wn->warm = take(nv);
  wn->fac = small_mats ? take(nv * nv) : -1;
  wn->a0 = take(nv);
  wn->grad = take(nv);
  wn->p = take(nv);
  wn->tmp = take(nv);
  wn->tmp2 = take(nv);
  wn->mp = take(nv);
  wn->vel = take(nv);
  wn->misc = take(8);
  wn->stride = off;
  // register Newton: rows and vectors over the factor and Newton vectors it
  // does not use (M stays put; the Hessian factor lives in registers)
  if (nv <= 16 && m.dof_blocks.size() / 2 == 1) {
    int need = ((16 * nv + 1) & ~1) + 16 + 32;
    int base = (wn->mp + ((nv + 1) & ~1)) - wn->fac >= need ? wn->fac : wn->stride;
    wn->sj = base;
    wn->sx = base + ((16 * nv + 1) & ~1);
    wn->sc = wn->sx + 16;
    wn->stride = std::max(wn->stride, wn->sc + 32);
    // the Hessian factor's entries below the diagonal, packed
    int ncol = nv * (nv - 1) / 2;
    if (wn->fac - wn->cdof >= ncol) {
      wn->sl = wn->cdof;
    } else {
      wn->sl = wn->stride;
      wn->stride += (ncol + 1) & ~1;
    }
  }

  // per-env work record
  off = 0;
  k->qm = take(nv * nv);
  k->cdof = take(6 * nv);
  k->a0 = take(nv);
  k->smooth = take(nv);
  k->bias = take(nv);
  k->lh = take(nv * nv);
  k->rinvh = take(nv);
  k->meta = take(K_META_SIZE);
  k->geoms = take(ng * G_STRIDE);
  k->contacts = take(maxcon * C_STRIDE);
  k->stride = off;

  off = 0;
  int rhs = nv + 6 * nb + 32;  // set_const right-hand sides + per-lane row copies
  s->geoms = -1;
  s->contacts = -1;
  s->jac = take(std::max(maxrows * nv, rhs * nv));
  s->rows = take(std::max(maxrows * R_STRIDE, rhs));
  s->chol = take(nv * nv);
  int multi = m.dof_blocks.size() / 2 > 1;
  s->sub_m = take(multi ? nv * nv : 0);
  s->sub_j = take(multi ? maxrows * nv : 0);
  s->sub_rows = take(multi ? maxrows * R_STRIDE : 0);
  s->isl_dof = take(nv + 2);
  s->isl_row = take(maxrows + (nv + maxrows + 1) / 2 + 2);
  s->isl_of_row = take(maxrows / 2 + 2);
  s->mj = take(maxrows * nv);
  s->stride = off;
}

// Model staging: the byte offset of every pointer field of DModel (the
// kernels rebase them onto the block's shared copy of the arena).
std::vector<int> dmodel_pointer_fields() {
  std::vector<int> o;
#define PF(f) o.push_back((int)offsetof(DModel, f))
  PF(body_parent); PF(body_jntadr); PF(body_jntnum); PF(body_dofadr); PF(body_dofnum); PF(body_lastdof);
  PF(body_dofmask); PF(body_pos); PF(body_quat); PF(level_adr); PF(level_body); PF(child_adr); PF(child_list);
  PF(jnt_type); PF(jnt_qposadr); PF(jnt_dofadr); PF(jnt_limited); PF(jnt_pos); PF(jnt_axis); PF(jnt_range);
  PF(jnt_stiffness); PF(jnt_springref); PF(dof_body); PF(dof_parent); PF(dof_armature); PF(dof_block);
  PF(block_adr); PF(dofact_adr); PF(dofact_u); PF(dofact_coef); PF(geom_type); PF(geom_body); PF(geom_dataid);
  PF(geom_pos); PF(geom_quat); PF(pair_g); PF(cam_body); PF(cam_pos); PF(cam_quat); PF(act_gear);
  PF(act_ctrllimited); PF(act_ctrlrange); PF(act_forcelimited); PF(act_forcerange); PF(act_moment_adr);
  PF(act_moment_num); PF(moment_jnt); PF(moment_coef); PF(eq_j1); PF(eq_j2); PF(eq_poly); PF(eq_solref);
  PF(eq_solimp); PF(qpos0); PF(hull_vadr); PF(hull_vnum); PF(hull_vert); PF(hull_fadr); PF(hull_fnum);
  PF(hull_face); PF(hull_fvadr); PF(hull_fvnum); PF(hull_fv); PF(hull_eadr); PF(hull_enum); PF(hull_edge);
  PF(hull_eface); PF(hull_nbadr); PF(hull_nbnum); PF(hull_nb); PF(hull_seed);
#undef PF
  return o;
}

// A kernel's dynamic shared-memory limit is one setting per device shared by
// every handle: it only ever rises, so a handle with a smaller launch shape
// cannot lower it under another handle's larger one.
int allow_smem(int device, const void* fn, size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> raised;
  std::lock_guard<std::mutex> g(mu);
  size_t& cur = raised[{device, fn}];
  if (smem <= cur) return PG_OK;
  CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cur = smem;
  return PG_OK;
}

// Resident grid of a launch shape for one phase. `phase` is K_SMOOTH (whose
// shape set_const and poses share), K_COLLIDE or K_NEWTON.
int choose_grid(Handle* h, int phase, const LaunchCfg& want, LaunchCfg* out) {
  LaunchCfg c = want;
  int threads = c.tiles_per_block * c.G;
  if (threads > 256 || threads < 32) return fail(PG_ERR_INVALID, "launch shape: 32..256 threads per block");
  StepArgs a = make_args(h);
  std::vector<int> kinds = {phase};
  if (phase == K_SMOOTH) kinds = {K_SMOOTH, K_SET_CONST, K_POSES};
  if (phase == K_NEWTON) kinds = {K_NEWTON, K_NEWTON_PLAIN};  // with and without the learned start's code
  int per_sm = 0;
  for (int k : kinds) {
    size_t smem = kernel_smem(k, a, c.tiles_per_block);
    if (smem > h->smem_optin) return fail(PG_ERR_INVALID, "launch shape needs more shared memory than a block has");
    const void* fn = tile_kernel(k, c.G);
    if (!fn) return fail(PG_ERR_INVALID, "lanes per env must be 8, 16 or 32");
    if (int rc = allow_smem(h->device, fn, smem)) return rc;
    int nb = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem));
    if (nb == 0) return fail(PG_ERR_INVALID, "launch shape does not fit on an SM");
    if (k == phase) per_sm = nb;
  }
  c.blocks = per_sm * h->sm_count;
  *out = c;
  return PG_OK;
}

// tile scratch for the Newton phase and set_const (which runs on the smooth shape)
int ensure_scratch(Handle* h, const SubstepCfg& c) {
  size_t tiles = std::max((size_t)c.newton.blocks * c.newton.tiles_per_block,
                          (size_t)c.smooth.blocks * c.smooth.tiles_per_block);
  if (tiles <= h->scratch_tiles) return PG_OK;
  if (h->scratch) cudaFree(h->scratch);
  h->scratch = nullptr;
  h->scratch_tiles = 0;
  CK(cudaMalloc(&h->scratch, tiles * h->s.stride * sizeof(double) + 64));
  h->scratch_tiles = tiles;
  return PG_OK;
}

int apply_cfg(Handle* h, const SubstepCfg& want) {
  SubstepCfg c;
  int rc = choose_grid(h, K_SMOOTH, want.smooth, &c.smooth);
  if (!rc) rc = choose_grid(h, K_COLLIDE, want.collide, &c.collide);
  if (!rc) rc = choose_grid(h, K_NEWTON, want.newton, &c.newton);
  if (rc) return rc;
  if ((rc = ensure_scratch(h, c))) return rc;
  h->cfg = c;
  h->version++;
  return PG_OK;
}

// no more blocks than the range needs
LaunchCfg fit(LaunchCfg c, int64_t count) {
  int64_t need = (count + c.tiles_per_block - 1) / c.tiles_per_block;
  if (need < c.blocks) c.blocks = (int)std::max<int64_t>(need, 1);
  return c;
}
SubstepCfg fit(const SubstepCfg& c, int64_t count) {
  return SubstepCfg{fit(c.smooth, count), fit(c.collide, count), fit(c.newton, count)};
}

int launch_status(cudaError_t e) { return e == cudaSuccess ? PG_OK : cuda_fail(e, "kernel launch"); }

int set_const_range(Handle* h, int64_t start, int64_t end) {
  if (end <= start) return PG_OK;
  StepArgs a = make_args(h);
  a.start = (int)start;
  a.count = (int)(end - start);
  return launch_status(launch_set_const(a, fit(h->cfg.smooth, end - start), nullptr, (int)(end - start), h->stream));
}

// One substep, or the graph-replayed sequence of `nstep` substeps, of envs
// [start, end) on the handle's stream.
int enqueue_substeps(Handle* h, StepArgs a, int64_t start, int64_t end, int64_t nstep) {
  a.start = (int)start;
  a.count = (int)(end - start);
  a.nstep = (int)nstep;
  SubstepCfg c = fit(h->cfg, end - start);
  for (int64_t k = 0; k < nstep; k++) {
    a.sidx = (int)k;
    cudaError_t e = launch_substep(a, c, h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "substep launch");
  }
  return PG_OK;
}

int check_range(Handle* h, int64_t start, int64_t end) {
  if (start < 0 || end < start || end > h->n)
    return fail(PG_ERR_INVALID, "env range [" + std::to_string(start) + ", " + std::to_string(end) + ") out of bounds (have " +
                                    std::to_string(h->n) + ")");
  return PG_OK;
}

int field_width(const HostModel& m, int f) {
  switch (f) {
    case PG_FIELD_QPOS: return m.nq;
    case PG_FIELD_QVEL: return m.nv;
    case PG_FIELD_CTRL: return m.nu;
    case PG_FIELD_QACC: return m.nv;
    case PG_FIELD_QFRC_APPLIED: return m.nv;
  }
  return -1;
}
double* field_ptr(Handle* h, int f) {
  switch (f) {
    case PG_FIELD_QPOS: return h->qpos;
    case PG_FIELD_QVEL: return h->qvel;
    case PG_FIELD_CTRL: return h->ctrl;
    case PG_FIELD_QACC: return h->qacc;
    case PG_FIELD_QFRC_APPLIED: return h->applied;
  }
  return nullptr;
}

// params.rs:61-83
int param_width(const HostModel& m, int p) {
  switch (p) {
    case PG_PARAM_GEOM_SIZE: case PG_PARAM_ACTUATOR_BIAS: case PG_PARAM_BODY_INERTIA: case PG_PARAM_BODY_IPOS: return 3;
    case PG_PARAM_GEOM_RGBA: return 4;
    case PG_PARAM_QPOS0: return m.nq;
    default: return 1;
  }
}
int param_count(const HostModel& m, int p) {
  switch (p) {
    case PG_PARAM_GEOM_FRICTION: case PG_PARAM_GEOM_SIZE: case PG_PARAM_GEOM_RGBA: case PG_PARAM_GEOM_CONTYPE:
    case PG_PARAM_GEOM_CONAFFINITY: return m.ngeom;
    case PG_PARAM_BODY_MASS: case PG_PARAM_BODY_INERTIA: case PG_PARAM_BODY_IPOS: return m.nbody;
    case PG_PARAM_QPOS0: return 1;
    case PG_PARAM_DOF_DAMPING: return m.nv;
    case PG_PARAM_ACTUATOR_GAIN: case PG_PARAM_ACTUATOR_BIAS: return m.nu;
  }
  return 0;
}
const char* param_name(int p) {
  static const char* n[] = {"GeomFriction", "GeomSize", "GeomRgba", "GeomContype", "GeomConaffinity", "BodyMass",
                            "DofDamping", "ActuatorGain", "ActuatorBias", "BodyInertia", "BodyIpos", "Qpos0"};
  return (p >= 0 && p < 12) ? n[p] : "?";
}

// params.rs:111-177 validation (values of one env)
bool validate_param(const HostModel& m, int p, int64_t id, const double* v, std::string* err) {
  int w = param_width(m, p);
  for (int k = 0; k < w; k++)
    if (!std::isfinite(v[k])) {
      *err = std::string(param_name(p)) + ": values must be finite";
      return false;
    }
  switch (p) {
    case PG_PARAM_GEOM_SIZE:
      if (m.geom_type[id] == GEOM_MESH || m.geom_type[id] == GEOM_PLANE) {
        *err = "geom_size applies to sphere, capsule, box, and cylinder geoms";
        return false;
      }
      for (int k = 0; k < 3; k++)
        if (v[k] < 0.0) {
          *err = "geom_size must be non-negative";
          return false;
        }
      break;
    case PG_PARAM_BODY_MASS:
      if (id == 0) {
        *err = "the world body has no mass";
        return false;
      }
      if (v[0] <= 0.0 && m.body_jntnum[id] > 0) {
        *err = "moving bodies need positive mass";
        return false;
      }
      break;
    case PG_PARAM_BODY_INERTIA:
      if (id == 0 || v[0] < 0.0 || v[1] < 0.0 || v[2] < 0.0) {
        *err = "body_inertia needs a non-world body and non-negative moments";
        return false;
      }
      break;
    case PG_PARAM_BODY_IPOS:
      if (id == 0) {
        *err = "the world body has no center of mass";
        return false;
      }
      break;
  }
  return true;
}


void read_param(const DModel& d, const double* prm, int p, int64_t id, double* o, int nq) {
  switch (p) {
    case PG_PARAM_GEOM_FRICTION: o[0] = prm[d.p_friction + id]; break;
    case PG_PARAM_GEOM_SIZE: for (int k = 0; k < 3; k++) o[k] = prm[d.p_size + 3 * id + k]; break;
    case PG_PARAM_GEOM_RGBA: for (int k = 0; k < 4; k++) o[k] = prm[d.p_rgba + 4 * id + k]; break;
    case PG_PARAM_GEOM_CONTYPE: o[0] = prm[d.p_contype + id]; break;
    case PG_PARAM_GEOM_CONAFFINITY: o[0] = prm[d.p_conaff + id]; break;
    case PG_PARAM_BODY_MASS: o[0] = prm[d.p_mass + id]; break;
    case PG_PARAM_DOF_DAMPING: o[0] = prm[d.p_damping + id]; break;
    case PG_PARAM_ACTUATOR_GAIN: o[0] = prm[d.p_gain + id]; break;
    case PG_PARAM_ACTUATOR_BIAS: for (int k = 0; k < 3; k++) o[k] = prm[d.p_bias + 3 * id + k]; break;
    case PG_PARAM_BODY_INERTIA: for (int k = 0; k < 3; k++) o[k] = prm[d.p_inertia + 9 * id + 4 * k]; break;
    case PG_PARAM_BODY_IPOS: for (int k = 0; k < 3; k++) o[k] = prm[d.p_ipos + 3 * id + k]; break;
    case PG_PARAM_QPOS0: for (int k = 0; k < nq; k++) o[k] = prm[d.p_qpos_reset + k]; break;
  }
}

int build_device_model(Handle* h) {
  HostModel& m = h->hm;
  DModel& d = h->dm;
  DevArena ar;
  int nb = m.nbody, nv = m.nv;
  // tree levels (world at level 0) and children in decreasing id
  std::vector<int> depth(nb, 0);
  int nlevel = 1;
  for (int b = 1; b < nb; b++) {
    depth[b] = depth[m.body_parent[b]] + 1;
    nlevel = std::max(nlevel, depth[b] + 1);
  }
  std::vector<int> level_adr(nlevel + 1, 0), level_body;
  for (int L = 0; L < nlevel; L++) {
    level_adr[L] = (int)level_body.size();
    for (int b = 0; b < nb; b++)
      if (depth[b] == L) level_body.push_back(b);
  }
  level_adr[nlevel] = (int)level_body.size();
  std::vector<int> child_adr(nb + 1, 0), child_list;
  for (int b = 0; b < nb; b++) {
    child_adr[b] = (int)child_list.size();
    for (int c = nb - 1; c > b; c--)
      if (m.body_parent[c] == b) child_list.push_back(c);
  }
  child_adr[nb] = (int)child_list.size();
  std::vector<unsigned long long> dofmask(nb, 0);
  for (int b = 0; b < nb; b++)
    for (int k = m.body_lastdof[b]; k != -1; k = m.dof_parent[k]) dofmask[b] |= 1ull << k;
  int nblock = (int)m.dof_blocks.size() / 2;
  std::vector<int> dof_block(std::max(nv, 1), 0);
  for (int b = 0; b < nblock; b++)
    for (int k = m.dof_blocks[2 * b]; k < m.dof_blocks[2 * b + 1]; k++) dof_block[k] = b;
  // actuator contributions per dof, in (actuator, moment entry) order
  std::vector<std::vector<std::pair<int, double>>> per(nv);
  for (int u = 0; u < m.nu; u++)
    for (int k = 0; k < m.act_moment_num[u]; k++) {
      int j = m.moment_jnt[m.act_moment_adr[u] + k];
      per[m.jnt_dofadr[j]].push_back({u, m.moment_coef[m.act_moment_adr[u] + k]});
    }
  std::vector<int> dofact_adr(nv + 1, 0), dofact_u;
  std::vector<double> dofact_coef;
  for (int k = 0; k < nv; k++) {
    dofact_adr[k] = (int)dofact_u.size();
    for (auto& pc : per[k]) {
      dofact_u.push_back(pc.first);
      dofact_coef.push_back(pc.second);
    }
  }
  dofact_adr[nv] = (int)dofact_u.size();
  // work caps: every candidate pair at its largest manifold
  int maxcon = 0;
  for (size_t k = 0; k + 1 < m.pairs.size(); k += 2) maxcon += max_hits(m.geom_type[m.pairs[k]], m.geom_type[m.pairs[k + 1]]);
  int nlim = 0;
  for (int j = 0; j < m.njnt; j++)
    if (m.jnt_limited[j] && (m.jnt_type[j] == JNT_HINGE || m.jnt_type[j] == JNT_SLIDE)) nlim++;
  int maxrows = 4 * maxcon + 2 * nlim + m.neq;
  // the two faces of each hull edge (the faces whose loops hold the edge),
  // for the edge-pair pruning of the general convex narrow phase
  std::vector<int> hull_eface(2 * m.hull_edge.size() / 2 + 2, -1);
  for (int i = 0; i < m.nmesh; i++)
    for (int e = m.hull_eadr[i]; e < m.hull_eadr[i] + m.hull_enum[i]; e++) {
      int a = m.hull_edge[2 * e], b = m.hull_edge[2 * e + 1];
      for (int f = 0; f < m.hull_fnum[i]; f++) {
        int fg = m.hull_fadr[i] + f;
        int n = m.hull_fvnum[fg];
        const int* l = &m.hull_fv[m.hull_fvadr[fg]];
        for (int k = 0; k < n; k++) {
          int x = l[k], y = l[(k + 1) % n];
          if ((x == a && y == b) || (x == b && y == a)) {
            if (hull_eface[2 * e] == -1) hull_eface[2 * e] = f;
            else if (hull_eface[2 * e + 1] == -1) hull_eface[2 * e + 1] = f;
          }
        }
      }
    }

  // the support walk of large hulls (fasthull.rs:52-75): each vertex's
  // neighbours along the hull's edges, and the vertex extreme along each of
  // the 26 seed directions (the first maximum)
  const int nhv = (int)m.hull_vert.size() / 3;
  std::vector<std::vector<int>> nbl(nhv);
  for (int i = 0; i < m.nmesh; i++)
    for (int e = m.hull_eadr[i]; e < m.hull_eadr[i] + m.hull_enum[i]; e++) {
      int a = m.hull_edge[2 * e], b = m.hull_edge[2 * e + 1];
      nbl[m.hull_vadr[i] + a].push_back(b);
      nbl[m.hull_vadr[i] + b].push_back(a);
    }
  std::vector<int> hull_nbadr(nhv + 1, 0), hull_nbnum(nhv + 1, 0), hull_nb;
  for (int v = 0; v < nhv; v++) {
    hull_nbadr[v] = (int)hull_nb.size();
    hull_nbnum[v] = (int)nbl[v].size();
    hull_nb.insert(hull_nb.end(), nbl[v].begin(), nbl[v].end());
  }
  hull_nb.push_back(0);
  std::vector<int> hull_seed(HULL_SEEDS * std::max(m.nmesh, 1), 0);
  for (int i = 0; i < m.nmesh; i++) {
    int k = 0;
    for (int x = -1; x <= 1; x++)
      for (int y = -1; y <= 1; y++)
        for (int z = -1; z <= 1; z++) {
          if (!x && !y && !z) continue;
          double inv = 1.0 / std::sqrt((double)(x * x + y * y + z * z));
          double bd = -INFINITY;
          int bv = 0;
          for (int v = 0; v < m.hull_vnum[i]; v++) {
            const double* p = &m.hull_vert[3 * (m.hull_vadr[i] + v)];
            double dv = (x * p[0] + y * p[1] + z * p[2]) * inv;
            if (dv > bd) {
              bd = dv;
              bv = v;
            }
          }
          hull_seed[HULL_SEEDS * i + k++] = bv;
        }
  }

  d.nq = m.nq;
  d.nv = nv;
  d.nu = m.nu;
  d.nbody = nb;
  d.njnt = m.njnt;
  d.ngeom = m.ngeom;
  d.ncam = m.ncam;
  d.neq = m.neq;
  d.npair = (int)m.pairs.size() / 2;
  d.nblock = nblock;
  d.nlevel = nlevel;
  d.nmesh = m.nmesh;
  d.maxcon = maxcon;
  d.maxrows = maxrows;
  d.maxbs = 0;
  for (int b = 0; b < nblock; b++) d.maxbs = std::max(d.maxbs, m.dof_blocks[2 * b + 1] - m.dof_blocks[2 * b]);
  // polytope sizes of the general pairs (mesh against anything, cylinder
  // against a non-plane): the collide kernel caches their world vertices
  // and face normals per tile
  d.gen_vmax = d.gen_fmax = d.gen_lmax = 0;
  for (size_t p = 0; p + 1 < m.pairs.size(); p += 2) {
    int ta = m.geom_type[m.pairs[p]], tb = m.geom_type[m.pairs[p + 1]];
    bool general = ta == GEOM_MESH || tb == GEOM_MESH || (ta == GEOM_CYLINDER && tb != GEOM_PLANE) ||
                   (tb == GEOM_CYLINDER && ta != GEOM_PLANE);
    if (!general) continue;
    for (int g : {m.pairs[p], m.pairs[p + 1]}) {
      int t = m.geom_type[g], nvx = 0, nfx = 0;
      if (t == GEOM_BOX) nvx = 8, nfx = 6;
      if (t == GEOM_CYLINDER) nvx = 2 * CYL_SIDES, nfx = CYL_SIDES + 2;
      int lx = t == GEOM_BOX ? 4 : t == GEOM_CYLINDER ? CYL_SIDES : 0;
      if (t == GEOM_MESH) {
        int mi = m.geom_dataid[g];
        nvx = m.hull_vnum[mi], nfx = m.hull_fnum[mi];
        for (int f = m.hull_fadr[mi]; f < m.hull_fadr[mi] + m.hull_fnum[mi]; f++) lx = std::max(lx, m.hull_fvnum[f]);
      }
      d.gen_vmax = std::max(d.gen_vmax, nvx);
      d.gen_fmax = std::max(d.gen_fmax, nfx);
      d.gen_lmax = std::max(d.gen_lmax, lx);
    }
  }
  // the polytope cache holds both polytopes' world vertices and normals
  // while it stays small; clip buffers move to shared memory when a face is
  // longer than a lane's own buffers take (an incident loop plus one vertex
  // per side plane, for two buffers, then the kept points)
  d.gen_cache = 6 * (d.gen_vmax + d.gen_fmax);
  if (d.gen_cache > GEN_CACHE_LIMIT) d.gen_cache = 0;
  d.gen_clip = d.gen_lmax > HULL_FACE_MAX ? 10 * (2 * d.gen_lmax) : 0;
  d.timestep = m.timestep;
  for (int k = 0; k < 3; k++) d.gravity[k] = m.gravity[k];
  d.integrator = m.integrator;
  d.solver = m.solver;
  d.iterations = m.iterations;
  d.tolerance = m.tolerance;
  d.margin = m.margin;
  d.solref[0] = m.solref[0];
  d.solref[1] = m.solref[1];
  for (int k = 0; k < 5; k++) d.solimp[k] = m.solimp[k];
  d.impratio = m.impratio;
  d.hertz = m.hertz;
  d.dampratio = m.dampratio;
  d.slop = m.slop;

  struct Fix {
    const void** slot;
    size_t off;
  };
  std::vector<Fix> fix;
  auto addv = [&](const void** slot, const void* p, size_t bytes) { fix.push_back({slot, ar.add(p, bytes)}); };
#define ADDI(field, vec) addv((const void**)&d.field, vec.data(), vec.size() * sizeof(int))
#define ADDD(field, vec) addv((const void**)&d.field, vec.data(), vec.size() * sizeof(double))
  ADDI(body_parent, m.body_parent);
  ADDI(body_jntadr, m.body_jntadr);
  ADDI(body_jntnum, m.body_jntnum);
  ADDI(body_dofadr, m.body_dofadr);
  ADDI(body_dofnum, m.body_dofnum);
  ADDI(body_lastdof, m.body_lastdof);
  addv((const void**)&d.body_dofmask, dofmask.data(), dofmask.size() * 8);
  ADDD(body_pos, m.body_pos);
  ADDD(body_quat, m.body_quat);
  ADDI(level_adr, level_adr);
  ADDI(level_body, level_body);
  ADDI(child_adr, child_adr);
  ADDI(child_list, child_list);
  ADDI(jnt_type, m.jnt_type);
  ADDI(jnt_qposadr, m.jnt_qposadr);
  ADDI(jnt_dofadr, m.jnt_dofadr);
  ADDI(jnt_limited, m.jnt_limited);
  ADDD(jnt_pos, m.jnt_pos);
  ADDD(jnt_axis, m.jnt_axis);
  ADDD(jnt_range, m.jnt_range);
  ADDD(jnt_stiffness, m.jnt_stiffness);
  ADDD(jnt_springref, m.jnt_springref);
  ADDI(dof_body, m.dof_body);
  ADDI(dof_parent, m.dof_parent);
  ADDD(dof_armature, m.dof_armature);
  ADDI(dof_block, dof_block);
  ADDI(block_adr, m.dof_blocks);
  ADDI(dofact_adr, dofact_adr);
  ADDI(dofact_u, dofact_u);
  ADDD(dofact_coef, dofact_coef);
  ADDI(geom_type, m.geom_type);
  ADDI(geom_body, m.geom_body);
  ADDI(geom_dataid, m.geom_dataid);
  ADDD(geom_pos, m.geom_pos);
  ADDD(geom_quat, m.geom_quat);
  ADDI(pair_g, m.pairs);
  ADDI(cam_body, m.cam_body);
  ADDD(cam_pos, m.cam_pos);
  ADDD(cam_quat, m.cam_quat);
  ADDD(act_gear, m.act_gear);
  ADDI(act_ctrllimited, m.act_ctrllimited);
  ADDD(act_ctrlrange, m.act_ctrlrange);
  ADDI(act_forcelimited, m.act_forcelimited);
  ADDD(act_forcerange, m.act_forcerange);
  ADDI(act_moment_adr, m.act_moment_adr);
  ADDI(act_moment_num, m.act_moment_num);
  ADDI(moment_jnt, m.moment_jnt);
  ADDD(moment_coef, m.moment_coef);
  ADDI(eq_j1, m.eq_j1);
  ADDI(eq_j2, m.eq_j2);
  ADDD(eq_poly, m.eq_poly);
  ADDD(eq_solref, m.eq_solref);
  ADDD(eq_solimp, m.eq_solimp);
  ADDD(qpos0, m.qpos0);
  ADDI(hull_vadr, m.hull_vadr);
  ADDI(hull_vnum, m.hull_vnum);
  ADDD(hull_vert, m.hull_vert);
  ADDI(hull_fadr, m.hull_fadr);
  ADDI(hull_fnum, m.hull_fnum);
  ADDD(hull_face, m.hull_fplane);
  ADDI(hull_fvadr, m.hull_fvadr);
  ADDI(hull_fvnum, m.hull_fvnum);
  ADDI(hull_fv, m.hull_fv);
  ADDI(hull_eadr, m.hull_eadr);
  ADDI(hull_enum, m.hull_enum);
  ADDI(hull_edge, m.hull_edge);
  ADDI(hull_eface, hull_eface);
  ADDI(hull_nbadr, hull_nbadr);
  ADDI(hull_nbnum, hull_nbnum);
  ADDI(hull_nb, hull_nb);
  ADDI(hull_seed, hull_seed);
#undef ADDI
#undef ADDD
  ar.host.resize((ar.host.size() + 15) & ~size_t(15));  // staged in 16-byte chunks
  CK(cudaMalloc(&h->d_model, ar.host.size()));
  CK(cudaMemcpy(h->d_model, ar.host.data(), ar.host.size(), cudaMemcpyHostToDevice));
  for (auto& f : fix) *f.slot = (const uint8_t*)h->d_model + f.off;
  d.arena = (const unsigned char*)h->d_model;
  d.arena_bytes = (int)ar.host.size();

  // per-env parameter block
  int off = 0;
  auto take = [&](int n) {
    int o = off;
    off += n;
    return o;
  };
  int ng = m.ngeom;
  d.p_friction = take(ng);
  d.p_size = take(3 * ng);
  d.p_contype = take(ng);
  d.p_conaff = take(ng);
  d.p_mass = take(nb);
  d.p_inertia = take(9 * nb);
  d.p_ipos = take(3 * nb);
  d.p_damping = take(nv);
  d.p_gain = take(m.nu);
  d.p_bias = take(3 * m.nu);
  d.p_qpos_reset = take(m.nq);
  d.p_body_invw = take(2 * nb);
  d.p_dof_invw = take(nv);
  d.p_rgba = take(4 * ng);
  d.pstride = (off + 3) & ~3;
  std::vector<double>& bp = h->base_params;
  bp.assign(d.pstride, 0.0);
  for (int g = 0; g < ng; g++) {
    bp[d.p_friction + g] = m.geom_friction[g];
    for (int k = 0; k < 3; k++) bp[d.p_size + 3 * g + k] = m.geom_size[3 * g + k];
    bp[d.p_contype + g] = m.geom_contype[g];
    bp[d.p_conaff + g] = m.geom_conaffinity[g];
    for (int k = 0; k < 4; k++) bp[d.p_rgba + 4 * g + k] = m.geom_rgba[4 * g + k];
  }
  for (int b = 0; b < nb; b++) {
    bp[d.p_mass + b] = m.body_mass[b];
    for (int k = 0; k < 9; k++) bp[d.p_inertia + 9 * b + k] = m.body_inertia[9 * b + k];
    for (int k = 0; k < 3; k++) bp[d.p_ipos + 3 * b + k] = m.body_ipos[3 * b + k];
  }
  for (int k = 0; k < nv; k++) bp[d.p_damping + k] = m.dof_damping[k];
  for (int u = 0; u < m.nu; u++) {
    bp[d.p_gain + u] = m.act_gain[u];
    for (int k = 0; k < 3; k++) bp[d.p_bias + 3 * u + k] = m.act_bias[3 * u + k];
  }
  for (int k = 0; k < m.nq; k++) bp[d.p_qpos_reset + k] = m.qpos_reset[k];
  layouts(m, maxcon, maxrows, &h->w, &h->wn, &h->s, &h->k);
  return PG_OK;
}

void destroy(pg_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  clear_graphs(h);
  void* ptrs[] = {h->d_model, h->qpos, h->qvel, h->ctrl, h->qacc, h->applied, h->params, h->iters, h->ncon,
                  h->nrows, h->status, h->scratch, h->work, h->prev_con, h->prev_ncon, h->queue, h->order, h->b_ctrl.p, h->b_qout.p, h->b_poses_g.p,
                  h->b_poses_c.p, h->b_dbg.p, h->b_vals.p, h->b_ids.p, h->learn.items, h->learn.feat, h->learn.force,
                  h->learn.rows, (void*)h->learn.mlp_w, (void*)h->learn.mlp_f, (void*)h->learn.mlp_err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int copy_rows_d2h(Handle* h, double* dst, const double* src, int64_t start, int64_t end, int width) {
  if (end <= start || width == 0) return PG_OK;
  CK(cudaMemcpyAsync(dst, src + start * width, sizeof(double) * (end - start) * width, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PG_OK;
}

// read the parameter blocks of [start, end) to the host
int read_params(Handle* h, int64_t start, int64_t end, std::vector<double>& out) {
  out.resize((size_t)(end - start) * h->dm.pstride);
  return copy_rows_d2h(h, out.data(), h->params, start, end, h->dm.pstride);
}

}  // namespace

namespace pg {
// Launch arguments of pg_step for [start, end), for entry points that launch
// the step kernel with other scratch (pg_noalloc.cu). Validates like pg_step.
int internal_step_args(pg_handle* h, int64_t start, int64_t end, int64_t nstep, StepArgs* a, SubstepCfg* cfg,
                       cudaStream_t* stream, int* device) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  if (nstep < 0 || nstep > (1 << 30)) return fail(PG_ERR_INVALID, "nstep out of range");
  CK(cudaSetDevice(h->device));
  *a = make_args(h);
  a->start = (int)start;
  a->count = (int)(end - start);
  a->nstep = (int)nstep;
  *cfg = fit(h->cfg, end - start);
  *stream = h->stream;
  *device = h->device;
  return PG_OK;
}
void internal_set_error(const std::string& msg) { g_err = msg; }
}  // namespace pg

extern "C" {

const char* pg_last_error(void) { return g_err.c_str(); }

int pg_create(const void* blob, size_t bytes, int64_t n_envs, int device, pg_handle** out) {
  g_err.clear();
  if (!out) return fail(PG_ERR_INVALID, "out is NULL");
  *out = nullptr;
  if (n_envs < 0 || n_envs > (1ll << 30)) return fail(PG_ERR_INVALID, "n_envs out of range");
  std::unique_ptr<pg_handle, void (*)(pg_handle*)> h(new pg_handle, [](pg_handle* p) { destroy(p); });
  std::string err;
  if (!load_model(blob, bytes, h->hm, &err)) return fail(PG_ERR_INVALID, err);
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(PG_ERR_INVALID, "no such CUDA device");
  h->device = device;
  CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(PG_ERR_UNSUPPORTED, "this library is built for sm_100a (B200)");
  h->sm_count = prop.multiProcessorCount;
  h->smem_optin = prop.sharedMemPerBlockOptin;
  CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  int rc = build_device_model(h.get());
  if (rc) return rc;
  h->n = n_envs;
  const HostModel& m = h->hm;
  size_t n = (size_t)std::max<int64_t>(n_envs, 1);
  CK(cudaMalloc(&h->qpos, sizeof(double) * n * std::max(m.nq, 1)));
  CK(cudaMalloc(&h->qvel, sizeof(double) * n * std::max(m.nv, 1)));
  CK(cudaMalloc(&h->ctrl, sizeof(double) * n * std::max(m.nu, 1)));
  CK(cudaMalloc(&h->qacc, sizeof(double) * n * std::max(m.nv, 1)));
  CK(cudaMalloc(&h->applied, sizeof(double) * n * std::max(m.nv, 1)));
  CK(cudaMalloc(&h->params, sizeof(double) * n * h->dm.pstride));
  CK(cudaMalloc(&h->iters, sizeof(int32_t) * n));
  CK(cudaMalloc(&h->ncon, sizeof(int32_t) * n));
  CK(cudaMalloc(&h->nrows, sizeof(int32_t) * n));
  CK(cudaMalloc(&h->status, sizeof(int32_t) * n));
  CK(cudaMalloc(&h->queue, sizeof(int) * QUEUE_INTS));
  CK(cudaMalloc(&h->order, sizeof(int) * std::max<int64_t>(n, 1)));
  CK(cudaMalloc(&h->work, sizeof(double) * n * h->k.stride));
  CK(cudaMemsetAsync(h->work, 0, sizeof(double) * n * h->k.stride, h->stream));
  CK(cudaMemsetAsync(h->qvel, 0, sizeof(double) * n * std::max(m.nv, 1), h->stream));
  CK(cudaMemsetAsync(h->ctrl, 0, sizeof(double) * n * std::max(m.nu, 1), h->stream));
  CK(cudaMemsetAsync(h->qacc, 0, sizeof(double) * n * std::max(m.nv, 1), h->stream));
  CK(cudaMemsetAsync(h->applied, 0, sizeof(double) * n * std::max(m.nv, 1), h->stream));
  CK(cudaMemsetAsync(h->iters, 0, sizeof(int32_t) * n, h->stream));
  CK(cudaMemsetAsync(h->ncon, 0, sizeof(int32_t) * n, h->stream));
  CK(cudaMemsetAsync(h->nrows, 0, sizeof(int32_t) * n, h->stream));
  CK(cudaMemsetAsync(h->status, 0, sizeof(int32_t) * n, h->stream));
  {
    std::vector<double> hq((size_t)n_envs * m.nq), hp((size_t)n_envs * h->dm.pstride);
    for (int64_t e = 0; e < n_envs; e++) {
      std::copy(m.qpos_reset.begin(), m.qpos_reset.end(), hq.begin() + e * m.nq);
      std::copy(h->base_params.begin(), h->base_params.end(), hp.begin() + e * h->dm.pstride);
    }
    if (n_envs > 0) {
      if (m.nq) CK(cudaMemcpyAsync(h->qpos, hq.data(), sizeof(double) * hq.size(), cudaMemcpyHostToDevice, h->stream));
      CK(cudaMemcpyAsync(h->params, hp.data(), sizeof(double) * hp.size(), cudaMemcpyHostToDevice, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
  }
  int g = m.nv > 16 ? 32 : 16;
  int npair = (int)m.pairs.size() / 2;
  int gc = npair > 16 ? 32 : (npair > 8 ? 16 : 8);
  SubstepCfg want{{g, 4, 0}, {gc, 4, 0}, {g, 4, 0}};
  {
    StepArgs a = make_args(h.get());
    while (want.collide.tiles_per_block > 1 && kernel_smem(K_COLLIDE, a, want.collide.tiles_per_block) > h->smem_optin)
      want.collide.tiles_per_block /= 2;
    while (want.collide.tiles_per_block * want.collide.G < 32) want.collide.G *= 2;
  }
  rc = apply_cfg(h.get(), want);
  if (rc) return rc;
  rc = set_const_range(h.get(), 0, n_envs);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  // a model compiled for PGS gets its warm-start buffers now
  if (h->dm.solver == SOLVER_PGS && (rc = pg_set_solver(h.get(), SOLVER_PGS, -1, -1.0, -1))) return rc;
  *out = h.release();
  return PG_OK;
}

int pg_destroy(pg_handle* h) {
  destroy(h);
  return PG_OK;
}

const char* pg_name(const pg_handle* h) { return h ? h->name.c_str() : ""; }
int64_t pg_num_envs(const pg_handle* h) { return h ? h->n : 0; }

int pg_dims(const pg_handle* h, pg_model_dims* out) {
  if (!h || !out) return fail(PG_ERR_INVALID, "NULL argument");
  out->nq = h->hm.nq;
  out->nv = h->hm.nv;
  out->nu = h->hm.nu;
  out->ngeom = h->hm.ngeom;
  out->ncam = h->hm.ncam;
  out->nbody = h->hm.nbody;
  out->njnt = h->hm.njnt;
  return PG_OK;
}

int pg_step(pg_handle* h, int64_t start, int64_t end, int64_t nstep) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  if (nstep < 0 || nstep > (1 << 30)) return fail(PG_ERR_INVALID, "nstep out of range");
  if (end == start || nstep == 0) return PG_OK;
  CK(cudaSetDevice(h->device));
  if (h->graph_version != h->version) {
    clear_graphs(h);
    h->graph_version = h->version;
  }
  // substeps are replayed from cached graphs of up to 16 substeps each; the
  // first substep of the call (sidx 0) restarts the per-env status word
  const int64_t CHUNK = 16;
  for (int64_t done = 0; done < nstep;) {
    int64_t c = std::min(CHUNK, nstep - done);
    int64_t first = done == 0 ? 0 : 1;
    auto key = std::make_tuple(start, end, c * 2 + first);
    auto it = h->graphs.find(key);
    if (it == h->graphs.end()) {
      if (h->graphs.size() >= 32) clear_graphs(h);
      StepArgs a = make_args(h);
      a.start = (int)start;
      a.count = (int)(end - start);
      a.nstep = (int)c;
      SubstepCfg cfg = fit(h->cfg, end - start);
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t le = cudaSuccess;
      for (int64_t k = 0; k < c && le == cudaSuccess; k++) {
        a.sidx = (int)(first + k);
        le = launch_substep(a, cfg, h->stream);
      }
      cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
      if (le != cudaSuccess) return cuda_fail(le, "substep launch");
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
      cudaGraphExec_t ex;
      ce = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
      it = h->graphs.emplace(key, ex).first;
    }
    CK(cudaGraphLaunch(it->second, h->stream));
    done += c;
  }
  return PG_OK;
}

int pg_step_device(pg_handle* h, int64_t start, int64_t end, int64_t nstep, const double* ctrl_dev) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  if (end > start && h->hm.nu > 0) {
    if (!ctrl_dev) return fail(PG_ERR_INVALID, "ctrl_dev is NULL");
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(h->ctrl + start * h->hm.nu, ctrl_dev, sizeof(double) * (end - start) * h->hm.nu,
                       cudaMemcpyDeviceToDevice, h->stream));
  }
  return pg_step(h, start, end, nstep);
}

int pg_rollout(pg_handle* h, int64_t start, int64_t end, int64_t nstep, const double* ctrl, double* qpos_out) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  if (nstep < 0) return fail(PG_ERR_INVALID, "nstep out of range");
  int64_t cnt = end - start;
  if (cnt == 0 || nstep == 0) return PG_OK;
  const HostModel& m = h->hm;
  if (!ctrl && m.nu > 0) return fail(PG_ERR_INVALID, "ctrl is NULL");
  CK(cudaSetDevice(h->device));
  size_t cb = sizeof(double) * cnt * nstep * std::max(m.nu, 1), qb = sizeof(double) * cnt * nstep * m.nq;
  if ((rc = grow(h, h->b_ctrl, cb))) return rc;
  if (qpos_out && (rc = grow(h, h->b_qout, qb))) return rc;
  if (m.nu) CK(cudaMemcpyAsync(h->b_ctrl.p, ctrl, sizeof(double) * cnt * nstep * m.nu, cudaMemcpyHostToDevice, h->stream));
  StepArgs a = make_args(h);
  a.start = (int)start;
  a.count = (int)cnt;
  a.nstep = (int)nstep;
  a.ctrl_seq = m.nu ? (const double*)h->b_ctrl.p : nullptr;
  a.qpos_out = qpos_out ? (double*)h->b_qout.p : nullptr;
  if ((rc = enqueue_substeps(h, a, start, end, nstep))) return rc;
  if (qpos_out) CK(cudaMemcpyAsync(qpos_out, h->b_qout.p, qb, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PG_OK;
}

int pg_reset(pg_handle* h, const int64_t* envs, int64_t n) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (n < 0 || (n > 0 && !envs)) return fail(PG_ERR_INVALID, "bad env list");
  for (int64_t k = 0; k < n; k++)
    if (envs[k] < 0 || envs[k] >= h->n) return fail(PG_ERR_INVALID, "env id " + std::to_string(envs[k]) + " out of range");
  if (n == 0) return PG_OK;
  CK(cudaSetDevice(h->device));
  int rc = grow(h, h->b_ids, sizeof(int64_t) * n);
  if (rc) return rc;
  CK(cudaMemcpyAsync(h->b_ids.p, envs, sizeof(int64_t) * n, cudaMemcpyHostToDevice, h->stream));
  StepArgs a = make_args(h);
  CK(launch_reset(a, (const int64_t*)h->b_ids.p, (int)n, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PG_OK;
}

int pg_get(pg_handle* h, int field, int64_t start, int64_t end, double* out, size_t len) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int w = field_width(h->hm, field);
  if (w < 0) return fail(PG_ERR_INVALID, "unknown field");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  if (len != (size_t)(end - start) * w)
    return fail(PG_ERR_LENGTH, "get: buffer has " + std::to_string(len) + " elements, expected " +
                                   std::to_string(end - start) + " x " + std::to_string(w));
  CK(cudaSetDevice(h->device));
  return copy_rows_d2h(h, out, field_ptr(h, field), start, end, w);
}

int pg_set(pg_handle* h, int field, int64_t start, int64_t end, const double* src, size_t len) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int w = field_width(h->hm, field);
  if (w < 0) return fail(PG_ERR_INVALID, "unknown field");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  if (len != (size_t)(end - start) * w)
    return fail(PG_ERR_LENGTH, "set: buffer has " + std::to_string(len) + " elements, expected " +
                                   std::to_string(end - start) + " x " + std::to_string(w));
  if (end == start || w == 0) return PG_OK;
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(field_ptr(h, field) + start * w, src, sizeof(double) * len, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PG_OK;
}

int pg_poses(pg_handle* h, int64_t start, int64_t end, pg_pose* geoms, size_t ngeoms_len, pg_pose* cams,
             size_t ncams_len) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  int64_t cnt = end - start;
  const HostModel& m = h->hm;
  if (ngeoms_len != (size_t)cnt * m.ngeom)
    return fail(PG_ERR_LENGTH, "poses(geoms): buffer has " + std::to_string(ngeoms_len) + " elements, expected " +
                                   std::to_string(cnt) + " x " + std::to_string(m.ngeom));
  if (ncams_len != (size_t)cnt * m.ncam)
    return fail(PG_ERR_LENGTH, "poses(cams): buffer has " + std::to_string(ncams_len) + " elements, expected " +
                                   std::to_string(cnt) + " x " + std::to_string(m.ncam));
  if (cnt == 0) return PG_OK;
  CK(cudaSetDevice(h->device));
  if ((rc = grow(h, h->b_poses_g, sizeof(pg_pose) * cnt * std::max(m.ngeom, 1)))) return rc;
  if ((rc = grow(h, h->b_poses_c, sizeof(pg_pose) * cnt * std::max(m.ncam, 1)))) return rc;
  StepArgs a = make_args(h);
  a.start = (int)start;
  a.count = (int)cnt;
  if ((rc = launch_status(
           launch_poses(a, fit(h->cfg.smooth, cnt), (float*)h->b_poses_g.p, (float*)h->b_poses_c.p, h->stream))))
    return rc;
  if (m.ngeom) CK(cudaMemcpyAsync(geoms, h->b_poses_g.p, sizeof(pg_pose) * cnt * m.ngeom, cudaMemcpyDeviceToHost, h->stream));
  if (m.ncam) CK(cudaMemcpyAsync(cams, h->b_poses_c.p, sizeof(pg_pose) * cnt * m.ncam, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PG_OK;
}

int pg_poses_device(pg_handle* h, int64_t start, int64_t end, pg_pose* geoms_dev, pg_pose* cams_dev) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  int64_t cnt = end - start;
  const HostModel& m = h->hm;
  if (cnt == 0) return PG_OK;
  if ((m.ngeom && !geoms_dev) || (m.ncam && !cams_dev)) return fail(PG_ERR_INVALID, "poses_device: NULL buffer");
  CK(cudaSetDevice(h->device));
  StepArgs a = make_args(h);
  a.start = (int)start;
  a.count = (int)cnt;
  return launch_status(launch_poses(a, fit(h->cfg.smooth, cnt), (float*)geoms_dev, (float*)cams_dev, h->stream));
}

int pg_hull_support(pg_handle* h, int mesh, const double* dirs, int64_t n, int32_t* vertex) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (mesh < 0 || mesh >= h->hm.nmesh) return fail(PG_ERR_INVALID, "hull_support: no mesh " + std::to_string(mesh));
  if (n < 0 || n > (int64_t)1 << 28) return fail(PG_ERR_INVALID, "hull_support: direction count out of range");
  if (n == 0) return PG_OK;
  if (!dirs || !vertex) return fail(PG_ERR_INVALID, "hull_support: NULL buffer");
  CK(cudaSetDevice(h->device));
  double* d_dirs = nullptr;
  int* d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_dirs, sizeof(double) * 3 * n);
  if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(int) * n);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_dirs, dirs, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = launch_hull_support(h->dm, mesh, d_dirs, (int)n, d_out, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(vertex, d_out, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_dirs);
  cudaFree(d_out);
  if (e != cudaSuccess) return cuda_fail(e, "hull_support");
  return PG_OK;
}

int pg_param_width(const pg_handle* h, int param) {
  if (!h || param < 0 || param > PG_PARAM_QPOS0) return -1;
  return param_width(h->hm, param);
}

int pg_set_param(pg_handle* h, int param, int64_t id, int64_t start, int64_t end, const double* values, size_t len) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (param < 0 || param > PG_PARAM_QPOS0) return fail(PG_ERR_INVALID, "unknown parameter");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  const HostModel& m = h->hm;
  int w = param_width(m, param);
  if (len != (size_t)(end - start) * w)
    return fail(PG_ERR_LENGTH, "set_param: buffer has " + std::to_string(len) + " elements, expected " +
                                   std::to_string(end - start) + " x " + std::to_string(w));
  if (id < 0 || id >= param_count(m, param))
    return fail(PG_ERR_INVALID, std::string(param_name(param)) + ": id " + std::to_string(id) +
                                    " out of range (have " + std::to_string(param_count(m, param)) + ")");
  std::string err;
  for (int64_t k = 0; k < end - start; k++)
    if (!validate_param(m, param, id, values + k * w, &err)) return fail(PG_ERR_INVALID, err);
  if (end == start) return PG_OK;
  CK(cudaSetDevice(h->device));
  // the values go to the device, where each env's parameter block takes them
  if ((rc = grow(h, h->b_vals, sizeof(double) * len))) return rc;
  CK(cudaMemcpyAsync(h->b_vals.p, values, sizeof(double) * len, cudaMemcpyHostToDevice, h->stream));
  CK(launch_apply_param(h->dm, h->params + start * h->dm.pstride, end - start, param, id, (const double*)h->b_vals.p, w,
                        m.nq, h->stream));
  if (param == PG_PARAM_BODY_MASS || param == PG_PARAM_BODY_INERTIA || param == PG_PARAM_BODY_IPOS) {
    if ((rc = set_const_range(h, start, end))) return rc;
  }
  CK(cudaStreamSynchronize(h->stream));
  return PG_OK;
}

int pg_get_param(pg_handle* h, int param, int64_t id, int64_t start, int64_t end, double* out, size_t len) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (param < 0 || param > PG_PARAM_QPOS0) return fail(PG_ERR_INVALID, "unknown parameter");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  const HostModel& m = h->hm;
  int w = param_width(m, param);
  if (len != (size_t)(end - start) * w)
    return fail(PG_ERR_LENGTH, "get_param: buffer has " + std::to_string(len) + " elements, expected " +
                                   std::to_string(end - start) + " x " + std::to_string(w));
  if (id < 0 || id >= param_count(m, param))
    return fail(PG_ERR_INVALID, std::string(param_name(param)) + ": id " + std::to_string(id) + " out of range");
  if (end == start) return PG_OK;
  CK(cudaSetDevice(h->device));
  std::vector<double> blk;
  if ((rc = read_params(h, start, end, blk))) return rc;
  for (int64_t k = 0; k < end - start; k++) read_param(h->dm, blk.data() + k * h->dm.pstride, param, id, out + k * w, m.nq);
  return PG_OK;
}

int pg_appearance(pg_handle* h, int64_t start, int64_t end, pg_geom_appearance* out, size_t len) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  const HostModel& m = h->hm;
  if (len != (size_t)(end - start) * m.ngeom)
    return fail(PG_ERR_LENGTH, "appearance: buffer has " + std::to_string(len) + " elements, expected " +
                                   std::to_string(end - start) + " x " + std::to_string(m.ngeom));
  if (end == start) return PG_OK;
  CK(cudaSetDevice(h->device));
  std::vector<double> blk;
  if ((rc = read_params(h, start, end, blk))) return rc;
  const DModel& d = h->dm;
  for (int64_t k = 0; k < end - start; k++) {
    const double* prm = blk.data() + k * d.pstride;
    for (int g = 0; g < m.ngeom; g++) {
      pg_geom_appearance& a = out[k * m.ngeom + g];
      for (int c = 0; c < 4; c++) a.rgba[c] = (float)prm[d.p_rgba + 4 * g + c];
      for (int c = 0; c < 3; c++) {
        double base = m.geom_size[3 * g + c];
        a.scale[c] = base > 0.0 ? (float)(prm[d.p_size + 3 * g + c] / base) : 1.0f;
      }
      a.pad = 0.0f;
    }
  }
  return PG_OK;
}

int pg_scene_counts(const pg_handle* h, int64_t* nbody, int64_t* ngeom, int64_t* nmesh, int64_t* ncam) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (nbody) *nbody = h->hm.nbody;
  if (ngeom) *ngeom = h->hm.ngeom;
  if (nmesh) *nmesh = h->hm.nmesh;
  if (ncam) *ncam = h->hm.ncam;
  return PG_OK;
}

int pg_scene_geoms(const pg_handle* h, pg_geom_visual* out, size_t len) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  const HostModel& m = h->hm;
  if (len != (size_t)m.ngeom) return fail(PG_ERR_LENGTH, "scene geoms: buffer must hold ngeom entries");
  for (int g = 0; g < m.ngeom; g++) {
    pg_geom_visual& v = out[g];
    v.shape = m.geom_type[g];
    v.mesh = m.geom_type[g] == GEOM_MESH ? m.geom_dataid[g] : -1;
    for (int k = 0; k < 3; k++) v.size[k] = (float)m.geom_size[3 * g + k];
    for (int k = 0; k < 4; k++) v.rgba[k] = (float)m.geom_rgba[4 * g + k];
    v.body = m.geom_body[g];
    v.group = m.geom_group[g];
  }
  return PG_OK;
}

int pg_scene_mesh(const pg_handle* h, int64_t mesh, float* vertices, size_t nvert_len, uint32_t* triangles,
                  size_t ntri_len, int64_t* nvert, int64_t* ntri) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  const HostModel& m = h->hm;
  if (mesh < 0 || mesh >= m.nmesh) return fail(PG_ERR_INVALID, "mesh id out of range");
  int nv = m.mesh_vnum[mesh], nt = m.mesh_tnum[mesh];
  if (nvert) *nvert = nv;
  if (ntri) *ntri = nt;
  if (vertices) {
    if (nvert_len != (size_t)nv * 3) return fail(PG_ERR_LENGTH, "mesh vertices: buffer must hold 3 x nvert floats");
    for (int k = 0; k < 3 * nv; k++) vertices[k] = (float)m.mesh_vert[3 * m.mesh_vadr[mesh] + k];
  }
  if (triangles) {
    if (ntri_len != (size_t)nt * 3) return fail(PG_ERR_LENGTH, "mesh triangles: buffer must hold 3 x ntri indices");
    for (int k = 0; k < 3 * nt; k++) triangles[k] = (uint32_t)m.mesh_tri[3 * m.mesh_tadr[mesh] + k];
  }
  return PG_OK;
}

int pg_camera_fovy(const pg_handle* h, int64_t cam, float* fovy) {
  if (!h || !fovy) return fail(PG_ERR_INVALID, "NULL argument");
  if (cam < 0 || cam >= h->hm.ncam) return fail(PG_ERR_INVALID, "camera id out of range");
  *fovy = (float)h->hm.cam_fovy[cam];
  return PG_OK;
}

int pg_name_of(const pg_handle* h, int table, int64_t id, char* buf, size_t len) {
  if (!h || !buf || len == 0) return fail(PG_ERR_INVALID, "NULL argument");
  if (table < 0 || table > 5) return fail(PG_ERR_INVALID, "unknown name table");
  const auto& t = h->hm.names[table];
  if (id < 0 || id >= (int64_t)t.size()) return fail(PG_ERR_INVALID, "name id out of range");
  size_t n = std::min(t[id].size(), len - 1);
  std::memcpy(buf, t[id].data(), n);
  buf[n] = 0;
  return PG_OK;
}

int pg_set_solver(pg_handle* h, int kind, int max_iter, double tolerance, int warm_mode) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (kind > 1 || warm_mode > 2) return fail(PG_ERR_INVALID, "unknown solver or warm-start mode");
  if (kind == PG_SOLVER_PGS && !h->prev_con && h->n > 0) {
    // the previous step's contacts and impulses of every env (solver.rs:254-289)
    CK(cudaSetDevice(h->device));
    size_t per = (size_t)std::max(h->dm.maxcon, 1) * P_STRIDE;
    CK(cudaMalloc(&h->prev_con, sizeof(double) * per * h->n));
    CK(cudaMalloc(&h->prev_ncon, sizeof(int32_t) * h->n));
    CK(cudaMemsetAsync(h->prev_ncon, 0, sizeof(int32_t) * h->n, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  if (warm_mode == PG_WARM_LEARNED && !h->mlp_loaded)
    return fail(PG_ERR_UNSUPPORTED, "no learned warm start is loaded (pg_set_warm_mlp)");
  if (kind >= 0) h->dm.solver = kind;
  if (max_iter >= 0) h->dm.iterations = max_iter;
  if (tolerance >= 0) h->dm.tolerance = tolerance;
  if (warm_mode >= 0) h->warm_mode = warm_mode;
  h->version++;
  return PG_OK;
}

int pg_stats(pg_handle* h, int64_t start, int64_t end, int32_t* iters, int32_t* ncon, int32_t* nrows, int32_t* status) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  if (end == start) return PG_OK;
  CK(cudaSetDevice(h->device));
  size_t b = sizeof(int32_t) * (end - start);
  if (iters) CK(cudaMemcpyAsync(iters, h->iters + start, b, cudaMemcpyDeviceToHost, h->stream));
  if (ncon) CK(cudaMemcpyAsync(ncon, h->ncon + start, b, cudaMemcpyDeviceToHost, h->stream));
  if (nrows) CK(cudaMemcpyAsync(nrows, h->nrows + start, b, cudaMemcpyDeviceToHost, h->stream));
  if (status) CK(cudaMemcpyAsync(status, h->status + start, b, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return PG_OK;
}

int pg_debug_forward(pg_handle* h, int64_t env, double* qm, double* qfrc_bias, double* contacts, int64_t maxcon,
                     int64_t* ncon) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (env < 0 || env >= h->n) return fail(PG_ERR_INVALID, "env out of range");
  if (maxcon < 0) return fail(PG_ERR_INVALID, "maxcon must be non-negative");
  CK(cudaSetDevice(h->device));
  int nv = h->hm.nv;
  // the smooth-dynamics and collision phases of one env leave M, the bias
  // force and the contacts in that env's work record
  StepArgs a = make_args(h);
  a.start = (int)env;
  a.count = 1;
  int rc = launch_status(launch_smooth_collide(a, fit(h->cfg, 1), h->stream));
  if (rc) return rc;
  const WorkLayout& k = h->k;
  std::vector<double> out(k.stride);
  CK(cudaMemcpyAsync(out.data(), h->work + (size_t)env * k.stride, sizeof(double) * k.stride, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (qm) std::memcpy(qm, out.data() + k.qm, sizeof(double) * nv * nv);
  if (qfrc_bias) std::memcpy(qfrc_bias, out.data() + k.bias, sizeof(double) * nv);
  int64_t n = (int64_t)out[k.meta + K_META_NCON];
  if (ncon) *ncon = n;
  if (contacts)
    for (int64_t c = 0; c < std::min(n, maxcon); c++)
      std::memcpy(contacts + 13 * c, out.data() + k.contacts + C_STRIDE * c, sizeof(double) * 13);
  return PG_OK;
}

int pg_invweight(pg_handle* h, int64_t env, double* body, double* dof) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (env < 0 || env >= h->n) return fail(PG_ERR_INVALID, "env out of range");
  std::vector<double> blk;
  int rc = read_params(h, env, env + 1, blk);
  if (rc) return rc;
  if (body) std::memcpy(body, blk.data() + h->dm.p_body_invw, sizeof(double) * 2 * h->hm.nbody);
  if (dof) std::memcpy(dof, blk.data() + h->dm.p_dof_invw, sizeof(double) * h->hm.nv);
  return PG_OK;
}

int pg_set_launch(pg_handle* h, int lanes_per_env, int envs_per_block) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  // the shape applies to every phase kernel of the substep
  SubstepCfg c = h->cfg;
  for (LaunchCfg* p : {&c.smooth, &c.collide, &c.newton}) {
    if (lanes_per_env > 0) p->G = lanes_per_env;
    if (envs_per_block > 0) p->tiles_per_block = envs_per_block;
  }
  CK(cudaSetDevice(h->device));
  return apply_cfg(h, c);
}

int pg_get_launch(const pg_handle* h, int* lanes_per_env, int* envs_per_block, int* blocks) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  // the Newton phase's shape (the longest-running kernel of a substep)
  if (lanes_per_env) *lanes_per_env = h->cfg.newton.G;
  if (envs_per_block) *envs_per_block = h->cfg.newton.tiles_per_block;
  if (blocks) *blocks = h->cfg.newton.blocks;
  return PG_OK;
}

int pg_phase_launch(const pg_handle* h, int phase, int* lanes_per_env, int* envs_per_block, int* blocks) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (phase < 0 || phase > 2) return fail(PG_ERR_INVALID, "phase must be 0, 1 or 2");
  const LaunchCfg& c = phase == 0 ? h->cfg.smooth : phase == 1 ? h->cfg.collide : h->cfg.newton;
  if (lanes_per_env) *lanes_per_env = c.G;
  if (envs_per_block) *envs_per_block = c.tiles_per_block;
  if (blocks) *blocks = c.blocks;
  return PG_OK;
}

int pg_autotune(pg_handle* h, int64_t nstep) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  if (h->n == 0) return PG_OK;
  if (nstep < 1) nstep = 1;
  CK(cudaSetDevice(h->device));
  const HostModel& m = h->hm;
  size_t n = h->n;
  // save the state the trial steps will overwrite
  std::vector<double*> fields = {h->qpos, h->qvel, h->ctrl, h->qacc, h->applied};
  std::vector<size_t> widths = {(size_t)m.nq, (size_t)m.nv, (size_t)m.nu, (size_t)m.nv, (size_t)m.nv};
  std::vector<void*> saved;
  for (size_t k = 0; k < fields.size(); k++) {
    void* p = nullptr;
    CK(cudaMalloc(&p, sizeof(double) * n * std::max<size_t>(widths[k], 1)));
    CK(cudaMemcpyAsync(p, fields[k], sizeof(double) * n * widths[k], cudaMemcpyDeviceToDevice, h->stream));
    saved.push_back(p);
  }
  auto restore = [&]() {
    for (size_t k = 0; k < fields.size(); k++)
      cudaMemcpyAsync(fields[k], saved[k], sizeof(double) * n * widths[k], cudaMemcpyDeviceToDevice, h->stream);
  };
  // coordinate search: each phase's shape in turn, the others held at the
  // best found so far. A candidate is timed on its own phase kernel only
  // (events around it in `nstep` substeps launched phase by phase), the
  // fastest of three runs from the saved state after one warm-up run: the
  // other phases' noise would otherwise decide between shapes a few percent
  // apart. Each run starts with the L2 cache flushed (a write twice its
  // size after the state is restored), as a step does when the caller's own
  // work runs between steps: with the work record already in L2 the smooth
  // phase's shapes tie, with a cold L2 they differ by 5%.
  SubstepCfg best = h->cfg;
  int l2_bytes = 0;
  if (cudaDeviceGetAttribute(&l2_bytes, cudaDevAttrL2CacheSize, h->device) != cudaSuccess) l2_bytes = 0;
  size_t flush_bytes = 2 * (size_t)std::max(l2_bytes, 0);
  void* flush = nullptr;
  if (flush_bytes) CK(cudaMalloc(&flush, flush_bytes));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int rc = PG_OK;
  auto trial = [&](const SubstepCfg& c, int phase, float* ms) -> int {
    if (ensure_scratch(h, c) != PG_OK) return 1;
    h->cfg = c;
    StepArgs a = make_args(h);
    a.start = 0;
    a.count = (int)n;
    a.nstep = (int)nstep;
    SubstepCfg f = fit(c, (int64_t)n);
    const LaunchCfg* shape[3] = {&f.smooth, &f.collide, &f.newton};
    *ms = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
      restore();
      if (flush) cudaMemsetAsync(flush, rep, flush_bytes, h->stream);
      float tot = 0.0f;
      for (int64_t k = 0; k < nstep; k++) {
        a.sidx = (int)k;
        cudaError_t e = reset_queue(a, h->stream);
        for (int p = 0; p < 3 && e == cudaSuccess; p++) {
          if (p == phase) e = cudaEventRecord(e0, h->stream);
          if (e == cudaSuccess) e = launch_phase(p, a, *shape[p], h->stream);
          if (e == cudaSuccess && p == phase) e = cudaEventRecord(e1, h->stream);
        }
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float t = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
        if (e != cudaSuccess) {
          rc = cuda_fail(e, "autotune trial");
          return 1;
        }
        tot += t;
      }
      if (rep > 0) *ms = std::min(*ms, tot);
    }
    return 0;
  };
  for (int phase : {K_SMOOTH, K_COLLIDE, K_NEWTON}) {
    if (rc) break;
    float best_ms = 1e30f;
    if (trial(best, phase, &best_ms)) best_ms = 1e30f;
    for (int G : {8, 16, 32}) {
      for (int tpb : {1, 2, 4, 8, 16}) {
        if (rc) break;
        if (tpb * G < 32 || tpb * G > 256) continue;
        SubstepCfg c = best;
        LaunchCfg& slot = phase == K_SMOOTH ? c.smooth : phase == K_COLLIDE ? c.collide : c.newton;
        if (choose_grid(h, phase, LaunchCfg{G, tpb, 0}, &slot) != PG_OK) continue;
        float ms = 0;
        if (trial(c, phase, &ms)) continue;
        if (ms < best_ms) {
          best_ms = ms;
          best = c;
        }
      }
    }
  }
  restore();
  cudaStreamSynchronize(h->stream);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (void* p : saved) cudaFree(p);
  if (flush) cudaFree(flush);
  if (!rc) g_err.clear();
  // re-apply the winner so every kernel's shared-memory attribute matches it
  if (!rc) rc = apply_cfg(h, best);
  clear_graphs(h);
  h->version++;
  return rc;
}

int pg_time_phases(pg_handle* h, int64_t start, int64_t end, int64_t nstep, const double* ctrl_dev, float* ms_out) {
  if (!h || !ms_out) return fail(PG_ERR_INVALID, "NULL argument");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  if (nstep < 0 || nstep > (1 << 30)) return fail(PG_ERR_INVALID, "nstep out of range");
  for (int k = 0; k < 4; k++) ms_out[k] = 0.0f;
  int64_t cnt = end - start;
  if (cnt == 0 || nstep == 0) return PG_OK;
  CK(cudaSetDevice(h->device));
  if (h->hm.nu > 0 && ctrl_dev)
    CK(cudaMemcpyAsync(h->ctrl + start * h->hm.nu, ctrl_dev, sizeof(double) * cnt * h->hm.nu, cudaMemcpyDeviceToDevice,
                       h->stream));
  StepArgs a = make_args(h);
  a.start = (int)start;
  a.count = (int)cnt;
  a.nstep = (int)nstep;
  SubstepCfg c = fit(h->cfg, cnt);
  // the learned start's inference runs between the collision and Newton
  // phases, as launch_substep orders it; it is timed on its own
  const bool learned = a.learn.mode == LEARN_PREDICT && a.warm_mode == WARM_LEARNED;
  cudaEvent_t ev[5];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  cudaError_t e = cudaSuccess;
  for (int64_t k = 0; k < nstep && e == cudaSuccess; k++) {
    a.sidx = (int)k;
    e = reset_queue(a, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[0], h->stream);
    if (e == cudaSuccess) e = launch_phase(K_SMOOTH, a, c.smooth, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[1], h->stream);
    if (e == cudaSuccess) e = launch_phase(K_COLLIDE, a, c.collide, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2], h->stream);
    if (e == cudaSuccess && learned) e = launch_learn(a, true, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[3], h->stream);
    if (e == cudaSuccess) e = launch_phase(K_NEWTON, a, c.newton, h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[4], h->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[4]);
    const int slot[4] = {0, 1, 3, 2};  // smooth, collide, mlp, newton -> ms_out order
    for (int p = 0; p < 4 && e == cudaSuccess; p++) {
      float ms = 0.0f;
      e = cudaEventElapsedTime(&ms, ev[p], ev[p + 1]);
      if (slot[p] != 3 || learned) ms_out[slot[p]] += ms;  // no inference launched: 0
    }
  }
  for (auto& x : ev) cudaEventDestroy(x);
  if (e != cudaSuccess) return cuda_fail(e, "pg_time_phases");
  return PG_OK;
}

// the learned warm start's contact list: every env's touching contacts, up
// to 32 per env on average
static int64_t learn_cap(const Handle* h) {
  int64_t cap = h->n * (int64_t)std::min(std::max(h->dm.maxcon, 1), 32);
  return std::min<int64_t>(cap, (1ll << 30) / LEARN_NF);
}
static int ensure_learn(Handle* h) {
  if (h->learn.feat) return PG_OK;
  int64_t cap = learn_cap(h);
  h->learn.cap = (int)cap;
  CK(cudaMalloc(&h->learn.items, sizeof(int) * cap * 2));
  CK(cudaMalloc(&h->learn.feat, sizeof(float) * cap * LEARN_NF));
  CK(cudaMalloc(&h->learn.force, sizeof(float) * cap * 3));
  CK(cudaMalloc(&h->learn.rows, sizeof(float) * cap * 4));
  return PG_OK;
}

int pg_set_warm_mlp(pg_handle* h, const float* weights, size_t len) {
  if (!h || !weights) return fail(PG_ERR_INVALID, "NULL argument");
  if (len != (size_t)MLP_SIZE) return fail(PG_ERR_LENGTH, "warm-start network must hold 36662 floats");
  for (size_t k = 0; k < len; k++)
    if (!std::isfinite(weights[k])) return fail(PG_ERR_INVALID, "warm-start network has a non-finite weight");
  CK(cudaSetDevice(h->device));
  int rc = ensure_learn(h);
  if (rc) return rc;
  if (!h->learn.mlp_w) {
    uint16_t* w = nullptr;
    float* f = nullptr;
    int* err = nullptr;
    CK(cudaMalloc(&w, sizeof(uint16_t) * MLP_BF16_ELEMS));
    CK(cudaMalloc(&f, sizeof(float) * MLP_F32_ELEMS));
    CK(cudaMalloc(&err, sizeof(int)));
    CK(cudaMemset(err, 0, sizeof(int)));
    h->learn.mlp_w = w;
    h->learn.mlp_f = f;
    h->learn.mlp_err = err;
  }
  std::vector<uint16_t> wb(MLP_BF16_ELEMS);
  std::vector<float> fb(MLP_F32_ELEMS);
  mlp_pack(weights, wb.data(), fb.data());
  CK(cudaMemcpyAsync((void*)h->learn.mlp_w, wb.data(), sizeof(uint16_t) * wb.size(), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync((void*)h->learn.mlp_f, fb.data(), sizeof(float) * fb.size(), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  CK(mlp_prepare());
  CK(learn_prepare());
  h->learn.mode = LEARN_PREDICT;
  h->mlp_loaded = true;
  h->version++;
  return PG_OK;
}

int pg_warm_samples(pg_handle* h, int64_t start, int64_t end, float* X, size_t xlen, float* rows, size_t rlen,
                    int64_t* n) {
  if (!h || !n) return fail(PG_ERR_INVALID, "NULL argument");
  int rc = check_range(h, start, end);
  if (rc) return rc;
  *n = 0;
  if (end == start) return PG_OK;
  CK(cudaSetDevice(h->device));
  if ((rc = ensure_learn(h))) return rc;
  if (xlen < (size_t)h->learn.cap * LEARN_NF || rlen < (size_t)h->learn.cap * 4)
    return fail(PG_ERR_LENGTH, "sample buffers must hold pg_warm_capacity samples");
  // one substep with the contact list on and the converged row forces
  // dumped; rows the dump does not reach stay NaN and are dropped
  CK(cudaMemsetAsync(h->learn.rows, 0xFF, sizeof(float) * h->learn.cap * 4, h->stream));
  StepArgs a = make_args(h);
  a.learn.mode = LEARN_DUMP;
  a.start = (int)start;
  a.count = (int)(end - start);
  a.nstep = 1;
  a.sidx = 0;
  if ((rc = launch_status(launch_substep(a, fit(h->cfg, end - start), h->stream)))) return rc;
  int count = 0;
  CK(cudaMemcpyAsync(&count, h->queue + Q_LEARN, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  int64_t m = std::min(count, h->learn.cap);
  std::vector<float> fx((size_t)m * LEARN_NF), fr((size_t)m * 4);
  if (m) {
    CK(cudaMemcpyAsync(fx.data(), h->learn.feat, sizeof(float) * fx.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(fr.data(), h->learn.rows, sizeof(float) * fr.size(), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  int64_t k = 0;
  for (int64_t i = 0; i < m; i++) {
    if (!(std::isfinite(fr[4 * i]) && std::isfinite(fr[4 * i + 1]) && std::isfinite(fr[4 * i + 2]) &&
          std::isfinite(fr[4 * i + 3])))
      continue;
    std::memcpy(X + k * LEARN_NF, &fx[i * LEARN_NF], sizeof(float) * LEARN_NF);
    std::memcpy(rows + k * 4, &fr[4 * i], sizeof(float) * 4);
    k++;
  }
  *n = k;
  return PG_OK;
}

int64_t pg_warm_capacity(const pg_handle* h) { return h ? learn_cap(h) : -1; }

int pg_synchronize(pg_handle* h) {
  if (!h) return fail(PG_ERR_INVALID, "NULL handle");
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  return PG_OK;
}

int pg_field_device_ptr(pg_handle* h, int field, double** dev_ptr) {
  if (!h || !dev_ptr) return fail(PG_ERR_INVALID, "NULL argument");
  double* p = field_ptr(h, field);
  if (!p) return fail(PG_ERR_INVALID, "unknown field");
  *dev_ptr = p;
  return PG_OK;
}

void* pg_stream(pg_handle* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"
