// Oracle (test infrastructure only): C API used from Python (ctypes) by the
// tests, the smoke check and bench.py's CPU-baseline leg. It mirrors the CPU
// backend behind the reference's Physics trait
// (crates/pippin-env/src/pippin_cpu.rs:14-206) and Batch::rollout
// (crates/pippin/src/batch.rs:46-59), threaded like the reference's rayon
// chunking (4 chunks per thread, batch.rs:70-72) on a persistent pool.
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <set>
#include <thread>

#include "om_model.h"

using namespace om;

namespace {

class Pool {
 public:
  explicit Pool(int n) : n_(n < 1 ? 1 : n) {
    for (int i = 1; i < n_; i++) th_.emplace_back([this, i] { loop(i); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
      gen_++;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  int size() const { return n_; }
  // run fn(chunk_begin, chunk_end) over [0, n) in chunks pulled dynamically
  void run(size_t n, size_t chunk, const std::function<void(size_t, size_t)>& fn) {
    if (n == 0) return;
    {
      std::lock_guard<std::mutex> g(mu_);
      fn_ = &fn;
      n_items_ = n;
      chunk_ = chunk < 1 ? 1 : chunk;
      next_.store(0);
      pending_ = n_ - 1;
      gen_++;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [this] { return pending_ == 0; });
    fn_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      size_t b = next_.fetch_add(chunk_);
      if (b >= n_items_) break;
      size_t e = std::min(n_items_, b + chunk_);
      (*fn_)(b, e);
    }
  }
  void loop(int) {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
      }
      work();
      {
        std::lock_guard<std::mutex> g(mu_);
        if (--pending_ == 0) done_cv_.notify_all();
      }
    }
  }
  int n_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  uint64_t gen_ = 0;
  bool stop_ = false;
  int pending_ = 0;
  const std::function<void(size_t, size_t)>* fn_ = nullptr;
  size_t n_items_ = 0, chunk_ = 1;
  std::atomic<size_t> next_{0};
};

struct Sim {
  std::shared_ptr<Model> base;
  std::vector<std::shared_ptr<Model>> models;
  std::vector<Data> envs;
  std::unique_ptr<Pool> pool;
  std::mutex flop_mu;
  double flops[ST_COUNT] = {0};
};

void copy_err(const std::string& s, char* err, size_t errlen) {
  if (!err || errlen == 0) return;
  size_t n = std::min(s.size(), errlen - 1);
  std::memcpy(err, s.data(), n);
  err[n] = 0;
}

// flops counted on worker threads are summed into the handle
void collect_flops(Sim* s) {
  std::lock_guard<std::mutex> g(s->flop_mu);
  for (int k = 0; k < ST_COUNT; k++) {
    s->flops[k] += g_flops[k];
    g_flops[k] = 0;
  }
}

// envs [start, end) in chunks of n / (4 * threads), each chunk's thread
// flushing its operation counters when the chunk is done
void run_and_collect(Sim* s, size_t start, size_t end, const std::function<void(size_t)>& body) {
  size_t n = end - start;
  size_t chunk = std::max<size_t>(1, n / (4 * (size_t)s->pool->size()));
  s->pool->run(n, chunk, [&](size_t b, size_t e) {
    for (size_t i = b; i < e; i++) body(start + i);
#if OM_COUNT_FLOPS
    collect_flops(s);
#endif
  });
}

Model& own_model(Sim* s, size_t i) {
  if (s->models[i].use_count() > 1) s->models[i] = std::make_shared<Model>(*s->models[i]);
  return *s->models[i];
}

Real* field_ptr(Data& d, int f) {
  switch (f) {
    case 0: return d.qpos.data();
    case 1: return d.qvel.data();
    case 2: return d.ctrl.data();
    case 3: return d.qacc.data();
    case 4: return d.qfrc_applied.data();
  }
  return nullptr;
}
int field_width(const Model& m, int f) {
  switch (f) {
    case 0: return m.nq;
    case 1: return m.nv;
    case 2: return m.nu;
    case 3: return m.nv;
    case 4: return m.nv;
  }
  return -1;
}

}  // namespace

extern "C" {

void* om_create(const void* blob, size_t bytes, int n_envs, int n_threads, char* err, size_t errlen) {
  std::string e;
  auto m = load_blob(blob, bytes, &e);
  if (!m) {
    copy_err(e, err, errlen);
    return nullptr;
  }
  if (n_envs < 0) {
    copy_err("n_envs must be non-negative", err, errlen);
    return nullptr;
  }
  Sim* s = new Sim;
  s->base = m;
  Data proto;
  data_init(*m, proto);
  kinematics(*m, proto);
  s->models.assign(n_envs, m);
  s->envs.assign(n_envs, proto);
  if (n_threads <= 0) n_threads = (int)std::thread::hardware_concurrency();
  s->pool.reset(new Pool(n_threads));
  for (int k = 0; k < ST_COUNT; k++) g_flops[k] = 0;
  return s;
}

void om_destroy(void* h) { delete (Sim*)h; }

int om_num_threads(void* h) { return ((Sim*)h)->pool->size(); }

// nq, nv, nu, nbody, njnt, ngeom, ncam, nmesh
void om_dims(void* h, int64_t* out) {
  const Model& m = *((Sim*)h)->base;
  out[0] = m.nq;
  out[1] = m.nv;
  out[2] = m.nu;
  out[3] = m.nbody();
  out[4] = m.njnt();
  out[5] = m.ngeom();
  out[6] = (int64_t)m.cam_body.size();
  out[7] = (int64_t)m.mesh_hull.size();
}

// solver kind (0 Newton, 1 PGS), iteration cap and tolerance for every env
void om_set_solver(void* h, int kind, int iterations, double tolerance) {
  Sim* s = (Sim*)h;
  auto apply = [&](Model& m) {
    if (kind >= 0) m.solver.kind = kind;
    if (iterations >= 0) m.solver.iterations = iterations;
    if (tolerance >= 0) m.solver.tolerance = tolerance;
  };
  // models may be shared between envs (copy on write): update each once
  std::set<Model*> seen;
  if (seen.insert(s->base.get()).second) apply(*s->base);
  for (auto& m : s->models)
    if (seen.insert(m.get()).second) apply(*m);
}

// pippin_cpu.rs:98-112: nstep steps per env, then kinematics for poses
void om_step(void* h, int64_t start, int64_t end, int nstep) {
  Sim* s = (Sim*)h;
  run_and_collect(s, start, end, [&](size_t i) {
    const Model& m = *s->models[i];
    Data& d = s->envs[i];
    for (int t = 0; t < nstep; t++) {
      step(m, d);
      if (d.status) break;
    }
    kinematics(m, d);
  });
}

// batch.rs:46-59: ctrl (envs, nstep, nu); qpos after every step (envs, nstep, nq)
void om_rollout(void* h, int64_t start, int64_t end, int nstep, const double* ctrl, double* qpos_out) {
  Sim* s = (Sim*)h;
  const Model& b = *s->base;
  int nu = b.nu, nq = b.nq;
  run_and_collect(s, start, end, [&](size_t i) {
    const Model& m = *s->models[i];
    Data& d = s->envs[i];
    size_t k = i - start;
    for (int t = 0; t < nstep; t++) {
      std::memcpy(d.ctrl.data(), ctrl + ((size_t)k * nstep + t) * nu, sizeof(double) * nu);
      step(m, d);
      if (qpos_out) std::memcpy(qpos_out + ((size_t)k * nstep + t) * nq, d.qpos.data(), sizeof(double) * nq);
    }
  });
}

// forward only (kinematics .. collide), no integration
void om_forward(void* h, int64_t start, int64_t end) {
  Sim* s = (Sim*)h;
  run_and_collect(s, start, end, [&](size_t i) { forward(*s->models[i], s->envs[i]); });
}

void om_kinematics(void* h, int64_t start, int64_t end) {
  Sim* s = (Sim*)h;
  for (int64_t i = start; i < end; i++) kinematics(*s->models[i], s->envs[i]);
}

// data.rs:122-131 + kinematics (pippin_cpu.rs:114-120)
void om_reset(void* h, const int64_t* ids, int64_t n) {
  Sim* s = (Sim*)h;
  for (int64_t k = 0; k < n; k++) {
    size_t i = ids[k];
    data_reset(*s->models[i], s->envs[i]);
    kinematics(*s->models[i], s->envs[i]);
  }
}

// fields: 0 qpos, 1 qvel, 2 ctrl, 3 qacc, 4 qfrc_applied; shaped (envs, width)
int om_get(void* h, int field, int64_t start, int64_t end, double* out) {
  Sim* s = (Sim*)h;
  int w = field_width(*s->base, field);
  if (w < 0) return -1;
  for (int64_t i = start; i < end; i++) std::memcpy(out + (i - start) * w, field_ptr(s->envs[i], field), 8 * w);
  return 0;
}
int om_set(void* h, int field, int64_t start, int64_t end, const double* src) {
  Sim* s = (Sim*)h;
  int w = field_width(*s->base, field);
  if (w < 0) return -1;
  for (int64_t i = start; i < end; i++) {
    std::memcpy(field_ptr(s->envs[i], field), src + (i - start) * w, 8 * w);
    if (field == 0) kinematics(*s->models[i], s->envs[i]);
  }
  return 0;
}

// pippin_cpu.rs:122-131: validate on a clone of the base model, then apply
int om_set_param(void* h, int p, int id, int64_t start, int64_t end, const double* vals, char* err, size_t errlen) {
  Sim* s = (Sim*)h;
  if (p < 0 || p >= P_COUNT) {
    copy_err("unknown parameter", err, errlen);
    return 1;
  }
  int w = param_width(*s->base, p);
  std::string e;
  if (end > start) {
    Model probe = *s->base;
    if (!set_param(probe, p, id, vals, w, &e)) {
      copy_err(e, err, errlen);
      return 1;
    }
  }
  for (int64_t i = start; i < end; i++)
    if (!set_param(own_model(s, i), p, id, vals + (i - start) * w, w, &e)) {
      copy_err(e, err, errlen);
      return 1;
    }
  return 0;
}
int om_get_param(void* h, int p, int id, int64_t start, int64_t end, double* out, char* err, size_t errlen) {
  Sim* s = (Sim*)h;
  if (p < 0 || p >= P_COUNT) {
    copy_err("unknown parameter", err, errlen);
    return 1;
  }
  if (id < 0 || id >= param_count(*s->base, p)) {
    copy_err("id out of range", err, errlen);
    return 1;
  }
  int w = param_width(*s->base, p);
  for (int64_t i = start; i < end; i++) get_param(*s->models[i], p, id, out + (i - start) * w);
  return 0;
}
int om_param_width(void* h, int p) { return param_width(*((Sim*)h)->base, p); }

// pippin_cpu.rs:189-205: Pose = {pos f32[3], mat f32[9]} (12 floats)
void om_poses(void* h, int64_t start, int64_t end, float* geoms, float* cams) {
  Sim* s = (Sim*)h;
  const Model& m = *s->base;
  int ng = m.ngeom(), nc = (int)m.cam_body.size();
  for (int64_t i = start; i < end; i++) {
    const Data& d = s->envs[i];
    int64_t k = i - start;
    for (int g = 0; g < ng; g++) {
      float* o = geoms + (k * ng + g) * 12;
      for (int a = 0; a < 3; a++) o[a] = (float)d.geom_xpos[g][a];
      for (int a = 0; a < 9; a++) o[3 + a] = (float)d.geom_xmat[g][a];
    }
    for (int c = 0; c < nc; c++) {
      int b = m.cam_body[c];
      Vec3 pos = d.xpos[b] + mul_vec(d.xmat[b], m.cam_pos[c]);
      Mat3 mat = mul_mat(d.xmat[b], qto_mat(m.cam_quat[c]));
      float* o = cams + (k * nc + c) * 12;
      for (int a = 0; a < 3; a++) o[a] = (float)pos[a];
      for (int a = 0; a < 9; a++) o[3 + a] = (float)mat[a];
    }
  }
}

// pippin_cpu.rs:145-157: Appearance = {rgba f32[4], scale f32[3], pad} (8 floats)
void om_appearance(void* h, int64_t start, int64_t end, float* out) {
  Sim* s = (Sim*)h;
  const Model& b = *s->base;
  int ng = b.ngeom();
  for (int64_t i = start; i < end; i++) {
    const Model& m = *s->models[i];
    for (int g = 0; g < ng; g++) {
      float* o = out + ((i - start) * ng + g) * 8;
      for (int a = 0; a < 4; a++) o[a] = (float)m.geom_rgba[g][a];
      for (int a = 0; a < 3; a++) o[4 + a] = b.geom_size[g][a] > 0.0 ? (float)(m.geom_size[g][a] / b.geom_size[g][a]) : 1.0f;
      o[7] = 0.0f;
    }
  }
}

// per-env diagnostics of the last step: Newton iterations, contacts, rows, status
void om_stats(void* h, int64_t start, int64_t end, int32_t* iters, int32_t* ncon, int32_t* nrows, int32_t* status) {
  Sim* s = (Sim*)h;
  for (int64_t i = start; i < end; i++) {
    const Data& d = s->envs[i];
    int64_t k = i - start;
    if (iters) iters[k] = d.newton_iters;
    if (ncon) ncon[k] = (int32_t)d.contacts.size();
    if (nrows) nrows[k] = d.nrows_last;
    if (status) status[k] = d.status;
  }
}

// Intermediate quantities of one env after om_forward / om_step:
// qm (nv*nv), qfrc_bias (nv), qfrc_constraint (nv); contacts as 13 doubles
// each: pos[3] normal[3] tangent[3] depth g1 g2 feature. Returns ncon.
int om_debug(void* h, int64_t env, double* qm, double* bias, double* qfrc_c, double* contacts, int maxcon) {
  Sim* s = (Sim*)h;
  const Data& d = s->envs[env];
  int nv = s->base->nv;
  if (qm) std::memcpy(qm, d.qm.data(), 8 * (size_t)nv * nv);
  if (bias) std::memcpy(bias, d.qfrc_bias.data(), 8 * (size_t)nv);
  if (qfrc_c) std::memcpy(qfrc_c, d.qfrc_constraint.data(), 8 * (size_t)nv);
  int n = (int)d.contacts.size();
  if (contacts)
    for (int c = 0; c < n && c < maxcon; c++) {
      const Contact& k = d.contacts[c];
      double* o = contacts + 13 * c;
      for (int a = 0; a < 3; a++) {
        o[a] = k.pos[a];
        o[3 + a] = k.normal[a];
        o[6 + a] = k.tangent[a];
      }
      o[9] = k.depth;
      o[10] = k.geom[0];
      o[11] = k.geom[1];
      o[12] = k.feature;
    }
  return n;
}

// per-body xpos/xmat (nbody*12) of one env
void om_body_poses(void* h, int64_t env, double* out) {
  Sim* s = (Sim*)h;
  const Data& d = s->envs[env];
  for (int b = 0; b < s->base->nbody(); b++) {
    for (int a = 0; a < 3; a++) out[12 * b + a] = d.xpos[b][a];
    for (int a = 0; a < 9; a++) out[12 * b + 3 + a] = d.xmat[b][a];
  }
}

// invweight0 of one env's model: body (nbody*2), dof (nv)
void om_invweight(void* h, int64_t env, double* body, double* dof) {
  Sim* s = (Sim*)h;
  const Model& m = *s->models[env];
  for (int b = 0; b < m.nbody(); b++) {
    body[2 * b] = m.body_invweight[b][0];
    body[2 * b + 1] = m.body_invweight[b][1];
  }
  for (int k = 0; k < m.nv; k++) dof[k] = m.dof_invweight[k];
}

// accumulated FP64 operation counts per stage (ST_COUNT entries); reset=1 clears
void om_flops(void* h, double* out, int reset) {
  Sim* s = (Sim*)h;
  collect_flops(s);
  std::lock_guard<std::mutex> g(s->flop_mu);
  for (int k = 0; k < ST_COUNT; k++) {
    if (out) out[k] = s->flops[k];
    if (reset) s->flops[k] = 0;
  }
}

// ---- known-answer hooks for the reference's unit tests ----
double om_impedance(const double* solimp, double pos) { return impedance(solimp, pos); }
double om_vdot(const double* a, const double* b, int64_t n) { return vdot(a, b, n); }
int om_cholesky_block(double* a, int64_t stride, int64_t s0, int64_t s1) { return cholesky_block(a, stride, s0, s1); }
void om_cholesky_solve_block(const double* l, int64_t stride, int64_t s0, int64_t s1, double* x) {
  cholesky_solve_block(l, stride, s0, s1, x);
}
void om_quat_from_axis_angle(const double* axis, double angle, double* q) {
  Quat r = qaxis_angle(v3(axis[0], axis[1], axis[2]), angle);
  for (int k = 0; k < 4; k++) q[k] = r[k];
}
int om_hull_support(const double* verts, int64_t nv, const int32_t* edges, int64_t ne, const double* dirs, int64_t nd,
                    int32_t* out) {
  std::vector<Vec3> pts;
  for (int64_t i = 0; i < nv; i++) pts.push_back(v3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]));
  std::vector<std::array<int, 2>> ed;
  for (int64_t e = 0; e < ne; e++) {
    if (edges[2 * e] < 0 || edges[2 * e] >= nv || edges[2 * e + 1] < 0 || edges[2 * e + 1] >= nv) return -1;
    ed.push_back({edges[2 * e], edges[2 * e + 1]});
  }
  for (int64_t k = 0; k < nd; k++) out[k] = hull_support_walk(pts, ed, v3(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]));
  return 0;
}
void om_quat_to_mat(const double* q, double* m) {
  Mat3 r = qto_mat(Quat{{q[0], q[1], q[2], q[3]}});
  for (int k = 0; k < 9; k++) m[k] = r[k];
}

}  // extern "C"
