// Oracle (test infrastructure only): constraint solvers. Restates
// crates/pippin/src/newton.rs:52-473 (soft rows, islands, dense primal Newton
// with exact line search, cost-gated warm start) and
// crates/pippin/src/solver.rs:38-289 (soft PGS with relax pass and per-contact
// warm start). Summation orders follow the reference: vdot() where it calls
// simd::dot, plain left-to-right sums where it uses Iterator::sum.
#include <algorithm>
#include <numeric>

#include "om_model.h"

namespace om {

// newton.rs:52-66
Real impedance(const Real solimp[5], Real pos) {
  Real dmin = solimp[0], dmax = solimp[1], width = solimp[2], mid = solimp[3], power = solimp[4];
  Real x = rmin(std::fabs(pos) / rmax(width, 1e-12), 1.0);
  if (x >= 1.0 || dmin == dmax) return dmax;
  auto pw = [](Real b, Real e) { return e == 2.0 ? b * b : (e == 1.0 ? b : std::pow(b, e)); };
  Real y = x <= mid ? pw(x, power) / pw(mid, power - 1.0) : 1.0 - pw(1.0 - x, power) / pw(1.0 - mid, power - 1.0);
  return clampr(dmin + y * (dmax - dmin), 1e-4, 0.9999);
}

// solver.rs:53-59
static void point_jac(const Model& m, const std::vector<Spatial>& cdof, int body, Vec3 p, Vec3 dir, Real sign,
                      Real* row) {
  int k = m.body_lastdof[body];
  while (k != -1) {
    row[k] += sign * dot(dir, point_velocity(cdof[k], p));
    k = m.dof_parent[k];
    OM_FLOPS(ST_ROWS, 2 + 5 + 12);
  }
}

// newton.rs:68-111: one dense subproblem
struct Workspace {
  int nv, nr;
  const Real* jac;
  const NRow* rows;
  const Real* qm;
  const Real* damp_h;

  void mul_m(const Real* x, Real* y) const {
    for (int i = 0; i < nv; i++) y[i] = vdot(qm + (size_t)i * nv, x, nv) + damp_h[i] * x[i];
    OM_FLOPS(ST_NEWTON, (Real)nv * (2 * nv + 2));
  }
  const Real* jrow(int r) const { return jac + (size_t)r * nv; }
  Real dot_j(int r, const Real* x) const { return vdot(jrow(r), x, nv); }
  Real cost(const Real* a, const Real* a0, Real* jar, Real* tmp, Real* tmp2) const {
    for (int k = 0; k < nv; k++) tmp[k] = a[k] - a0[k];
    mul_m(tmp, tmp2);
    Real s = 0.0;
    for (int k = 0; k < nv; k++) s += tmp[k] * tmp2[k];
    Real c = 0.5 * s;
    for (int r = 0; r < nr; r++) {
      jar[r] = dot_j(r, a) - rows[r].aref;
      if (rows[r].active(jar[r])) c += 0.5 * rows[r].d * jar[r] * jar[r];
    }
    OM_FLOPS(ST_NEWTON, 3 * nv + 1 + (Real)nr * (2 * nv + 4));
    return c;
  }
};

// newton.rs:113-218
static int build_rows(const Model& m, Data& d) {
  int nv = m.nv;
  Real h = m.timestep;
  const SolverOptions& opt = m.solver;
  std::vector<Real>& jac = d.jac;
  std::vector<NRow>& rows = d.nrows;
  std::vector<Real>& pos = d.pos;
  std::vector<Real>& diag = d.diag;
  jac.clear();
  rows.clear();
  pos.clear();
  diag.clear();
  std::vector<Real> jn(nv), jt1(nv), jt2(nv);
  for (const Contact& c : d.contacts) {
    if (c.depth <= 0.0) continue;  // within margin but not touching
    int g1 = c.geom[0], g2 = c.geom[1];
    int b1 = m.geom_body[g1], b2 = m.geom_body[g2];
    Real mu = rmax(m.geom_friction[g1], m.geom_friction[g2]);
    Vec3 t1, t2;
    contact_frame(c, &t1, &t2);
    std::vector<Real>* rr[3] = {&jn, &jt1, &jt2};
    Vec3 dirs[3] = {c.normal, t1, t2};
    for (int q = 0; q < 3; q++) {
      std::fill(rr[q]->begin(), rr[q]->end(), 0.0);
      point_jac(m, d.cdof, b2, c.pos, dirs[q], 1.0, rr[q]->data());
      point_jac(m, d.cdof, b1, c.pos, dirs[q], -1.0, rr[q]->data());
    }
    Real tran = m.body_invweight[b1][0] + m.body_invweight[b2][0];
    Real dpyr = 2.0 * mu * mu * (1.0 + mu * mu) * tran / opt.impratio;
    OM_FLOPS(ST_ROWS, 8 + 25);
    for (const std::vector<Real>* t : {&jt1, &jt2})
      for (Real s : {1.0, -1.0}) {
        for (int k = 0; k < nv; k++) jac.push_back(jn[k] + s * mu * (*t)[k]);
        pos.push_back(-c.depth);
        diag.push_back(dpyr);
        OM_FLOPS(ST_ROWS, 3 * nv);
      }
  }
  for (int j = 0; j < m.njnt(); j++) {
    if (!m.jnt_limited[j] || !(m.jnt_type[j] == JNT_HINGE || m.jnt_type[j] == JNT_SLIDE)) continue;
    Real q = d.qpos[m.jnt_qposadr[j]];
    int da = m.jnt_dofadr[j];
    Real lo = m.jnt_range[j][0], hi = m.jnt_range[j][1];
    const Real seps[2] = {q - lo, hi - q}, signs[2] = {1.0, -1.0};
    for (int t = 0; t < 2; t++)
      if (seps[t] < 0.0) {
        size_t start = jac.size();
        jac.resize(start + nv, 0.0);
        jac[start + da] = signs[t];
        pos.push_back(seps[t]);
        diag.push_back(m.dof_invweight[da]);
      }
  }
  int n_ineq = (int)pos.size();
  std::vector<std::pair<std::array<Real, 2>, std::array<Real, 5>>> eq_params;
  for (size_t e = 0; e < m.eq_joint1.size(); e++) {
    int j1 = m.eq_joint1[e], j2 = m.eq_joint2[e];
    const auto& c = m.eq_polycoef[e];
    Real q1 = d.qpos[m.jnt_qposadr[j1]] - m.qpos0[m.jnt_qposadr[j1]];
    Real poly = c[0], dpoly = 0.0;
    if (j2 != -1) {
      Real x = d.qpos[m.jnt_qposadr[j2]] - m.qpos0[m.jnt_qposadr[j2]];
      poly = c[0] + x * (c[1] + x * (c[2] + x * (c[3] + x * c[4])));
      dpoly = c[1] + x * (2.0 * c[2] + x * (3.0 * c[3] + x * 4.0 * c[4]));
    }
    size_t start = jac.size();
    jac.resize(start + nv, 0.0);
    jac[start + m.jnt_dofadr[j1]] += 1.0;
    Real dg = m.dof_invweight[m.jnt_dofadr[j1]];
    if (j2 != -1) {
      jac[start + m.jnt_dofadr[j2]] -= dpoly;
      dg += m.dof_invweight[m.jnt_dofadr[j2]];
    }
    pos.push_back(q1 - poly);
    diag.push_back(dg);
    eq_params.push_back({m.eq_solref[e], m.eq_solimp[e]});
  }
  int nr = (int)pos.size();
  if (nr == 0) return 0;
  for (int r = 0; r < nr; r++) {
    bool bilateral = r >= n_ineq;
    std::array<Real, 2> solref;
    std::array<Real, 5> solimp;
    if (bilateral) {
      solref = eq_params[r - n_ineq].first;
      solimp = eq_params[r - n_ineq].second;
    } else {
      solref = {opt.solref[0], opt.solref[1]};
      for (int k = 0; k < 5; k++) solimp[k] = opt.solimp[k];
    }
    Real tc = rmax(solref[0], 2.0 * h), dr = solref[1];
    Real dmax = solimp[1];
    Real b = 2.0 / (dmax * tc);
    Real k = 1.0 / (dmax * dmax * tc * tc * dr * dr);
    const Real* jr = &jac[(size_t)r * nv];
    Real vel = 0.0;
    for (int i = 0; i < nv; i++) vel += jr[i] * d.qvel[i];
    Real imp = impedance(solimp.data(), pos[r]);
    Real reg = rmax((1.0 - imp) / imp * diag[r], 1e-15);
    rows.push_back(NRow{-b * vel - k * imp * pos[r], 1.0 / reg, bilateral});
    OM_FLOPS(ST_ROWS, 2 * nv + 30);
  }
  return nr;
}

// newton.rs:224-358
static int newton_dense(const Workspace& w, Real* a, const Real* warm, int max_iters, Real tolerance,
                        std::vector<Real>& buf) {
  int nv = w.nv, nr = w.nr;
  buf.assign(6 * (size_t)nv + 2 * (size_t)nr + (size_t)nv * nv, 0.0);
  Real* a0 = buf.data();
  Real* grad = a0 + nv;
  Real* p = grad + nv;
  Real* tmp = p + nv;
  Real* tmp2 = tmp + nv;
  Real* mp = tmp2 + nv;
  Real* jar = mp + nv;
  Real* jp = jar + nr;
  Real* hess = jp + nr;
  std::copy(a, a + nv, a0);

  if (warm) {  // newton.rs:238-245: warm start only when it lowers the cost
    Real c0 = w.cost(a0, a0, jar, tmp, tmp2);
    Real c1 = w.cost(warm, a0, jar, tmp, tmp2);
    if (c1 < c0) std::copy(warm, warm + nv, a);
  }
  w.mul_m(a0, tmp);
  Real ss = 0.0;
  for (int k = 0; k < nv; k++) ss += tmp[k] * tmp[k];
  Real scale = 1.0 + std::sqrt(ss);
  OM_FLOPS(ST_NEWTON, 2 * nv + 2);

  int iters = 0;
  bool have_prev = false;
  unsigned __int128 prev_active = 0;
  int maxit = std::max(max_iters, 1);
  while (iters < maxit) {
    iters++;
    unsigned __int128 active = 0;
    for (int k = 0; k < nv; k++) tmp[k] = a[k] - a0[k];
    w.mul_m(tmp, grad);
    OM_FLOPS(ST_NEWTON, nv);
    for (int r = 0; r < nr; r++) {
      jar[r] = w.dot_j(r, a) - w.rows[r].aref;
      OM_FLOPS(ST_NEWTON, 2 * nv);
      if (w.rows[r].active(jar[r])) {
        if (r < 128) active |= ((unsigned __int128)1) << r;
        Real f = w.rows[r].d * jar[r];
        const Real* jr = w.jrow(r);
        for (int k = 0; k < nv; k++) grad[k] += f * jr[k];
        OM_FLOPS(ST_NEWTON, 1 + 2 * nv);
      }
    }
    Real gs = 0.0;
    for (int k = 0; k < nv; k++) gs += grad[k] * grad[k];
    Real gnorm = std::sqrt(gs);
    OM_FLOPS(ST_NEWTON, 2 * nv + 1);
    // newton.rs:273-276 (prev_active starts at u128::MAX, which no 128-row
    // mask equals once iters > 1 compares a real previous mask)
    if (gnorm < tolerance * scale || (nr <= 128 && have_prev && active == prev_active && iters > 1)) break;
    prev_active = active;
    have_prev = true;

    for (int i = 0; i < nv; i++) {
      for (int j = 0; j < nv; j++) hess[(size_t)i * nv + j] = w.qm[(size_t)i * nv + j];
      hess[(size_t)i * nv + i] += w.damp_h[i];
    }
    for (int r = 0; r < nr; r++) {
      if (!w.rows[r].active(jar[r])) continue;
      Real dr = w.rows[r].d;
      const Real* jr = w.jrow(r);
      for (int i = 0; i < nv; i++) {
        if (jr[i] == 0.0) continue;
        Real di = dr * jr[i];
        for (int j = 0; j < nv; j++) hess[(size_t)i * nv + j] += di * jr[j];
        OM_FLOPS(ST_NEWTON, 1 + 2 * nv);
      }
    }
    OM_FLOPS(ST_NEWTON, (Real)nv * nv / 3.0 * nv + nv * nv);
    if (!cholesky(hess, nv)) break;
    for (int k = 0; k < nv; k++) p[k] = -grad[k];
    cholesky_solve(hess, nv, p);
    OM_FLOPS(ST_NEWTON, 2 * nv * nv);

    w.mul_m(p, mp);
    Real mpp = 0.0, mpg = 0.0;
    for (int k = 0; k < nv; k++) mpp += p[k] * mp[k];
    for (int k = 0; k < nv; k++) mpg += tmp[k] * mp[k];
    for (int r = 0; r < nr; r++) jp[r] = w.dot_j(r, p);
    OM_FLOPS(ST_NEWTON, 4 * nv + 2 * (Real)nr * nv);
    auto deriv = [&](Real al, Real* d1o, Real* d2o) {
      Real d1 = al * mpp + mpg, d2 = mpp;
      for (int r = 0; r < nr; r++) {
        Real v = jar[r] + al * jp[r];
        if (w.rows[r].active(v)) {
          Real dq = w.rows[r].d * jp[r];
          d1 += dq * v;
          d2 += dq * jp[r];
          OM_FLOPS(ST_NEWTON, 5);
        }
      }
      OM_FLOPS(ST_NEWTON, 2 + 2 * nr);
      *d1o = d1;
      *d2o = d2;
    };
    Real lo = 0.0, hi = INFINITY, al = 1.0;
    Real d1_0, d2_0;
    deriv(0.0, &d1_0, &d2_0);
    Real ltol = 1e-12 * rmax(std::fabs(d1_0), 1e-30);
    for (int it = 0; it < 50; it++) {
      Real d1, d2;
      deriv(al, &d1, &d2);
      if (std::fabs(d1) <= ltol) break;
      if (d1 < 0.0) lo = al;
      else hi = al;
      Real next = al - d1 / rmax(d2, 1e-30);
      if (next <= lo || next >= hi) next = std::isfinite(hi) ? 0.5 * (lo + hi) : 2.0 * rmax(al, lo);
      if (std::fabs(next - al) <= 1e-14 * rmax(std::fabs(al), 1.0)) {
        al = next;
        break;
      }
      al = next;
    }
    for (int k = 0; k < nv; k++) a[k] += al * p[k];
    OM_FLOPS(ST_NEWTON, 2 * nv);
  }
  return iters;
}

// newton.rs:361-371
static void add_constraint_force(const Workspace& w, const Real* a, const int* idx, Real* qfrc) {
  for (int r = 0; r < w.nr; r++) {
    Real v = w.dot_j(r, a) - w.rows[r].aref;
    if (w.rows[r].active(v)) {
      Real f = -w.rows[r].d * v;
      const Real* jr = w.jrow(r);
      for (int k = 0; k < w.nv; k++) qfrc[idx ? idx[k] : k] += f * jr[k];
    }
  }
}

// newton.rs:378-473
void newton_solve(const Model& m, Data& d, Real* a) {
  int nv = m.nv;
  int nr = build_rows(m, d);
  d.nrows_last = nr;
  std::fill(d.qfrc_constraint.begin(), d.qfrc_constraint.end(), 0.0);
  d.newton_iters = 0;
  if (nr == 0) return;
  std::vector<Real> damp_h(nv, 0.0), buf;
  int max_iters = m.solver.iterations;
  Real tol = m.solver.tolerance;

  int nb = (int)m.dof_blocks.size();
  std::vector<int> block_of(nv, 0);
  for (int b = 0; b < nb; b++)
    for (int k = m.dof_blocks[b].first; k < m.dof_blocks[b].second; k++) block_of[k] = b;
  std::vector<int> parent(nb);
  std::iota(parent.begin(), parent.end(), 0);
  auto find = [&](int x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  std::vector<int> row_block(nr, -1);
  for (int r = 0; r < nr; r++)
    for (int k = 0; k < nv; k++)
      if (d.jac[(size_t)r * nv + k] != 0.0) {
        int b = block_of[k];
        if (row_block[r] == -1) row_block[r] = b;
        else {
          int x = find(row_block[r]), y = find(b);
          if (x != y) parent[std::max(x, y)] = std::min(x, y);
        }
      }
  std::vector<int> island_of_block(nb);
  for (int b = 0; b < nb; b++) island_of_block[b] = find(b);
  std::vector<int> islands;
  for (int r = 0; r < nr; r++)
    if (row_block[r] != -1) islands.push_back(island_of_block[row_block[r]]);
  std::sort(islands.begin(), islands.end());
  islands.erase(std::unique(islands.begin(), islands.end()), islands.end());

  bool single = islands.size() == 1;
  if (single)
    for (int b = 0; b < nb; b++)
      if (island_of_block[b] != islands[0]) single = false;
  int iters = 0;
  if (single) {
    Workspace w{nv, nr, d.jac.data(), d.nrows.data(), d.qm.data(), damp_h.data()};
    iters = newton_dense(w, a, d.qacc.data(), max_iters, tol, buf);
    add_constraint_force(w, a, nullptr, d.qfrc_constraint.data());
  } else {
    std::vector<int> idx, rws;
    std::vector<Real> qm, jac, zeros, sub, warm;
    std::vector<NRow> nrows;
    for (int isl : islands) {
      idx.clear();
      for (int b = 0; b < nb; b++)
        if (island_of_block[b] == isl)
          for (int k = m.dof_blocks[b].first; k < m.dof_blocks[b].second; k++) idx.push_back(k);
      rws.clear();
      for (int r = 0; r < nr; r++)
        if (row_block[r] != -1 && island_of_block[row_block[r]] == isl) rws.push_back(r);
      int k = (int)idx.size();
      qm.clear();
      for (int i : idx)
        for (int j : idx) qm.push_back(d.qm[(size_t)i * nv + j]);
      jac.clear();
      for (int r : rws)
        for (int c : idx) jac.push_back(d.jac[(size_t)r * nv + c]);
      nrows.clear();
      for (int r : rws) nrows.push_back(d.nrows[r]);
      zeros.assign(k, 0.0);
      sub.clear();
      for (int i : idx) sub.push_back(a[i]);
      warm.clear();
      for (int i : idx) warm.push_back(d.qacc[i]);
      Workspace w{k, (int)rws.size(), jac.data(), nrows.data(), qm.data(), zeros.data()};
      iters = std::max(iters, newton_dense(w, sub.data(), warm.data(), max_iters, tol, buf));
      for (int t = 0; t < k; t++) a[idx[t]] = sub[t];
      add_constraint_force(w, sub.data(), idx.data(), d.qfrc_constraint.data());
    }
  }
  d.newton_iters = iters;
}

// ---------------------------------------------------------------- PGS
// solver.rs:38-50
static const Real MAX_BIAS_VELOCITY = 1.0;
static const Real PGS_TOLERANCE = 1e-5;

// solver.rs:254-289
static void pgs_warm_start(Data& d, Real* lambda) {
  const Real MATCH_DIST2 = 0.01 * 0.01;
  if (d.prev_contacts.empty()) return;
  size_t r = 0;
  while (r < d.rows.size()) {
    int ci = d.rows[r].contact;
    if (ci == -1) {
      r++;
      continue;
    }
    const Contact& c = d.contacts[ci];
    Real bd = MATCH_DIST2;
    int bi = -1;
    for (size_t pi = 0; pi < d.prev_contacts.size(); pi++) {
      const Contact& p = d.prev_contacts[pi];
      if (p.geom[0] == c.geom[0] && p.geom[1] == c.geom[1]) {
        Real d2 = norm2(p.pos - c.pos);
        if (d2 < bd) {
          bd = d2;
          bi = (int)pi;
        }
      }
    }
    if (bi != -1) {
      const Contact& p = d.prev_contacts[bi];
      const auto& l = d.prev_lambda[bi];
      Vec3 pt1, pt2, t1, t2;
      contact_frame(p, &pt1, &pt2);
      contact_frame(c, &t1, &t2);
      Vec3 f = pt1 * l[1] + pt2 * l[2];
      lambda[r] = l[0];
      lambda[r + 1] = dot(f, t1);
      lambda[r + 2] = dot(f, t2);
    }
    r += 3;
  }
}

// solver.rs:63-251
void pgs_solve(const Model& m, Data& d, Real* v, std::vector<Real>& v_pos) {
  int nv = m.nv;
  Real h = m.timestep;
  const SolverOptions& opt = m.solver;
  std::vector<PgsRow>& rows = d.rows;
  std::vector<Real>& jac = d.jac;
  rows.clear();
  jac.clear();
  auto push_row = [&]() {
    jac.resize(jac.size() + nv, 0.0);
    return (int)(jac.size() / nv) - 1;
  };
  for (size_t ci = 0; ci < d.contacts.size(); ci++) {
    const Contact& c = d.contacts[ci];
    int g1 = c.geom[0], g2 = c.geom[1];
    int b1 = m.geom_body[g1], b2 = m.geom_body[g2];
    Real mu = rmax(m.geom_friction[g1], m.geom_friction[g2]);
    Vec3 t1, t2;
    contact_frame(c, &t1, &t2);
    int base = (int)rows.size();
    Vec3 dirs[3] = {c.normal, t1, t2};
    for (int r = 0; r < 3; r++) {
      int idx = push_row();
      Real* row = &jac[(size_t)idx * nv];
      point_jac(m, d.cdof, b2, c.pos, dirs[r], 1.0, row);
      point_jac(m, d.cdof, b1, c.pos, dirs[r], -1.0, row);
      PgsRow pr{};
      if (r == 0) {
        pr.kind = ROW_NORMAL;
        pr.sep = -c.depth;
      } else {
        pr.kind = ROW_FRICTION;
        pr.normal = base;
        pr.mu = mu;
      }
      pr.inv_a = 0.0;
      pr.contact = (int)ci;
      rows.push_back(pr);
    }
  }
  for (int j = 0; j < m.njnt(); j++) {
    if (!m.jnt_limited[j] || !(m.jnt_type[j] == JNT_HINGE || m.jnt_type[j] == JNT_SLIDE)) continue;
    Real q = d.qpos[m.jnt_qposadr[j]];
    int da = m.jnt_dofadr[j];
    Real lo = m.jnt_range[j][0], hi = m.jnt_range[j][1];
    Real reach = opt.contact_margin + 2.0 * h * std::fabs(v[da]);
    const Real seps[2] = {q - lo, hi - q}, signs[2] = {1.0, -1.0};
    for (int t = 0; t < 2; t++)
      if (seps[t] < reach) {
        int idx = push_row();
        jac[(size_t)idx * nv + da] = signs[t];
        PgsRow pr{};
        pr.kind = ROW_NORMAL;
        pr.sep = seps[t];
        pr.contact = -1;
        rows.push_back(pr);
      }
  }
  for (size_t e = 0; e < m.eq_joint1.size(); e++) {
    int j1 = m.eq_joint1[e], j2 = m.eq_joint2[e];
    const auto& c = m.eq_polycoef[e];
    Real q1 = d.qpos[m.jnt_qposadr[j1]] - m.qpos0[m.jnt_qposadr[j1]];
    int idx = push_row();
    jac[(size_t)idx * nv + m.jnt_dofadr[j1]] += 1.0;
    Real poly = c[0];
    if (j2 != -1) {
      Real x = d.qpos[m.jnt_qposadr[j2]] - m.qpos0[m.jnt_qposadr[j2]];
      poly = c[0] + x * (c[1] + x * (c[2] + x * (c[3] + x * c[4])));
      jac[(size_t)idx * nv + m.jnt_dofadr[j2]] -= c[1] + x * (2.0 * c[2] + x * (3.0 * c[3] + x * 4.0 * c[4]));
    }
    PgsRow pr{};
    pr.kind = ROW_BILATERAL;
    pr.sep = q1 - poly;
    pr.contact = -1;
    rows.push_back(pr);
  }

  int nr = (int)rows.size();
  d.nrows_last = nr;
  v_pos.assign(v, v + nv);
  if (nr == 0) {
    d.newton_iters = 0;
    std::fill(d.qfrc_constraint.begin(), d.qfrc_constraint.end(), 0.0);
    d.prev_contacts.clear();
    d.prev_lambda.clear();
    return;
  }
  std::vector<Real>& mj = d.minv_jt;
  mj = jac;
  for (int r = 0; r < nr; r++) {
    Real* x = &mj[(size_t)r * nv];
    mass_solve(m, d.qm_chol.data(), x);
    Real a = 0.0;
    for (int k = 0; k < nv; k++) a += jac[(size_t)r * nv + k] * x[k];
    rows[r].inv_a = a > 1e-12 ? 1.0 / a : 0.0;
    OM_FLOPS(ST_PGS, 2 * nv + 1);
  }
  std::vector<Real>& lambda = d.lambda;
  lambda.assign(nr, 0.0);
  pgs_warm_start(d, lambda.data());
  for (int r = 0; r < nr; r++)
    if (lambda[r] != 0.0)
      for (int k = 0; k < nv; k++) v[k] += mj[(size_t)r * nv + k] * lambda[r];

  // solver.rs:44-50
  Real omega = 2.0 * M_PI * opt.contact_hertz;
  Real a1 = 2.0 * opt.contact_damping_ratio + h * omega;
  Real a2 = h * omega * a1;
  Real a3 = 1.0 / (1.0 + a2);
  Real bias_rate = omega / a1, mass_scale = a2 * a3, impulse_scale = a3;

  auto iterate = [&](bool use_bias) {
    Real max_dv = 0.0;
    for (int r = 0; r < nr; r++) {
      const PgsRow row = rows[r];
      if (row.inv_a == 0.0) continue;
      const Real* jr = &jac[(size_t)r * nv];
      Real jv = 0.0;
      for (int k = 0; k < nv; k++) jv += jr[k] * v[k];
      Real nw;
      if (row.kind == ROW_NORMAL) {
        Real s = row.sep + opt.contact_slop;
        Real bias, ms, is;
        if (s > 0.0) {
          bias = s / h;
          ms = 1.0;
          is = 0.0;
        } else if (use_bias) {
          bias = rmax(bias_rate * s, -MAX_BIAS_VELOCITY);
          ms = mass_scale;
          is = impulse_scale;
        } else {
          bias = 0.0;
          ms = 1.0;
          is = 0.0;
        }
        Real delta = -row.inv_a * ms * (jv + bias) - is * lambda[r];
        nw = rmax(lambda[r] + delta, 0.0);
      } else if (row.kind == ROW_BILATERAL) {
        Real bias, ms, is;
        if (use_bias) {
          bias = clampr(bias_rate * row.sep, -MAX_BIAS_VELOCITY, MAX_BIAS_VELOCITY);
          ms = mass_scale;
          is = impulse_scale;
        } else {
          bias = 0.0;
          ms = 1.0;
          is = 0.0;
        }
        nw = lambda[r] - row.inv_a * ms * (jv + bias) - is * lambda[r];
      } else {
        Real bound = row.mu * lambda[row.normal];
        nw = clampr(lambda[r] - row.inv_a * jv, -bound, bound);
      }
      Real dl = nw - lambda[r];
      OM_FLOPS(ST_PGS, 2 * nv + 8);
      if (dl != 0.0) {
        max_dv = rmax(max_dv, std::fabs(dl) / row.inv_a);
        const Real* mr = &mj[(size_t)r * nv];
        for (int k = 0; k < nv; k++) v[k] += mr[k] * dl;
        lambda[r] = nw;
        OM_FLOPS(ST_PGS, 2 * nv + 2);
      }
    }
    return max_dv;
  };
  int sweeps = 0;
  for (int it = 0; it < opt.iterations; it++) {
    sweeps++;
    if (iterate(true) < PGS_TOLERANCE) break;
  }
  v_pos.assign(v, v + nv);
  for (int it = 0; it < std::max(opt.iterations / 3, 2); it++) {
    sweeps++;
    if (iterate(false) < PGS_TOLERANCE) break;
  }
  d.newton_iters = sweeps;  // reported as the solver's iteration count

  std::fill(d.qfrc_constraint.begin(), d.qfrc_constraint.end(), 0.0);
  for (int r = 0; r < nr; r++)
    for (int k = 0; k < nv; k++) d.qfrc_constraint[k] += jac[(size_t)r * nv + k] * lambda[r] / h;
  d.prev_contacts = d.contacts;
  d.prev_lambda.assign(d.contacts.size(), {0.0, 0.0, 0.0});
  for (int r = 0; r < nr; r++) {
    int c = rows[r].contact;
    if (c == -1) continue;
    int slot;
    if (rows[r].kind == ROW_NORMAL) slot = 0;
    else if (rows[r].kind == ROW_FRICTION) slot = r - rows[r].normal;
    else continue;
    d.prev_lambda[c][slot] = lambda[r];
  }
}

}  // namespace om
