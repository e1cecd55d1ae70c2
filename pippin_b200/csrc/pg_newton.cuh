// Contacts, constraint rows and the primal Newton solver of one environment
// on a tile of G lanes. Restates crates/pippin/src/forward.rs:214-260
// (broad + narrow phase), crates/pippin/src/newton.rs:113-473 (pyramidal
// contact rows, joint-limit and joint-equality rows with soft-constraint
// constants, islands over dof blocks, dense Newton with exact line search
// and the cost-gated warm start) and forward.rs:336-480 (substep driver,
// implicit damping, integration).
#pragma once
#include "pg_general.cuh"
#include "pg_dynamics.cuh"
#include "pg_small.cuh"

namespace pg {

// ---------------------------------------------------------------- collide
// Returns the contact count; contacts land in scratch in pair order (and
// hit order within a pair), as in the reference's sequential pair loop.
// The broad phase runs over the pairs G at a time and queues the survivors
// (in pair order) in `queue` (2G ints of shared memory); the narrow phase
// takes them G at a time, one pair per lane, so a batch of narrow-phase
// work waits for G survivors instead of running once per G candidates.
// gs: the tile's shared scratch for general pairs (pointers nullptr when absent).
template <int G>
__device__ int collide(const Tile<G>& T, const DModel& m, const WsLayout& w, const ScrLayout& s, const EnvCtx& e,
                       int* status, int* queue, const GenScratch& gs) {
  int lane = T.lane();
  const double* prm = e.prm;
  const double* gr = e.geo;  // poses and boxes from the tree walk
  double* con = e.con;
  int ncon = 0;
  int st = 0;
  // narrow phase of the queued pairs [0, cnt), contacts appended in order
  auto pose = [&](int g) {
    const double* r = gr + G_STRIDE * g;
    return GPose{m.geom_type[g], ld3(r + G_POS), ld9(r + G_MAT), ld3(prm + m.p_size + 3 * g), m.geom_dataid[g]};
  };
  auto narrow = [&](int cnt) {
    Hits hits;
    hits.n = 0;
    int g1 = 0, g2 = 0;
    bool general = false;
    if (lane < cnt) {
      int p = queue[lane];
      g1 = m.pair_g[2 * p];
      g2 = m.pair_g[2 * p + 1];
      general = needs_general(m.geom_type[g1], m.geom_type[g2]);
      if (!general) collide_primitive(pose(g1), pose(g2), m.margin, hits);
    }
    // the general pairs one after another, each on the whole tile
    for (unsigned gm = T.ballot(general); gm; gm &= gm - 1) {
      int d = __ffs(gm) - 1;
      int h1 = T.bcast(g1, d), h2 = T.bcast(g2, d);
      collide_general(T, m, pose(h1), pose(h2), m.margin, hits, gs, d);
    }
    int nh = hits.n < MAX_HITS ? hits.n : MAX_HITS;
    int tot;
    int off = T.excl_scan(nh, &tot);
    for (int k = 0; k < nh; k++) {
      int c = ncon + off + k;
      if (c >= m.maxcon) {
        st |= ST_CAP_EXCEEDED;
        break;
      }
      double* r = con + C_STRIDE * c;
      const Hit& h = hits.h[k];
      st3(r + C_POS, h.pos);
      st3(r + C_NORMAL, h.normal);
      st3(r + C_TANGENT, h.tangent);
      r[C_DEPTH] = h.depth;
      r[C_G1] = g1;
      r[C_G2] = g2;
      r[C_FEATURE] = k;
      V3 t1, t2;
      contact_frame(h.normal, h.tangent, &t1, &t2);
      st3(r + C_T1, t1);
      st3(r + C_T2, t2);
    }
    ncon += tot;
  };
  int queued = 0;
  for (int base = 0; base < m.npair; base += G) {
    int p = base + lane;
    bool keep = false;
    if (p < m.npair) {
      int g1 = m.pair_g[2 * p], g2 = m.pair_g[2 * p + 1];
      unsigned t1 = (unsigned)prm[m.p_contype + g1], a1 = (unsigned)prm[m.p_conaff + g1];
      unsigned t2 = (unsigned)prm[m.p_contype + g2], a2 = (unsigned)prm[m.p_conaff + g2];
      bool masks = (t1 & a2) != 0 || (t2 & a1) != 0;
      if (masks) {
        const double* r1 = gr + G_STRIDE * g1;
        const double* r2 = gr + G_STRIDE * g2;
        V3 c1 = ld3(r1 + G_AABB), h1 = ld3(r1 + G_AABB + 3);
        V3 c2 = ld3(r2 + G_AABB), h2 = ld3(r2 + G_AABB + 3);
        bool sep = fabs(c1.x - c2.x) > h1.x + h2.x + m.margin || fabs(c1.y - c2.y) > h1.y + h2.y + m.margin ||
                   fabs(c1.z - c2.z) > h1.z + h2.z + m.margin;
        keep = !sep;
      }
    }
    int tot;
    int off = T.excl_scan(keep ? 1 : 0, &tot);
    if (keep) queue[queued + off] = p;  // queued < G before, tot <= G: within 2G
    queued += tot;
    T.sync();
    if (queued >= G) {
      narrow(G);
      T.sync();  // the batch is read; move the rest (fewer than G) to the front
      if (lane < queued - G) queue[lane] = queue[G + lane];
      queued -= G;
      T.sync();
    }
  }
  if (queued > 0) narrow(queued);
  if (ncon > m.maxcon) ncon = m.maxcon;
  *status |= T.ior(st);
  T.sync();
  return ncon;
}

// ---------------------------------------------------------------- rows
// newton.rs:52-66
__device__ inline double impedance(const double* solimp, double pos) {
  double dmin = solimp[0], dmax = solimp[1], width = solimp[2], mid = solimp[3], power = solimp[4];
  double x = fmin(fabs(pos) / fmax(width, 1e-12), 1.0);
  if (x >= 1.0 || dmin == dmax) return dmax;
  auto pw = [](double b, double ex) { return ex == 2.0 ? b * b : (ex == 1.0 ? b : pow(b, ex)); };
  double y = x <= mid ? pw(x, power) / pw(mid, power - 1.0) : 1.0 - pw(1.0 - x, power) / pw(1.0 - mid, power - 1.0);
  return clampd(dmin + y * (dmax - dmin), 1e-4, 0.9999);
}

// Jacobian entry k of a world point on the pair (b1, b2) along `dir`
// (solver.rs:53-59 applied to b2 with +1, then b1 with -1).
__device__ inline double pair_jac(const DModel& m, const double* cdof, int b1, int b2, V3 p, V3 dir, int k) {
  double v = 0.0;
  unsigned long long bit = 1ull << k;
  if (m.body_dofmask[b2] & bit) v += dot(dir, point_vel(ld6(cdof + 6 * k), p));
  if (m.body_dofmask[b1] & bit) v += -1.0 * dot(dir, point_vel(ld6(cdof + 6 * k), p));
  return v;
}

// The learned warm start's contact list: each touching contact (depth > 0,
// in contact order, the order build_rows gives their pyramid rows) takes
// one slot of the env-shared list, recording (env, contact); the env's
// first slot and count go to its work-record meta (count -1 when the list
// is full, and that env's slots below the capacity are marked unused). The
// features and the prediction are formed per slot by learn_kernel.
template <int G>
__device__ void learn_list(const Tile<G>& T, const LearnArgs& L, const EnvCtx& e, int ncon, double* meta) {
  int lane = T.lane();
  const double* con = e.con;
  int nt = 0;
  for (int c = lane; c < ncon; c += G) nt += con[C_STRIDE * c + C_DEPTH] > 0.0 ? 1 : 0;
  nt = T.isum(nt);
  int base = 0;
  if (lane == 0 && nt > 0) base = atomicAdd(L.count, nt);
  base = T.bcast(base, 0);
  bool room = base + nt <= L.cap;
  if (lane == 0) {
    meta[K_META_LBASE] = base;
    meta[K_META_LNUM] = room ? nt : -1;
  }
  if (nt == 0) return;
  if (!room) {
    for (int t = base + lane; t < L.cap && t < base + nt; t += G) L.items[2 * t] = -1;
    return;
  }
  int done = 0;
  for (int c0 = 0; c0 < ncon; c0 += G) {
    int c = c0 + lane;
    bool touch = c < ncon && con[C_STRIDE * c + C_DEPTH] > 0.0;
    int tot;
    int rank = done + T.excl_scan(touch ? 1 : 0, &tot);
    if (touch) {
      L.items[2 * (base + rank)] = e.env;
      L.items[2 * (base + rank) + 1] = c;
    }
    done += tot;
  }
}

// newton.rs:113-218. Returns the row count. Row order: 4 pyramid rows per
// touching contact (contact order), violated joint limits (joint order,
// lower side first), joint equalities.
template <int G>
__device__ int build_rows(const Tile<G>& T, const DModel& m, const WsLayout& w, const ScrLayout& s, const EnvCtx& e,
                          int ncon, int* status) {
  int lane = T.lane(), nv = m.nv;
  const double* ws = e.ws;
  const double* prm = e.prm;
  double* con = e.con;
  double* J = e.scr + s.jac;
  double* R = e.scr + s.rows;
  const double* cdof = ws + w.cdof;
  // touching contacts get 4 rows each; C_ROW records the first one
  int nt = 0;
  for (int base = 0; base < ncon; base += G) {
    int c = base + lane;
    bool touch = c < ncon && con[C_STRIDE * c + C_DEPTH] > 0.0;
    int tot;
    int off = T.excl_scan(touch ? 1 : 0, &tot);
    if (c < ncon) {
      double* r = con + C_STRIDE * c;
      int row = touch ? 4 * (nt + off) : -1;
      if (row + 4 > m.maxrows) row = -1;
      r[C_ROW] = row;
      if (row >= 0) {
        int g1 = (int)r[C_G1], g2 = (int)r[C_G2];
        int b1 = m.geom_body[g1], b2 = m.geom_body[g2];
        double mu = fmax(prm[m.p_friction + g1], prm[m.p_friction + g2]);
        double tran = prm[m.p_body_invw + 2 * b1] + prm[m.p_body_invw + 2 * b2];
        double dpyr = 2.0 * mu * mu * (1.0 + mu * mu) * tran / m.impratio;
        for (int q = 0; q < 4; q++) {
          double* rr = R + R_STRIDE * (row + q);
          rr[R_POS] = -r[C_DEPTH];
          rr[R_DIAG] = dpyr;
          rr[R_FLAGS] = 0.0;
        }
      }
    }
    nt += tot;
  }
  int ncrow = 4 * nt;
  if (ncrow > m.maxrows) {
    *status |= ST_CAP_EXCEEDED;
    ncrow = m.maxrows & ~3;
  }
  T.sync();
  // Jacobian entries: one item per (contact, dof)
  for (int it = lane; it < ncon * nv; it += G) {
    int c = it / nv, k = it % nv;
    const double* r = con + C_STRIDE * c;
    int row = (int)r[C_ROW];
    if (row < 0) continue;
    int g1 = (int)r[C_G1], g2 = (int)r[C_G2];
    int b1 = m.geom_body[g1], b2 = m.geom_body[g2];
    double mu = fmax(prm[m.p_friction + g1], prm[m.p_friction + g2]);
    V3 p = ld3(r + C_POS);
    double jn = pair_jac(m, cdof, b1, b2, p, ld3(r + C_NORMAL), k);
    double jt1 = pair_jac(m, cdof, b1, b2, p, ld3(r + C_T1), k);
    double jt2 = pair_jac(m, cdof, b1, b2, p, ld3(r + C_T2), k);
    J[(row + 0) * nv + k] = jn + mu * jt1;
    J[(row + 1) * nv + k] = jn + (-mu) * jt1;
    J[(row + 2) * nv + k] = jn + mu * jt2;
    J[(row + 3) * nv + k] = jn + (-mu) * jt2;
  }
  // joint limits: count violated sides per joint, then place
  int nl = 0;
  for (int base = 0; base < m.njnt; base += G) {
    int j = base + lane;
    int cnt = 0;
    double sep[2] = {0.0, 0.0};
    int da = 0;
    if (j < m.njnt && m.jnt_limited[j] && (m.jnt_type[j] == JNT_HINGE || m.jnt_type[j] == JNT_SLIDE)) {
      double q = ws[w.qpos + m.jnt_qposadr[j]];
      da = m.jnt_dofadr[j];
      sep[0] = q - m.jnt_range[2 * j];
      sep[1] = m.jnt_range[2 * j + 1] - q;
      cnt = (sep[0] < 0.0 ? 1 : 0) + (sep[1] < 0.0 ? 1 : 0);
    }
    int tot;
    int off = T.excl_scan(cnt, &tot);
    int row = ncrow + nl + off;
    for (int t = 0; t < 2; t++) {
      if (!(sep[t] < 0.0) || cnt == 0) continue;
      if (row < m.maxrows) {
        double* jr = J + row * nv;
        for (int k = 0; k < nv; k++) jr[k] = 0.0;
        jr[da] = t == 0 ? 1.0 : -1.0;
        double* rr = R + R_STRIDE * row;
        rr[R_POS] = sep[t];
        rr[R_DIAG] = prm[m.p_dof_invw + da];
        rr[R_FLAGS] = 0.0;
      }
      row++;
    }
    nl += tot;
  }
  int nineq = ncrow + nl;
  // joint equality rows (bilateral)
  for (int q = lane; q < m.neq; q += G) {
    int row = nineq + q;
    if (row >= m.maxrows) continue;
    int j1 = m.eq_j1[q], j2 = m.eq_j2[q];
    const double* c = m.eq_poly + 5 * q;
    double q1 = ws[w.qpos + m.jnt_qposadr[j1]] - m.qpos0[m.jnt_qposadr[j1]];
    double poly = c[0], dpoly = 0.0;
    if (j2 != -1) {
      double x = ws[w.qpos + m.jnt_qposadr[j2]] - m.qpos0[m.jnt_qposadr[j2]];
      poly = c[0] + x * (c[1] + x * (c[2] + x * (c[3] + x * c[4])));
      dpoly = c[1] + x * (2.0 * c[2] + x * (3.0 * c[3] + x * 4.0 * c[4]));
    }
    double* jr = J + row * nv;
    for (int k = 0; k < nv; k++) jr[k] = 0.0;
    jr[m.jnt_dofadr[j1]] += 1.0;
    double dg = prm[m.p_dof_invw + m.jnt_dofadr[j1]];
    if (j2 != -1) {
      jr[m.jnt_dofadr[j2]] -= dpoly;
      dg += prm[m.p_dof_invw + m.jnt_dofadr[j2]];
    }
    double* rr = R + R_STRIDE * row;
    rr[R_POS] = q1 - poly;
    rr[R_DIAG] = dg;
    rr[R_FLAGS] = 1.0;
  }
  int nr = nineq + m.neq;
  if (nr > m.maxrows) {
    *status |= ST_CAP_EXCEEDED;
    nr = m.maxrows;
  }
  T.sync();
  // reference acceleration and regularisation per row
  const double* qvel = ws + w.qvel;
  for (int r = lane; r < nr; r += G) {
    double* rr = R + R_STRIDE * r;
    bool bil = rr[R_FLAGS] != 0.0;
    const double* solref = m.solref;
    const double* solimp = m.solimp;
    if (bil) {
      int q = r - nineq;
      solref = m.eq_solref + 2 * q;
      solimp = m.eq_solimp + 5 * q;
    }
    double tc = fmax(solref[0], 2.0 * m.timestep), dr = solref[1];
    double dmax = solimp[1];
    double b = 2.0 / (dmax * tc);
    double kk = 1.0 / (dmax * dmax * tc * tc * dr * dr);
    const double* jr = J + r * nv;
    double vel = 0.0;
    for (int i = 0; i < nv; i++) vel += jr[i] * qvel[i];
    double imp = impedance(solimp, rr[R_POS]);
    double reg = fmax((1.0 - imp) / imp * rr[R_DIAG], 1e-15);
    rr[R_AREF] = -b * vel - kk * imp * rr[R_POS];
    rr[R_D] = 1.0 / reg;
  }
  T.sync();
  return nr;
}

// ---------------------------------------------------------------- dense Newton
struct NewtonBufs {
  double *a0, *grad, *p, *tmp, *tmp2, *mp, *hess, *rinv;
};

__device__ inline bool row_active(const double* rr, double v) { return rr[R_FLAGS] != 0.0 || v < 0.0; }

// y = M x (newton.rs:75-81; the damping term there is zero)
template <int G>
__device__ inline void mul_m(const Tile<G>& T, const double* M, int k, const double* x, double* y) {
  for (int i = T.lane(); i < k; i += G) y[i] = dot_ref(M + i * k, 1, x, 1, k);
  T.sync();
}

// newton.rs:96-110: total cost at aa (fills R_JAR)
template <int G>
__device__ double cost(const Tile<G>& T, int k, int nr, const double* J, double* R, const double* M, const double* aa,
                       const double* a0, double* tmp, double* tmp2) {
  int lane = T.lane();
  for (int i = lane; i < k; i += G) tmp[i] = aa[i] - a0[i];
  T.sync();
  mul_m(T, M, k, tmp, tmp2);
  double s = 0.0;
  for (int i = lane; i < k; i += G) s += tmp[i] * tmp2[i];
  double c = 0.5 * T.sum(s);
  double cr = 0.0;
  for (int r = lane; r < nr; r += G) {
    double* rr = R + R_STRIDE * r;
    double jar = dot_ref(J + r * k, 1, aa, 1, k) - rr[R_AREF];
    rr[R_JAR] = jar;
    if (row_active(rr, jar)) cr += 0.5 * rr[R_D] * jar * jar;
  }
  T.sync();
  return c + T.sum(cr);
}

// Row field the learned start reuses once build_rows has formed aref and D
// from it: the row's predicted activity (-1: none; set by newton_solve).
constexpr int R_PRED = R_DIAG;

// The learned candidate on the tile path, as newton_small forms it: the
// minimiser of the cost with the rows' R_PRED activity held fixed (rows
// without a prediction take their activity at a0), out = a0 - H^-1 g(a0)
// with H = M + J_P' D J_P and g = J_P' D (J a0 - aref) over that set P.
// Uses the Hessian slot, p and grad (free until Newton starts; out must be
// none of them); leaves the set P in R_ACT. False if H is not positive
// definite.
template <int G>
__device__ bool learned_candidate(const Tile<G>& T, int k, int nr, const double* J, double* R, const double* M,
                                  const double* a0, const NewtonBufs& B, double* out) {
  int lane = T.lane();
  double *grad = B.grad, *p = B.p, *H = B.hess;
  for (int r = lane; r < nr; r += G) {
    double* rr = R + R_STRIDE * r;
    double jar = dot_ref(J + r * k, 1, a0, 1, k) - rr[R_AREF];
    rr[R_JAR] = jar;
    rr[R_ACT] = rr[R_PRED] >= 0.0 ? rr[R_PRED] : (row_active(rr, jar) ? 1.0 : 0.0);
  }
  T.sync();
  for (int i = lane; i < k; i += G) {
    double g = 0.0;
    for (int r = 0; r < nr; r++) {
      const double* rr = R + R_STRIDE * r;
      if (rr[R_ACT] != 0.0) g += (rr[R_D] * rr[R_JAR]) * J[r * k + i];
    }
    grad[i] = g;
  }
  for (int t = lane; t < k * (k + 1) / 2; t += G) {
    int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((i + 1) * (i + 2) / 2 <= t) i++;
    while (i * (i + 1) / 2 > t) i--;
    int j = t - i * (i + 1) / 2;
    double h = M[i * k + j];
    for (int r = 0; r < nr; r++) {
      const double* rr = R + R_STRIDE * r;
      if (rr[R_ACT] == 0.0) continue;
      double ji = J[r * k + i];
      if (ji == 0.0) continue;
      h += (rr[R_D] * ji) * J[r * k + j];
    }
    H[i * k + j] = h;
  }
  T.sync();
  bool ok = chol_auto(T, H, k, k, 1, nullptr, nullptr, k, B.rinv);
  if (ok) {
    for (int i = lane; i < k; i += G) p[i] = -grad[i];
    T.sync();
    solve_auto(T, H, k, k, 1, nullptr, nullptr, k, B.rinv, p);
    for (int i = lane; i < k; i += G) out[i] = a0[i] + p[i];
  }
  T.sync();
  return ok;
}

// newton.rs:224-358: `a` holds the unconstrained acceleration on entry and
// the constrained one on exit. Returns the iteration count. With `cand`,
// the learned candidate (learned_candidate) is the start the cost gate
// judges against a0.
template <int G>
__device__ __noinline__ int newton_dense(const Tile<G>& T, int k, int nr, const double* J, double* R, const double* M,
                                         double* a,
                            const double* warm, int max_iters, double tol, const NewtonBufs& B, bool cand = false) {
  int lane = T.lane();
  double *a0 = B.a0, *grad = B.grad, *p = B.p, *tmp = B.tmp, *tmp2 = B.tmp2, *mp = B.mp, *H = B.hess;
  for (int i = lane; i < k; i += G) a0[i] = a[i];
  T.sync();
  // (mp is free until the line search, and the gate's cost() leaves it alone)
  if (cand && learned_candidate(T, k, nr, J, R, M, a0, B, B.mp)) warm = B.mp;
  // when the gate keeps the start, its cost evaluation leaves the first
  // iteration's products there: M (a - a0) in tmp2, J a - aref in R_JAR
  bool have = false;
  if (warm) {
    // the quadratic term of the cost is exactly zero at a0
    double cr0 = 0.0;
    for (int r = lane; r < nr; r += G) {
      const double* rr = R + R_STRIDE * r;
      double jar = dot_ref(J + r * k, 1, a0, 1, k) - rr[R_AREF];
      if (row_active(rr, jar)) cr0 += 0.5 * rr[R_D] * jar * jar;
    }
    double c0 = T.sum(cr0);
    double c1 = cost(T, k, nr, J, R, M, warm, a0, tmp, tmp2);
    if (c1 < c0) {
      for (int i = lane; i < k; i += G) {
        a[i] = warm[i];
        grad[i] = tmp2[i];
      }
      have = true;
    }
    T.sync();
  }
  // no previous iteration's active set (the candidate's stays out of it:
  // iterations count as the reference counts them, from the kept start)
  if (cand)
    for (int r = lane; r < nr; r += G) R[R_STRIDE * r + R_ACT] = -1.0;
  T.sync();
  mul_m(T, M, k, a0, tmp);
  double ss = 0.0;
  for (int i = lane; i < k; i += G) ss += tmp[i] * tmp[i];
  double scale = 1.0 + sqrt(T.sum(ss));
  int iters = 0;
  int maxit = max_iters > 1 ? max_iters : 1;
  while (iters < maxit) {
    iters++;
    for (int i = lane; i < k; i += G) tmp[i] = a[i] - a0[i];
    T.sync();
    if (!have) mul_m(T, M, k, tmp, grad);
    // residuals, active set; R_ACT keeps the previous iteration's set
    bool same = true;
    for (int r = lane; r < nr; r += G) {
      double* rr = R + R_STRIDE * r;
      double jar = have ? rr[R_JAR] : dot_ref(J + r * k, 1, a, 1, k) - rr[R_AREF];
      rr[R_JAR] = jar;
      double act = row_active(rr, jar) ? 1.0 : 0.0;
      if (act != rr[R_ACT]) same = false;
      rr[R_ACT] = act;
    }
    T.sync();
    have = false;
    for (int i = lane; i < k; i += G) {
      double g = grad[i];
      for (int r = 0; r < nr; r++) {
        const double* rr = R + R_STRIDE * r;
        if (rr[R_ACT] != 0.0) g += (rr[R_D] * rr[R_JAR]) * J[r * k + i];
      }
      grad[i] = g;
    }
    T.sync();
    double gs = 0.0;
    for (int i = lane; i < k; i += G) gs += grad[i] * grad[i];
    double gnorm = sqrt(T.sum(gs));
    bool unchanged = T.all(same);
    if (gnorm < tol * scale || (nr <= 128 && unchanged && iters > 1)) break;
    // H = M + J_A' D J_A (lower triangle)
    for (int t = lane; t < k * (k + 1) / 2; t += G) {
      int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
      while ((i + 1) * (i + 2) / 2 <= t) i++;
      while (i * (i + 1) / 2 > t) i--;
      int j = t - i * (i + 1) / 2;
      double h = M[i * k + j];
      for (int r = 0; r < nr; r++) {
        const double* rr = R + R_STRIDE * r;
        if (rr[R_ACT] == 0.0) continue;
        double ji = J[r * k + i];
        if (ji == 0.0) continue;
        h += (rr[R_D] * ji) * J[r * k + j];
      }
      H[i * k + j] = h;
    }
    T.sync();
    if (!chol_auto(T, H, k, k, 1, nullptr, nullptr, k, B.rinv)) break;
    for (int i = lane; i < k; i += G) p[i] = -grad[i];
    T.sync();
    solve_auto(T, H, k, k, 1, nullptr, nullptr, k, B.rinv, p);
    // exact line search on the piecewise quadratic along p
    mul_m(T, M, k, p, mp);
    double s1 = 0.0, s2 = 0.0;
    for (int i = lane; i < k; i += G) {
      s1 += p[i] * mp[i];
      s2 += tmp[i] * mp[i];
    }
    double mpp = T.sum(s1), mpg = T.sum(s2);
    for (int r = lane; r < nr; r += G) {
      double* rr = R + R_STRIDE * r;
      rr[R_JP] = dot_ref(J + r * k, 1, p, 1, k);
    }
    T.sync();
    auto deriv = [&](double al, double* d1o, double* d2o) {
      double d1 = 0.0, d2 = 0.0;
      for (int r = lane; r < nr; r += G) {
        const double* rr = R + R_STRIDE * r;
        double v = rr[R_JAR] + al * rr[R_JP];
        if (row_active(rr, v)) {
          double dq = rr[R_D] * rr[R_JP];
          d1 += dq * v;
          d2 += dq * rr[R_JP];
        }
      }
      *d1o = (al * mpp + mpg) + T.sum(d1);
      *d2o = mpp + T.sum(d2);
    };
    double lo = 0.0, hi = INFINITY, al = 1.0;
    double d10, d20;
    deriv(0.0, &d10, &d20);
    double ltol = 1e-12 * fmax(fabs(d10), 1e-30);
    for (int it = 0; it < 50; it++) {
      double d1, d2;
      deriv(al, &d1, &d2);
      if (fabs(d1) <= ltol) break;
      if (d1 < 0.0) lo = al;
      else hi = al;
      double next = al - d1 / fmax(d2, 1e-30);
      if (next <= lo || next >= hi) next = isfinite(hi) ? 0.5 * (lo + hi) : 2.0 * fmax(al, lo);
      if (fabs(next - al) <= 1e-14 * fmax(fabs(al), 1.0)) {
        al = next;
        break;
      }
      al = next;
    }
    for (int i = lane; i < k; i += G) a[i] += al * p[i];
    T.sync();
  }
  return iters;
}

// newton.rs:361-371: qfrc[idx[i]] += -J' D (J a - aref) over active rows
template <int G>
__device__ __noinline__ void add_constraint_force(const Tile<G>& T, int k, int nr, const double* J, double* R, const double* a,
                                     const int* idx, double* qfrc) {
  int lane = T.lane();
  for (int r = lane; r < nr; r += G) {
    double* rr = R + R_STRIDE * r;
    double v = dot_ref(J + r * k, 1, a, 1, k) - rr[R_AREF];
    rr[R_JAR] = row_active(rr, v) ? -rr[R_D] * v : 0.0;
    rr[R_ACT] = row_active(rr, v) ? 1.0 : 0.0;
  }
  T.sync();
  for (int i = lane; i < k; i += G) {
    int o = idx ? idx[i] : i;
    double q = qfrc[o];
    for (int r = 0; r < nr; r++) {
      const double* rr = R + R_STRIDE * r;
      if (rr[R_ACT] != 0.0) q += rr[R_JAR] * J[r * k + i];
    }
    qfrc[o] = q;
  }
  T.sync();
}

// ------------------------------------------------------- register-resident Newton
// Shared buffers of newton_small (offsets sj, sl, sx, sc of the workspace).
struct SmallBufs {
  double* J;  // [16][k] the first 16 constraint rows, copied in
  double* L;  // [k(k-1)/2] the Hessian factor's entries below the diagonal, packed by rows
  double* x;  // [16] the vector being multiplied
  double* c;  // [32] per-row coefficients
};

constexpr int SMALL_ROWS = 2 * SMALL_N;  // rows the register Newton takes (two per lane)

// newton.rs:224-371 for k <= 16 unknowns and nr <= 32 rows: lane i holds
// unknown i and rows i and i + 16. M stays in shared memory, the lane's row
// of the Hessian (and of its factor) in registers, the factor also packed
// in B.L; the first 16 rows of J are copied into shared memory
// (rows 16..31, rare, are read where build_rows left them); each product
// M x / J x reads the published x with broadcast loads. On 16-lane tiles
// every per-lane partial sum holds the same terms in the same order as
// newton_dense's, so the sums agree with it exactly; only the factorisation
// differs (chol_regx). Adds the constraint force to qfrc (newton.rs:361-371)
// and leaves the solution in a; returns the iteration count. J rows are
// read from Jsrc (stride k), row constants from R.
//
// Learned warm start (lforce != nullptr, lnum touching contacts whose
// pyramid rows are the first 4 lnum rows): the predicted frame forces
// (f_n, f_t1, f_t2) become row forces f_n / 4 +- f_tk / (2 mu) (so that
// sum_r f_r J_r = f_n J_n + f_t1 J_t1 + f_t2 J_t2), and a row is predicted
// active when its force is positive; every other row takes its activity at
// a0. The candidate start is the minimiser of the cost with that active set
// held fixed, a0 - H^-1 g(a0), and it goes behind the same cost gate as the
// previous-step start (newton.rs:238-245). When the prediction is the
// solution's active set, the gradient there is zero to rounding and the
// first iteration ends the solve. With ldump, the converged forces of those
// rows are written there (4 per contact) as training targets.
template <int G>
__device__ inline int newton_small(const Tile<G>& T, int k, int nr, const double* Jsrc, const double* R,
                                         const double* M, double* a, const double* warm, int max_iters, double tol,
                                         const SmallBufs& B, double* qfrc, const float* lfeat, const float* lforce,
                                         int lnum, float* ldump) {
  static_assert(G >= SMALL_N, "one lane per unknown");
  const int i = T.lane();
  const bool dof = i < k;
  const double* mrow = M + i * k;  // this lane's row of M (shared memory, dof lanes only)
  const double a0 = dof ? a[i] : 0.0;
  const double wi = (warm && dof) ? warm[i] : 0.0;
  // rows i and i + 16 of this lane
  bool has[2];
  double aref[2], dr[2];
  bool bil[2];
#pragma unroll
  for (int s = 0; s < 2; s++) {
    int r = i + SMALL_N * s;
    has[s] = i < SMALL_N && r < nr;
    aref[s] = dr[s] = 0.0;
    bil[s] = false;
    if (has[s]) {
      const double* rr = R + R_STRIDE * r;
      aref[s] = rr[R_AREF];
      dr[s] = rr[R_D];
      bil[s] = rr[R_FLAGS] != 0.0;
    }
  }
  int ncopy = (nr < SMALL_N ? nr : SMALL_N) * k;
  for (int t = i; t < ncopy; t += G) B.J[t] = Jsrc[t];
  auto jrow = [&](int r) -> const double* { return r < SMALL_N ? B.J + r * k : Jsrc + r * k; };
  // publish one component per lane for the broadcast reads that follow
  auto publish = [&](double v) {
    T.sync();
    if (dof) B.x[i] = v;
    T.sync();
  };
  // per-row values v[s] of this lane's rows, readable as B.c[r]
  auto coeffs = [&](const double* v) {
    T.sync();
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (has[s]) B.c[i + SMALL_N * s] = v[s];
    T.sync();
  };
  auto jdot = [&](int s) { return dot_ref_sm(jrow(i + SMALL_N * s), B.x, k); };

  double ai = a0;
  double wl = wi;
  bool use_warm = warm != nullptr;
  if (lforce && lnum > 0 && 4 * lnum <= nr) {
    // residuals at a0, and each of this lane's rows' predicted activity
    publish(a0);
    double jr0[2], on[2];
#pragma unroll
    for (int s = 0; s < 2; s++) {
      int r = i + SMALL_N * s;
      jr0[s] = has[s] ? jdot(s) - aref[s] : 0.0;
      on[s] = (bil[s] || jr0[s] < 0.0) ? 1.0 : 0.0;
      if (has[s] && r < 4 * lnum) {
        int c = r / 4, q = r % 4;
        double mu = lfeat[c * LEARN_NF + 1];
        double fn = lforce[3 * c], ft = lforce[3 * c + 1 + q / 2];
        double f = 0.25 * fn + (mu > 0.0 ? ((q & 1) ? -ft : ft) / (2.0 * mu) : 0.0);
        on[s] = f > 0.0 ? 1.0 : 0.0;
      }
    }
    // H = M + J_P' D J_P over the predicted set P, and g(a0) = J_P' D jar0
    double cv0[2];
#pragma unroll
    for (int s = 0; s < 2; s++) cv0[s] = on[s] != 0.0 ? dr[s] : 0.0;
    coeffs(cv0);
    double hl[SMALL_N];
#pragma unroll
    for (int q = 0; q < SMALL_N; q++) hl[q] = (dof && q <= i) ? mrow[q] : 0.0;
    if (dof)
      for (int r = 0; r < nr; r++) {
        double d = B.c[r];
        if (d == 0.0) continue;
        const double* jr = jrow(r);
        double ji = jr[i];
        if (ji == 0.0) continue;
        double e = d * ji;
#pragma unroll
        for (int q = 0; q < SMALL_N; q++)
          if (q <= i && q < k) hl[q] += e * jr[q];
      }
#pragma unroll
    for (int s = 0; s < 2; s++) cv0[s] = on[s] != 0.0 ? dr[s] * jr0[s] : 0.0;
    coeffs(cv0);
    double g0 = 0.0;
    if (dof)
      for (int r = 0; r < nr; r++) {
        double cf = B.c[r];
        if (cf != 0.0) g0 += cf * jrow(r)[i];
      }
    double rv = 0.0;
    if (chol_regx(T, hl, k, B.L, &rv)) {
      wl = a0 + solve_regx(T, hl, k, B.L, rv, dof ? -g0 : 0.0);
      use_warm = true;
    }
  }
  // x = a0 once: M a0 for the scale, and J a0 for the cold cost, whose
  // quadratic term is exactly zero (a - a0 = 0)
  publish(a0);
  double ma0 = dof ? dot_ref_sm(mrow, B.x, k) : 0.0;
  double gw = 0.0, jw[2] = {0.0, 0.0};
  bool have = false;
  if (use_warm) {
    double cr = 0.0;
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (has[s]) {
        double jar = jdot(s) - aref[s];
        if (bil[s] || jar < 0.0) cr += 0.5 * dr[s] * jar * jar;
      }
    double c0 = T.sum(cr);
    // the cost at wl (newton.rs:96-110), keeping its products M (wl - a0)
    // and J wl - aref: the first iteration's when the gate keeps wl
    double tw = wl - a0;
    publish(tw);
    double mw = dof ? dot_ref_sm(mrow, B.x, k) : 0.0;
    double c = 0.5 * T.sum(dof ? tw * mw : 0.0);
    publish(wl);
    double cr1 = 0.0;
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (has[s]) {
        jw[s] = jdot(s) - aref[s];
        if (bil[s] || jw[s] < 0.0) cr1 += 0.5 * dr[s] * jw[s] * jw[s];
      }
    double c1 = c + T.sum(cr1);
    if (c1 < c0) {
      ai = wl;
      gw = mw;
      have = true;
    }
  }
  double scale = 1.0 + sqrt(T.sum(ma0 * ma0));
  // iterations count as the reference counts them, from the start the gate
  // kept (forming the learned candidate costs one factorisation before them)
  int iters = 0;
  int maxit = max_iters > 1 ? max_iters : 1;
  double prev[2] = {-1.0, -1.0};  // the rows' activity in the previous iteration (none yet)
  double jar[2] = {0.0, 0.0}, act[2] = {0.0, 0.0}, cv[2];
  bool fresh = false;  // left at the convergence check: B.c holds D_r jar_r of the final a
  while (iters < maxit) {
    iters++;
    // gradient M (a - a0) + sum over active rows of D jar J_r (newton.rs:254-270)
    double tmp = ai - a0;
    double grad;
    if (have) {  // the gate's products at the start it kept
      grad = gw;
      jar[0] = jw[0];
      jar[1] = jw[1];
      have = false;
    } else {
      publish(tmp);
      grad = dof ? dot_ref_sm(mrow, B.x, k) : 0.0;
      publish(ai);
#pragma unroll
      for (int s = 0; s < 2; s++)
        if (has[s]) jar[s] = jdot(s) - aref[s];
    }
    bool same = true;
#pragma unroll
    for (int s = 0; s < 2; s++)
      if (has[s]) {
        act[s] = (bil[s] || jar[s] < 0.0) ? 1.0 : 0.0;
        if (act[s] != prev[s]) same = false;
        prev[s] = act[s];
      }
#pragma unroll
    for (int s = 0; s < 2; s++) cv[s] = act[s] != 0.0 ? dr[s] * jar[s] : 0.0;
    coeffs(cv);
    if (dof)
      for (int r = 0; r < nr; r++) {
        double cf = B.c[r];
        if (cf != 0.0) grad += cf * jrow(r)[i];
      }
    double gnorm = sqrt(T.sum(dof ? grad * grad : 0.0));
    bool unchanged = T.all(same);
    if (gnorm < tol * scale || (nr <= 128 && unchanged && iters > 1)) {
      fresh = true;
      break;
    }
    // H = M + J_A' D J_A, this lane's row (lower part)
    double h[SMALL_N];
#pragma unroll
    for (int q = 0; q < SMALL_N; q++) h[q] = (dof && q <= i) ? mrow[q] : 0.0;
#pragma unroll
    for (int s = 0; s < 2; s++) cv[s] = act[s] != 0.0 ? dr[s] : 0.0;
    coeffs(cv);
    if (dof)
      for (int r = 0; r < nr; r++) {
        double d = B.c[r];
        if (d == 0.0) continue;
        const double* jr = jrow(r);
        double ji = jr[i];
        if (ji == 0.0) continue;
        double e = d * ji;
#pragma unroll
        for (int q = 0; q < SMALL_N; q++)
          if (q <= i && q < k) h[q] += e * jr[q];
      }
    double rv = 0.0;
    if (!chol_regx(T, h, k, B.L, &rv)) break;
    double p = solve_regx(T, h, k, B.L, rv, dof ? -grad : 0.0);
    // exact line search on the piecewise quadratic along p (newton.rs:317-354)
    publish(p);
    double mp = dof ? dot_ref_sm(mrow, B.x, k) : 0.0;
    double jp[2];
#pragma unroll
    for (int s = 0; s < 2; s++) jp[s] = has[s] ? jdot(s) : 0.0;
    double mpp = T.sum(dof ? p * mp : 0.0), mpg = T.sum(dof ? tmp * mp : 0.0);
    auto deriv = [&](double al, double* d1o, double* d2o) {
      double d1 = 0.0, d2 = 0.0;
#pragma unroll
      for (int s = 0; s < 2; s++)
        if (has[s]) {
          double v = jar[s] + al * jp[s];
          if (bil[s] || v < 0.0) {
            double dq = dr[s] * jp[s];
            d1 += dq * v;
            d2 += dq * jp[s];
          }
        }
      *d1o = (al * mpp + mpg) + T.sum(d1);
      *d2o = mpp + T.sum(d2);
    };
    double lo = 0.0, hi = INFINITY, al = 1.0;
    double d10, d20;
    deriv(0.0, &d10, &d20);
    double ltol = 1e-12 * fmax(fabs(d10), 1e-30);
    for (int it = 0; it < 50; it++) {
      double d1, d2;
      deriv(al, &d1, &d2);
      if (fabs(d1) <= ltol) break;
      if (d1 < 0.0) lo = al;
      else hi = al;
      double next = al - d1 / fmax(d2, 1e-30);
      if (next <= lo || next >= hi) next = isfinite(hi) ? 0.5 * (lo + hi) : 2.0 * fmax(al, lo);
      if (fabs(next - al) <= 1e-14 * fmax(fabs(al), 1.0)) {
        al = next;
        break;
      }
      al = next;
    }
    ai += al * p;
  }
  // qfrc_constraint += -D (J a - aref) J' over active rows (newton.rs:361-371).
  // After the convergence check the last gradient's coefficients D_r jar_r
  // are those of the final a (same a, same active rows): their negatives,
  // bit for bit; otherwise (iteration cap, failed factorisation) they are
  // formed again.
  double sgn = 1.0;
  if (fresh) {
    sgn = -1.0;
  } else {
    publish(ai);
#pragma unroll
    for (int s = 0; s < 2; s++) {
      cv[s] = 0.0;
      if (has[s]) {
        double v = jdot(s) - aref[s];
        cv[s] = (bil[s] || v < 0.0) ? -dr[s] * v : 0.0;
      }
    }
    coeffs(cv);
  }
  if (dof) {
    double q = qfrc[i];
    for (int r = 0; r < nr; r++) {
      double cf = B.c[r];
      if (cf != 0.0) q += (sgn * cf) * jrow(r)[i];
    }
    qfrc[i] = q;
    a[i] = ai;
  }
  if (ldump && lnum > 0 && 4 * lnum <= nr)
    for (int t = i; t < 4 * lnum; t += G) {
      double cf = B.c[t];
      ldump[t] = cf != 0.0 ? (float)(sgn * cf) : 0.0f;
    }
  T.sync();
  return iters;
}

// newton.rs:391-473 for models with several dof blocks: islands are the
// blocks joined by rows touching more than one; each is solved as its own
// dense subproblem (in place when one island spans every block).
template <int G>
__device__ __noinline__ int newton_islands(const Tile<G>& T, const DModel& m, const WsLayout& w, const ScrLayout& s,
                                           const EnvCtx& e, int nr, double* a, const double* warm,
                                           const NewtonBufs& B, bool cand) {
  int lane = T.lane(), nv = m.nv;
  double* ws = e.ws;
  double* qfrc = ws + w.qfrc_c;
  double* J = e.scr + s.jac;
  double* R = e.scr + s.rows;
  int max_iters = m.iterations;
  double tol = m.tolerance;
  // rows -> touched blocks (bit mask), then union-find on lane 0
  int* iscr = (int*)(e.scr + s.isl_of_row);       // [maxrows] island of each row (-1 none)
  int* blk_isl = (int*)(e.scr + s.isl_dof);       // [nblock] island id (min block of component)
  unsigned long long* rmask = (unsigned long long*)(e.scr + s.isl_row);  // [maxrows]
  for (int r = lane; r < nr; r += G) {
    unsigned long long mk = 0;
    for (int k = 0; k < nv; k++)
      if (J[r * nv + k] != 0.0) mk |= 1ull << m.dof_block[k];
    rmask[r] = mk;
  }
  T.sync();
  if (lane == 0) {
    int par[64];
    for (int b = 0; b < m.nblock; b++) par[b] = b;
    auto find = [&](int x) {
      while (par[x] != x) {
        par[x] = par[par[x]];
        x = par[x];
      }
      return x;
    };
    for (int r = 0; r < nr; r++) {
      unsigned long long mk = rmask[r];
      if (!mk) continue;
      int first = __ffsll((long long)mk) - 1;
      mk &= mk - 1;
      while (mk) {
        int b = __ffsll((long long)mk) - 1;
        mk &= mk - 1;
        int x = find(first), y = find(b);
        if (x != y) par[x > y ? x : y] = x < y ? x : y;
      }
    }
    for (int b = 0; b < m.nblock; b++) blk_isl[b] = find(b);
    for (int r = 0; r < nr; r++) iscr[r] = rmask[r] ? blk_isl[__ffsll((long long)rmask[r]) - 1] : -1;
  }
  T.sync();
  // islands in increasing id order; single island spanning all blocks -> in place
  int n_isl = 0, only = -1;
  bool all_one = true;
  for (int isl = 0; isl < m.nblock; isl++) {
    bool has = false;
    for (int r = lane; r < nr; r += G) has |= iscr[r] == isl;
    if (T.any(has)) {
      n_isl++;
      only = isl;
    }
  }
  for (int b = 0; b < m.nblock; b++) all_one &= blk_isl[b] == only;
  if (n_isl == 1 && all_one) {
    int it = newton_dense(T, nv, nr, J, R, e.qm, a, warm, max_iters, tol, B, cand);
    add_constraint_force(T, nv, nr, J, R, a, (const int*)nullptr, qfrc);
    return it;
  }
  int iters = 0;
  double* subM = e.scr + s.sub_m;
  double* subJ = e.scr + s.sub_j;
  double* subR = e.scr + s.sub_rows;
  int* idx = (int*)(e.scr + s.isl_row) + 2 * m.maxrows;  // after rmask words
  double* suba = ws + w.vel;   // free until the solve returns
  double* wsub = ws + w.warm;  // gathered warm start
  for (int isl = 0; isl < m.nblock; isl++) {
    bool has = false;
    for (int r = lane; r < nr; r += G) has |= iscr[r] == isl;
    if (!T.any(has)) continue;
    // dofs of the island's blocks, in block order
    int kk = 0;
    for (int b = 0; b < m.nblock; b++) {
      if (blk_isl[b] != isl) continue;
      int s0 = m.block_adr[2 * b], s1 = m.block_adr[2 * b + 1];
      for (int i = s0 + lane; i < s1; i += G) idx[kk + (i - s0)] = i;
      kk += s1 - s0;
    }
    // rows of the island, in row order
    int nri = 0;
    bool pred = false;  // a row of the island has a learned prediction
    for (int base = 0; base < nr; base += G) {
      int r = base + lane;
      bool in = r < nr && iscr[r] == isl;
      int tot;
      int off = T.excl_scan(in ? 1 : 0, &tot);
      if (in) idx[nv + nri + off] = r;
      if (in && cand) pred |= R[R_STRIDE * r + R_PRED] >= 0.0;
      nri += tot;
    }
    pred = T.any(pred);
    T.sync();
    for (int t = lane; t < kk * kk; t += G) subM[t] = e.qm[idx[t / kk] * nv + idx[t % kk]];
    for (int t = lane; t < nri * kk; t += G) subJ[t] = J[idx[nv + t / kk] * nv + idx[t % kk]];
    for (int t = lane; t < nri * R_STRIDE; t += G) subR[t] = R[R_STRIDE * idx[nv + t / R_STRIDE] + t % R_STRIDE];
    for (int i = lane; i < kk; i += G) {
      suba[i] = a[idx[i]];
      wsub[i] = warm ? warm[idx[i]] : 0.0;
    }
    T.sync();
    int it = newton_dense(T, kk, nri, subJ, subR, subM, suba, warm ? wsub : nullptr, max_iters, tol, B, pred);
    iters = it > iters ? it : iters;
    for (int i = lane; i < kk; i += G) a[idx[i]] = suba[i];
    T.sync();
    add_constraint_force(T, kk, nri, subJ, subR, suba, idx, qfrc);
  }
  return iters;
}

// The converged forces -D_r (J_r a - aref_r) of rows [0, nrows) (zero where
// the row is inactive) as training targets of the learned warm start
// (newton.rs:361-371).
template <int G>
__device__ void dump_row_forces(const Tile<G>& T, int nv, const double* J, const double* R, const double* a,
                                int nrows, float* ldump) {
  for (int r = T.lane(); r < nrows; r += G) {
    const double* rr = R + R_STRIDE * r;
    double v = dot_ref_sm(J + r * nv, a, nv) - rr[R_AREF];
    ldump[r] = (rr[R_FLAGS] != 0.0 || v < 0.0) ? (float)(-rr[R_D] * v) : 0.0f;
  }
  T.sync();
}

// newton.rs:378-473. LEARN = false compiles the learned start's inputs out
// (a kernel for the other warm-start modes carries none of its code).
template <int G, bool LEARN = true>
__device__ int newton_solve(const Tile<G>& T, const DModel& m, const WsLayout& w, const ScrLayout& s,
                            const EnvCtx& e, int nr, double* a, const double* warm, const float* lfeat = nullptr,
                            const float* lforce = nullptr, int lnum = 0, float* ldump = nullptr) {
  if constexpr (!LEARN) {
    lfeat = nullptr;
    lforce = nullptr;
    lnum = 0;
    ldump = nullptr;
  }
  int lane = T.lane(), nv = m.nv;
  double* ws = e.ws;
  double* qfrc = ws + w.qfrc_c;
  for (int i = lane; i < nv; i += G) qfrc[i] = 0.0;
  T.sync();
  if (nr == 0) return 0;
  double* J = e.scr + s.jac;
  double* R = e.scr + s.rows;
  bool learned = lnum > 0 && 4 * lnum <= nr;
  bool cand = learned && lforce;
  for (int r = lane; r < nr; r += G) {
    double* rr = R + R_STRIDE * r;
    rr[R_ACT] = -1.0;  // no previous active set
    // the learned start's predicted activity of the touching contacts'
    // pyramid rows (row force f_n / 4 +- f_tk / (2 mu) > 0), as newton_small
    // forms it; -1 for every other row
    double pred = -1.0;
    if (cand && r < 4 * lnum) {
      int c = r / 4, q = r % 4;
      double mu = lfeat[c * LEARN_NF + 1];
      double fn = lforce[3 * c], ft = lforce[3 * c + 1 + q / 2];
      double f = 0.25 * fn + (mu > 0.0 ? ((q & 1) ? -ft : ft) / (2.0 * mu) : 0.0);
      pred = f > 0.0 ? 1.0 : 0.0;
    }
    rr[R_PRED] = pred;
  }
  T.sync();
  NewtonBufs B{ws + w.a0, ws + w.grad, ws + w.p, ws + w.tmp, ws + w.tmp2, ws + w.mp, e.fac, ws + w.rinv};
  if (m.nblock > 1) {
    int it = newton_islands(T, m, w, s, e, nr, a, warm, B, cand);
    if (learned && ldump) dump_row_forces(T, nv, J, R, a, 4 * lnum, ldump);
    return it;
  }
  // one tree: the rows either touch it (one island spanning everything)
  // or none has a nonzero entry (no island: nothing is solved)
  bool nz = false;
  for (int t = lane; t < nr * nv; t += G) nz |= J[t] != 0.0;
  if (!T.any(nz)) return 0;
  if constexpr (G >= SMALL_N) {
    if (nv <= SMALL_N && nr <= SMALL_ROWS && w.sj >= 0) {
      SmallBufs S{ws + w.sj, ws + w.sl, ws + w.sx, ws + w.sc};
      // (this path keeps M in the workspace: its loads are shared-memory loads)
      return newton_small(T, nv, nr, J, R, ws + w.qm, a, warm, m.iterations, m.tolerance, S, qfrc, lfeat, lforce,
                          lnum, ldump);
    }
  }
  int it = newton_dense(T, nv, nr, J, R, e.qm, a, warm, m.iterations, m.tolerance, B, cand);
  add_constraint_force(T, nv, nr, J, R, a, (const int*)nullptr, qfrc);
  if (learned && ldump) dump_row_forces(T, nv, J, R, a, 4 * lnum, ldump);
  return it;
}

// forward.rs:412-429: the implicitfast actuator terms h kv g_x g_y of the
// dofs on one chain, added to F (rare path, lane 0)
template <int G>
__device__ void add_actuator_kv(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e, double h,
                                double* F) {
  const double* ws = e.ws;
  int nv = m.nv;
  if (m.integrator == 1 && T.lane() == 0) {
    for (int u = 0; u < m.nu; u++) {
      double kv = -e.prm[m.p_bias + 3 * u + 2] * m.act_gear[u] * m.act_gear[u];
      if (kv == 0.0 || ws[w.actclamped + u] != 0.0) continue;
      int a0 = m.act_moment_adr[u], an = m.act_moment_num[u];
      for (int x = 0; x < an; x++)
        for (int y = 0; y < an; y++) {
          int da = m.jnt_dofadr[m.moment_jnt[a0 + x]], db = m.jnt_dofadr[m.moment_jnt[a0 + y]];
          bool rel = da == db;
          for (int q = m.dof_parent[db]; q != -1 && !rel; q = m.dof_parent[q]) rel = q == da;
          for (int q = m.dof_parent[da]; q != -1 && !rel; q = m.dof_parent[q]) rel = q == db;
          if (rel) F[da * nv + db] += h * kv * m.moment_coef[a0 + x] * m.moment_coef[a0 + y];
        }
    }
  }
}

// forward.rs:407-431,392-401: factor M + h D per dof block into ws fac;
// M (nv x nv) is read from global memory
template <int G>
__device__ bool factor_mass(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e, double h,
                            const double* qm) {
  int lane = T.lane(), nv = m.nv;
  double* ws = e.ws;
  double* F = ws + w.fac;
  load_async(T, F, qm, nv * nv);
  load_wait();
  T.sync();
  if (h != 0.0) {
    for (int k = lane; k < nv; k += G) F[k * nv + k] += h * e.prm[m.p_damping + k];
    T.sync();
  }
  add_actuator_kv(T, m, w, e, h, F);
  T.sync();
  return chol_auto(T, F, nv, nv, m.nblock, m.block_adr, m.dof_block, m.maxbs, ws + w.rinv);
}

// The smooth phase's two factors from one load of M: M itself into ws fac
// (for a0 = M^-1 f) and M + h D into ws fac2 (forward.rs:356-366, for the
// damped solve after Newton, or PGS), factored side by side on the
// small-matrix path so that their column chains overlap. False if either is
// not positive definite.
template <int G>
__device__ bool factor_mass2(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e, double h,
                             const double* qm) {
  int lane = T.lane(), nv = m.nv;
  double* ws = e.ws;
  double *F = ws + w.fac, *F2 = ws + w.fac2;
  load_async(T, F, qm, nv * nv);
  load_async(T, F2, qm, nv * nv);
  load_wait();
  T.sync();
  for (int k = lane; k < nv; k += G) F2[k * nv + k] += h * e.prm[m.p_damping + k];
  T.sync();
  add_actuator_kv(T, m, w, e, h, F2);
  T.sync();
  if constexpr (G >= SMALL_N) {
    if (nv <= SMALL_N) return chol_small2(T, F, F2, nv, nv, ws + w.rinv, ws + w.rinv2);
  }
  if (!chol_blocks(T, F, nv, nv, m.nblock, m.block_adr, m.dof_block, m.maxbs, ws + w.rinv)) return false;
  return chol_blocks(T, F2, nv, nv, m.nblock, m.block_adr, m.dof_block, m.maxbs, ws + w.rinv2);
}

// forward.rs:454-456 (the tile checks its share of dofs and actuators at once)
template <int G>
__device__ inline bool has_implicit_terms(const Tile<G>& T, const DModel& m, const double* prm) {
  bool any = false;
  for (int k = T.lane(); k < m.nv; k += G) any |= prm[m.p_damping + k] != 0.0;
  if (m.integrator == 1)
    for (int u = T.lane(); u < m.nu; u += G) any |= prm[m.p_bias + 3 * u + 2] != 0.0;
  return T.any(any);
}

// forward.rs:459-480
template <int G>
__device__ void integrate_pos(const Tile<G>& T, const DModel& m, double* qpos, const double* v, double h) {
  for (int j = T.lane(); j < m.njnt; j += G) {
    int qa = m.jnt_qposadr[j], da = m.jnt_dofadr[j];
    int type = m.jnt_type[j];
    if (type == JNT_FREE) {
      for (int k = 0; k < 3; k++) qpos[qa + k] += h * v[da + k];
      Q4 q = q_integrate_local(ld4(qpos + qa + 3), ld3(v + da + 3), h);
      st4(qpos + qa + 3, q);
    } else if (type == JNT_BALL) {
      Q4 q = q_integrate_local(ld4(qpos + qa), ld3(v + da), h);
      st4(qpos + qa, q);
    } else {
      qpos[qa] += h * v[da];
    }
  }
  T.sync();
}

}  // namespace pg
