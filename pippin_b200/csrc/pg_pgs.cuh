// Projected Gauss-Seidel (crates/pippin/src/solver.rs:38-289) for one env,
// run by the Newton-phase kernel when the model's solver is PGS.
//
// Rows follow the reference's order: [normal, tangent 1, tangent 2] per
// contact (every contact of the narrow phase, not only touching ones), then
// the joint-limit sides within reach, then the joint equalities. The rows of
// M^-1 J' are formed one per lane with the reference's solve (division by the
// pivot, dot-product order of math.rs), so each lane's row matches the CPU
// bit for bit up to FMA contraction. The sweeps are sequential over rows, as
// Gauss-Seidel must be: every lane forms J_r . v itself in the reference's
// summation order (no reduction tree), and the velocity update v += dl M^-1
// J_r' runs one dof per lane. Impulses live in the row records.
#pragma once
#include "pg_newton.cuh"

namespace pg {

constexpr double PGS_MAX_BIAS_VELOCITY = 1.0;  // solver.rs:34
constexpr double PGS_TOLERANCE = 1e-5;         // solver.rs:36
constexpr double PGS_MATCH_DIST2 = 0.01 * 0.01;  // solver.rs:255

// Rows of the PGS problem (solver.rs:63-163) into J (stride nv) and R
// (PR_* records). Returns the row count, capped at maxrows.
template <int G>
__device__ int pgs_rows(const Tile<G>& T, const DModel& m, const WsLayout& w, const EnvCtx& e, int ncon,
                        const double* v, double* J, double* R, int* status) {
  int lane = T.lane(), nv = m.nv;
  const double* ws = e.ws;
  const double* prm = e.prm;
  const double* con = e.con;
  const double* cdof = ws + w.cdof;
  int ncrow = 3 * ncon;
  if (ncrow > m.maxrows) {
    *status |= ST_CAP_EXCEEDED;
    ncrow = m.maxrows / 3 * 3;
  }
  int nc = ncrow / 3;
  // contact rows: records, then one Jacobian item per (contact, dof)
  for (int c = lane; c < nc; c += G) {
    const double* r = con + C_STRIDE * c;
    int g1 = (int)r[C_G1], g2 = (int)r[C_G2];
    double mu = fmax(prm[m.p_friction + g1], prm[m.p_friction + g2]);
    for (int q = 0; q < 3; q++) {
      double* rr = R + PR_STRIDE * (3 * c + q);
      rr[PR_KIND] = q == 0 ? PK_NORMAL : PK_FRICTION;
      rr[PR_SEP] = q == 0 ? -r[C_DEPTH] : 0.0;
      rr[PR_MU] = q == 0 ? 0.0 : mu;
      rr[PR_NORMAL] = 3 * c;
      rr[PR_CONTACT] = c;
      rr[PR_INVA] = 0.0;
      rr[PR_LAMBDA] = 0.0;
    }
  }
  for (int it = lane; it < nc * nv; it += G) {
    int c = it / nv, k = it % nv;
    const double* r = con + C_STRIDE * c;
    int b1 = m.geom_body[(int)r[C_G1]], b2 = m.geom_body[(int)r[C_G2]];
    V3 p = ld3(r + C_POS);
    J[(3 * c + 0) * nv + k] = pair_jac(m, cdof, b1, b2, p, ld3(r + C_NORMAL), k);
    J[(3 * c + 1) * nv + k] = pair_jac(m, cdof, b1, b2, p, ld3(r + C_T1), k);
    J[(3 * c + 2) * nv + k] = pair_jac(m, cdof, b1, b2, p, ld3(r + C_T2), k);
  }
  // joint-limit sides within reach (solver.rs:115-139)
  int nl = 0;
  for (int base = 0; base < m.njnt; base += G) {
    int j = base + lane;
    int cnt = 0, da = 0;
    double sep[2] = {0.0, 0.0};
    bool hit[2] = {false, false};
    if (j < m.njnt && m.jnt_limited[j] && (m.jnt_type[j] == JNT_HINGE || m.jnt_type[j] == JNT_SLIDE)) {
      double q = ws[w.qpos + m.jnt_qposadr[j]];
      da = m.jnt_dofadr[j];
      double reach = m.margin + 2.0 * m.timestep * fabs(v[da]);
      sep[0] = q - m.jnt_range[2 * j];
      sep[1] = m.jnt_range[2 * j + 1] - q;
      for (int t = 0; t < 2; t++) {
        hit[t] = sep[t] < reach;
        cnt += hit[t] ? 1 : 0;
      }
    }
    int tot;
    int off = T.excl_scan(cnt, &tot);
    int row = ncrow + nl + off;
    for (int t = 0; t < 2; t++) {
      if (!hit[t]) continue;
      if (row < m.maxrows) {
        double* jr = J + row * nv;
        for (int k = 0; k < nv; k++) jr[k] = 0.0;
        jr[da] = t == 0 ? 1.0 : -1.0;
        double* rr = R + PR_STRIDE * row;
        rr[PR_KIND] = PK_NORMAL;
        rr[PR_SEP] = sep[t];
        rr[PR_MU] = 0.0;
        rr[PR_NORMAL] = -1.0;
        rr[PR_CONTACT] = -1.0;
        rr[PR_INVA] = 0.0;
        rr[PR_LAMBDA] = 0.0;
      }
      row++;
    }
    nl += tot;
  }
  int nineq = ncrow + nl;
  // joint equalities (solver.rs:141-162)
  for (int q = lane; q < m.neq; q += G) {
    int row = nineq + q;
    if (row >= m.maxrows) continue;
    int j1 = m.eq_j1[q], j2 = m.eq_j2[q];
    const double* c = m.eq_poly + 5 * q;
    double q1 = ws[w.qpos + m.jnt_qposadr[j1]] - m.qpos0[m.jnt_qposadr[j1]];
    double* jr = J + row * nv;
    for (int k = 0; k < nv; k++) jr[k] = 0.0;
    jr[m.jnt_dofadr[j1]] += 1.0;
    double poly = c[0];
    if (j2 != -1) {
      double x = ws[w.qpos + m.jnt_qposadr[j2]] - m.qpos0[m.jnt_qposadr[j2]];
      poly = c[0] + x * (c[1] + x * (c[2] + x * (c[3] + x * c[4])));
      jr[m.jnt_dofadr[j2]] -= c[1] + x * (2.0 * c[2] + x * (3.0 * c[3] + x * 4.0 * c[4]));
    }
    double* rr = R + PR_STRIDE * row;
    rr[PR_KIND] = PK_BILATERAL;
    rr[PR_SEP] = q1 - poly;
    rr[PR_MU] = 0.0;
    rr[PR_NORMAL] = -1.0;
    rr[PR_CONTACT] = -1.0;
    rr[PR_INVA] = 0.0;
    rr[PR_LAMBDA] = 0.0;
  }
  int nr = nineq + m.neq;
  if (nr > m.maxrows) {
    *status |= ST_CAP_EXCEEDED;
    nr = m.maxrows;
  }
  T.sync();
  return nr;
}

// x <- (L L')^-1 x for one right-hand side, by one lane, per dof block, with
// the reference's operations (math.rs:451-463: row-oriented forward sweep
// dividing by the pivot, then column-oriented backward sweep).
__device__ inline void lane_mass_solve(const DModel& m, const double* L, double* x) {
  int nv = m.nv;
  for (int b = 0; b < m.nblock; b++) {
    int s0 = m.block_adr[2 * b], s1 = m.block_adr[2 * b + 1];
    for (int i = s0; i < s1; i++) x[i] = (x[i] - dot_ref(L + i * nv + s0, 1, x + s0, 1, i - s0)) / L[i * nv + i];
    for (int i = s1 - 1; i >= s0; i--) {
      x[i] /= L[i * nv + i];
      double xi = -x[i];
      for (int k = s0; k < i; k++) x[k] += xi * L[i * nv + k];
    }
  }
}

// solver.rs:63-251 and the warm start of :254-289. On entry v holds the
// unconstrained velocity qvel + h (M + hD)^-1 f; on exit v is the final
// velocity and vpos the velocity after the biased sweeps (which positions
// integrate with). L is the factor of M + hD (stride nv). prev / prev_ncon are
// the env's previous-step contacts and impulses, replaced by this step's.
// Returns the number of sweeps; *nrows gets the row count.
template <int G>
__device__ __noinline__ int pgs_solve(const Tile<G>& T, const DModel& m, const WsLayout& w, const ScrLayout& s,
                                      const EnvCtx& e, int ncon, double* v, double* vpos, const double* L,
                                      double* prev, int32_t* prev_ncon, int* nrows, int* status) {
  int lane = T.lane(), nv = m.nv;
  double h = m.timestep;
  double* J = e.scr + s.jac;
  double* R = e.scr + s.rows;
  double* MJ = e.scr + s.mj;
  const double* con = e.con;
  int nr = pgs_rows(T, m, w, e, ncon, v, J, R, status);
  *nrows = nr;
  for (int k = lane; k < nv; k += G) vpos[k] = v[k];
  if (nr == 0) {
    if (lane == 0) *prev_ncon = 0;
    T.sync();
    return 0;
  }
  // M^-1 J_r' and 1 / (J_r M^-1 J_r') per row, one row per lane
  for (int r = lane; r < nr; r += G) {
    double* x = MJ + r * nv;
    const double* jr = J + r * nv;
    for (int k = 0; k < nv; k++) x[k] = jr[k];
    lane_mass_solve(m, L, x);
    double a = 0.0;
    for (int k = 0; k < nv; k++) a += jr[k] * x[k];
    R[PR_STRIDE * r + PR_INVA] = a > 1e-12 ? 1.0 / a : 0.0;
  }
  // warm start: the nearest previous contact of the same geom pair within
  // 1 cm lends its impulses, the tangent ones re-projected on the new frame
  int np = *prev_ncon;
  int nc = min(ncon, nr / 3);
  for (int c = lane; c < nc; c += G) {
    const double* cr = con + C_STRIDE * c;
    double g1 = cr[C_G1], g2 = cr[C_G2];
    V3 pos = ld3(cr + C_POS);
    double bd = PGS_MATCH_DIST2;
    int bi = -1;
    for (int p = 0; p < np; p++) {
      const double* pr = prev + P_STRIDE * p;
      if (pr[P_G1] == g1 && pr[P_G2] == g2) {
        V3 dp = ld3(pr + P_POS) - pos;
        double d2 = dot(dp, dp);
        if (d2 < bd) {
          bd = d2;
          bi = p;
        }
      }
    }
    if (bi != -1) {
      const double* pr = prev + P_STRIDE * bi;
      V3 f = ld3(pr + P_T1) * pr[P_LAMBDA + 1] + ld3(pr + P_T2) * pr[P_LAMBDA + 2];
      R[PR_STRIDE * (3 * c) + PR_LAMBDA] = pr[P_LAMBDA];
      R[PR_STRIDE * (3 * c + 1) + PR_LAMBDA] = dot(f, ld3(cr + C_T1));
      R[PR_STRIDE * (3 * c + 2) + PR_LAMBDA] = dot(f, ld3(cr + C_T2));
    }
  }
  T.sync();
  for (int k = lane; k < nv; k += G) {
    double vk = v[k];
    for (int r = 0; r < nr; r++) {
      double l = R[PR_STRIDE * r + PR_LAMBDA];
      if (l != 0.0) vk += MJ[r * nv + k] * l;
    }
    v[k] = vk;
  }
  T.sync();
  // solver.rs:44-50
  double omega = 2.0 * M_PI * m.hertz;
  double a1 = 2.0 * m.dampratio + h * omega;
  double a2 = h * omega * a1;
  double a3 = 1.0 / (1.0 + a2);
  double bias_rate = omega / a1, mass_scale = a2 * a3, impulse_scale = a3;
  // one Gauss-Seidel sweep; returns the largest velocity change
  auto sweep = [&](bool use_bias) -> double {
    double max_dv = 0.0;
    for (int r = 0; r < nr; r++) {
      double* rr = R + PR_STRIDE * r;
      double inv_a = rr[PR_INVA];
      if (inv_a == 0.0) continue;
      const double* jr = J + r * nv;
      double jv = 0.0;
      for (int k = 0; k < nv; k++) jv += jr[k] * v[k];
      double lam = rr[PR_LAMBDA];
      int kind = (int)rr[PR_KIND];
      double nw;
      if (kind == PK_NORMAL) {
        double sl = rr[PR_SEP] + m.slop;
        double bias, ms, is;
        if (sl > 0.0) {
          bias = sl / h;
          ms = 1.0;
          is = 0.0;
        } else if (use_bias) {
          bias = fmax(bias_rate * sl, -PGS_MAX_BIAS_VELOCITY);
          ms = mass_scale;
          is = impulse_scale;
        } else {
          bias = 0.0;
          ms = 1.0;
          is = 0.0;
        }
        double delta = -inv_a * ms * (jv + bias) - is * lam;
        nw = fmax(lam + delta, 0.0);
      } else if (kind == PK_BILATERAL) {
        double bias, ms, is;
        if (use_bias) {
          bias = fmin(fmax(bias_rate * rr[PR_SEP], -PGS_MAX_BIAS_VELOCITY), PGS_MAX_BIAS_VELOCITY);
          ms = mass_scale;
          is = impulse_scale;
        } else {
          bias = 0.0;
          ms = 1.0;
          is = 0.0;
        }
        nw = lam - inv_a * ms * (jv + bias) - is * lam;
      } else {
        double bound = rr[PR_MU] * R[PR_STRIDE * (int)rr[PR_NORMAL] + PR_LAMBDA];
        nw = fmin(fmax(lam - inv_a * jv, -bound), bound);
      }
      double dl = nw - lam;
      if (dl != 0.0) {
        max_dv = fmax(max_dv, fabs(dl) / inv_a);
        T.sync();  // every lane has read v and the impulses
        const double* mr = MJ + r * nv;
        for (int k = lane; k < nv; k += G) v[k] += mr[k] * dl;
        if (lane == 0) rr[PR_LAMBDA] = nw;
        T.sync();
      }
    }
    return max_dv;
  };
  int sweeps = 0;
  for (int it = 0; it < m.iterations; it++) {
    sweeps++;
    if (sweep(true) < PGS_TOLERANCE) break;
  }
  for (int k = lane; k < nv; k += G) vpos[k] = v[k];
  T.sync();
  int nrelax = max(m.iterations / 3, 2);
  for (int it = 0; it < nrelax; it++) {
    sweeps++;
    if (sweep(false) < PGS_TOLERANCE) break;
  }
  // this step's contacts and impulses for the next warm start
  for (int c = lane; c < nc; c += G) {
    const double* cr = con + C_STRIDE * c;
    double* pr = prev + P_STRIDE * c;
    for (int q = 0; q < 3; q++) {
      pr[P_POS + q] = cr[C_POS + q];
      pr[P_T1 + q] = cr[C_T1 + q];
      pr[P_T2 + q] = cr[C_T2 + q];
      pr[P_LAMBDA + q] = R[PR_STRIDE * (3 * c + q) + PR_LAMBDA];
    }
    pr[P_G1] = cr[C_G1];
    pr[P_G2] = cr[C_G2];
  }
  if (lane == 0) *prev_ncon = nc;
  T.sync();
  return sweeps;
}

}  // namespace pg
