// Oracle (test infrastructure only): narrow-phase collision. Restates
// crates/pippin/src/collision.rs:1-531 (primitive routines, contact frame,
// type-ordered dispatch with normal flip). Rust's Iterator::min_by keeps the
// FIRST of equal minima and max_by the LAST of equal maxima; the helpers
// below reproduce that tie-breaking.
#include <algorithm>

#include "om_model.h"

namespace om {

static Hit mkhit(Vec3 pos, Vec3 n, Real depth) { return Hit{pos, n, depth, v3zero()}; }

// collision.rs:47-55
void contact_frame(const Contact& c, Vec3* t1, Vec3* t2) {
  Vec3 t = c.tangent - c.normal * dot(c.normal, c.tangent);
  if (norm2(t) > 1e-12) {
    *t1 = normalized(t);
    *t2 = cross(c.normal, *t1);
  } else {
    tangents(c.normal, t1, t2);
  }
}

// collision.rs:98-100, 104-107
static bool pair_supported(int a, int b) { return !(a == GEOM_PLANE && b == GEOM_PLANE); }
bool needs_general(int a, int b) {
  return a == GEOM_MESH || b == GEOM_MESH || (a == GEOM_CYLINDER && b != GEOM_PLANE) ||
         (b == GEOM_CYLINDER && a != GEOM_PLANE);
}

// collision.rs:149-152
static void segment(const GeomPose& g, Vec3* p0, Vec3* p1) {
  Vec3 ax = col(g.mat, 2) * g.size[1];
  *p0 = g.pos - ax;
  *p1 = g.pos + ax;
}

// collision.rs:154-162
Vec3 closest_on_segment(Vec3 a, Vec3 b, Vec3 p) {
  Vec3 d = b - a;
  Real l2 = norm2(d);
  if (l2 < 1e-18) return a;
  Real t = clampr(dot(p - a, d) / l2, 0.0, 1.0);
  return a + d * t;
}

// collision.rs:165-201
void closest_segments(Vec3 p0, Vec3 p1, Vec3 q0, Vec3 q1, Vec3* x, Vec3* y) {
  Vec3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
  Real a = norm2(d1), e = norm2(d2), f = dot(d2, r);
  Real s, t;
  if (a < 1e-18 && e < 1e-18) {
    *x = p0;
    *y = q0;
    return;
  }
  if (a < 1e-18) {
    s = 0.0;
    t = clampr(f / e, 0.0, 1.0);
  } else {
    Real c = dot(d1, r);
    if (e < 1e-18) {
      t = 0.0;
      s = clampr(-c / a, 0.0, 1.0);
    } else {
      Real b = dot(d1, d2);
      Real denom = a * e - b * b;
      Real s0 = denom > 1e-18 ? clampr((b * f - c * e) / denom, 0.0, 1.0) : 0.0;
      Real t0 = (b * s0 + f) / e;
      if (t0 < 0.0) {
        t0 = 0.0;
        s0 = clampr(-c / a, 0.0, 1.0);
      } else if (t0 > 1.0) {
        t0 = 1.0;
        s0 = clampr((b - c) / a, 0.0, 1.0);
      }
      s = s0;
      t = t0;
    }
  }
  *x = p0 + d1 * s;
  *y = q0 + d2 * t;
}

// collision.rs:203-212
static void plane_sphere(const GeomPose& plane, Vec3 c, Real r, Real margin, std::vector<Hit>& out) {
  Vec3 n = col(plane.mat, 2);
  Real dist = dot(c - plane.pos, n);
  Real depth = r - dist;
  if (depth > -margin) out.push_back(mkhit(c - (n * (dist + r)) * 0.5, n, depth));
}

void stable_sort_dist(std::vector<DistPt>& v) {
  std::stable_sort(v.begin(), v.end(), [](const DistPt& a, const DistPt& b) { return a.d < b.d; });
}

// collision.rs:214-236
static void plane_box(const GeomPose& plane, const GeomPose& b, Real margin, std::vector<Hit>& out) {
  Vec3 n = col(plane.mat, 2);
  std::vector<DistPt> hits;
  for (int i = 0; i < 8; i++) {
    Vec3 s = v3((i & 1) == 0 ? -1.0 : 1.0, (i & 2) == 0 ? -1.0 : 1.0, (i & 4) == 0 ? -1.0 : 1.0);
    Vec3 corner = b.pos + mul_vec(b.mat, mul_elem(b.size, s));
    Real dist = dot(corner - plane.pos, n);
    if (dist < margin) hits.push_back({dist, corner});
  }
  stable_sort_dist(hits);
  for (size_t k = 0; k < hits.size() && k < 4; k++)
    out.push_back(mkhit(hits[k].p - n * (hits[k].d * 0.5), n, -hits[k].d));
}

// collision.rs:238-267
static void plane_cylinder(const GeomPose& plane, const GeomPose& c, Real margin, std::vector<Hit>& out) {
  Vec3 n = col(plane.mat, 2);
  Vec3 axis = col(c.mat, 2);
  Real r = c.size[0], h = c.size[1];
  Vec3 radial = n - axis * dot(axis, n);
  Real rl = norm(radial);
  std::vector<Vec3> pts;
  for (Real cap : {-1.0, 1.0}) {
    Vec3 cc = c.pos + axis * (h * cap);
    if (rl > 0.05) {
      Vec3 dd = radial * (-1.0 / rl);
      pts.push_back(cc + dd * r);
    } else {
      Vec3 t1, t2;
      tangents(axis, &t1, &t2);
      for (Vec3 v : {t1, -t1, t2, -t2}) pts.push_back(cc + v * r);
    }
  }
  std::vector<DistPt> hits;
  for (Vec3 p : pts) {
    Real d = dot(p - plane.pos, n);
    if (d < margin) hits.push_back({d, p});
  }
  stable_sort_dist(hits);
  for (size_t k = 0; k < hits.size() && k < 4; k++)
    out.push_back(mkhit(hits[k].p - n * (hits[k].d * 0.5), n, -hits[k].d));
}

// collision.rs:269-279
static void sphere_sphere(Vec3 c1, Real r1, Vec3 c2, Real r2, Real margin, std::vector<Hit>& out) {
  Vec3 d = c2 - c1;
  Real dist = norm(d);
  Real depth = r1 + r2 - dist;
  if (depth <= -margin) return;
  Vec3 n = dist > 1e-12 ? d * (1.0 / dist) : v3(0, 0, 1);
  Vec3 pos = c1 + n * (r1 - depth * 0.5);
  out.push_back(mkhit(pos, n, depth));
}

// collision.rs:282-316 (normal from sphere to box)
static void sphere_box(Vec3 c, Real r, const GeomPose& b, Real margin, std::vector<Hit>& out) {
  Vec3 local = tmul_vec(b.mat, c - b.pos);
  Vec3 h = b.size;
  Vec3 clamped = v3(clampr(local[0], -h[0], h[0]), clampr(local[1], -h[1], h[1]), clampr(local[2], -h[2], h[2]));
  Vec3 diff = local - clamped;
  Real dist = norm(diff);
  if (dist > 1e-12) {
    Real depth = r - dist;
    if (depth <= -margin) return;
    Vec3 n_local = diff * (-1.0 / dist);
    Vec3 n = mul_vec(b.mat, n_local);
    Vec3 surf = b.pos + mul_vec(b.mat, clamped);
    out.push_back(mkhit(surf - n * (depth * 0.5), n, depth));
  } else {
    Real bd = INFINITY, bs = 1.0;
    int bi = 0;
    for (int i = 0; i < 3; i++)
      for (Real s : {-1.0, 1.0}) {
        Real dd = h[i] - s * local[i];
        if (dd < bd) {
          bd = dd;
          bi = i;
          bs = s;
        }
      }
    Vec3 nl = v3zero();
    nl[bi] = -bs;
    Vec3 n = mul_vec(b.mat, nl);
    Real depth = r + bd;
    out.push_back(mkhit(c + n * (r - depth * 0.5), n, depth));
  }
}

// collision.rs:318-335
static void capsule_capsule(const GeomPose& a, const GeomPose& b, Real margin, std::vector<Hit>& out) {
  Vec3 p0, p1, q0, q1;
  segment(a, &p0, &p1);
  segment(b, &q0, &q1);
  Real ra = a.size[0], rb = b.size[0];
  Vec3 x, y;
  closest_segments(p0, p1, q0, q1, &x, &y);
  sphere_sphere(x, ra, y, rb, margin, out);
  Vec3 da = normalized(p1 - p0), db = normalized(q1 - q0);
  if (norm(cross(da, db)) < 0.05) {
    for (Vec3 p : {p0, p1}) {
      Vec3 q = closest_on_segment(q0, q1, p);
      if (norm(q - y) > 0.25 * (ra + rb) || norm(p - x) > 0.25 * (ra + rb)) sphere_sphere(p, ra, q, rb, margin, out);
    }
  }
}

// collision.rs:338-344
static Real box_sdf(const GeomPose& b, Vec3 p) {
  Vec3 l = tmul_vec(b.mat, p - b.pos);
  Vec3 q = vabs(l) - b.size;
  Real outside = norm(vmax(q, v3zero()));
  Real inside = rmin(rmax(rmax(q[0], q[1]), q[2]), 0.0);
  return outside + inside;
}

// collision.rs:346-380
static void capsule_box(const GeomPose& a, const GeomPose& b, Real margin, std::vector<Hit>& out) {
  Vec3 p0, p1;
  segment(a, &p0, &p1);
  Real r = a.size[0];
  auto f = [&](Real t) { return box_sdf(b, p0 + (p1 - p0) * t); };
  const Real g = 0.61803398875;
  Real lo = 0.0, hi = 1.0;
  Real x1 = hi - g * (hi - lo), x2 = lo + g * (hi - lo);
  Real f1 = f(x1), f2 = f(x2);
  for (int it = 0; it < 30; it++) {
    if (f1 < f2) {
      hi = x2;
      x2 = x1;
      f2 = f1;
      x1 = hi - g * (hi - lo);
      f1 = f(x1);
    } else {
      lo = x1;
      x1 = x2;
      f1 = f2;
      x2 = lo + g * (hi - lo);
      f2 = f(x2);
    }
  }
  Real tmin = 0.5 * (lo + hi);
  std::vector<Real> ts{tmin};
  for (Real t : {0.0, 1.0})
    if (std::fabs(t - tmin) > 0.1 && f(t) < r + margin) ts.push_back(t);
  for (Real t : ts) sphere_box(p0 + (p1 - p0) * t, r, b, margin, out);
}

// collision.rs:496-511: Sutherland-Hodgman, keep pn.p <= off
std::vector<Vec3> clip(const std::vector<Vec3>& poly, Vec3 pn, Real off) {
  std::vector<Vec3> out;
  size_t n = poly.size();
  for (size_t i = 0; i < n; i++) {
    Vec3 a = poly[i], b = poly[(i + 1) % n];
    Real da = dot(pn, a) - off, db = dot(pn, b) - off;
    if (da <= 0.0) out.push_back(a);
    if ((da < 0.0) != (db < 0.0) && std::fabs(da - db) > 1e-15) out.push_back(a + (b - a) * (da / (da - db)));
  }
  return out;
}

// collision.rs:514-531
void reduce_to_four(std::vector<DistPt>& pts) {
  if (pts.size() <= 4) return;
  std::vector<DistPt> keep;
  DistPt deepest = pts[0];  // min_by: first minimum
  for (auto& p : pts)
    if (p.d < deepest.d) deepest = p;
  keep.push_back(deepest);
  auto lastmax = [&](auto key) {
    DistPt best = pts[0];
    Real bv = key(pts[0].p);
    for (size_t i = 1; i < pts.size(); i++) {
      Real v = key(pts[i].p);
      if (!(v < bv)) {  // max_by: later element wins ties
        bv = v;
        best = pts[i];
      }
    }
    return best;
  };
  keep.push_back(lastmax([&](Vec3 p) { return norm2(p - deepest.p); }));
  keep.push_back(lastmax([&](Vec3 p) { return norm(cross(keep[1].p - keep[0].p, p - keep[0].p)); }));
  keep.push_back(lastmax([&](Vec3 p) {
    Real s = INFINITY;
    for (auto& k : keep) s = rmin(s, norm(k.p - p));
    return s;
  }));
  pts = keep;
}

// collision.rs:383-493
static void box_box(const GeomPose& a, const GeomPose& b, Real margin, std::vector<Hit>& out) {
  Vec3 d = b.pos - a.pos;
  Vec3 ax[3] = {col(a.mat, 0), col(a.mat, 1), col(a.mat, 2)};
  Vec3 bx[3] = {col(b.mat, 0), col(b.mat, 1), col(b.mat, 2)};
  auto proj = [](const Vec3* axes, Vec3 h, Vec3 l) {
    return h[0] * std::fabs(dot(axes[0], l)) + h[1] * std::fabs(dot(axes[1], l)) + h[2] * std::fabs(dot(axes[2], l));
  };
  bool have_best = false, have_face = false;
  Real best_o = 0, face_o = 0;
  Vec3 best_l = v3zero(), face_l = v3zero();
  int best_k = 0, face_k = 0;
  for (int k = 0; k < 15; k++) {
    Vec3 l;
    if (k < 3) l = ax[k];
    else if (k < 6) l = bx[k - 3];
    else {
      Vec3 c = cross(ax[(k - 6) / 3], bx[(k - 6) % 3]);
      Real n = norm(c);
      if (n < 1e-6) continue;
      l = c * (1.0 / n);
    }
    Real overlap = proj(ax, a.size, l) + proj(bx, b.size, l) - std::fabs(dot(d, l));
    if (overlap < -margin) return;
    if (dot(d, l) < 0.0) l = -l;
    if (!have_best || overlap < best_o) {
      have_best = true;
      best_o = overlap;
      best_l = l;
      best_k = k;
    }
    if (k < 6 && (!have_face || overlap < face_o)) {
      have_face = true;
      face_o = overlap;
      face_l = l;
      face_k = k;
    }
  }
  if (!have_best || !have_face) return;
  if (best_k >= 6 && face_o < best_o * 1.05 + 1e-4) {
    best_o = face_o;
    best_l = face_l;
    best_k = face_k;
  }
  Real overlap = best_o;
  Vec3 n = best_l;
  int k = best_k;
  if (k >= 6) {
    int i = (k - 6) / 3, j = (k - 6) % 3;
    Vec3 pa = a.pos;
    for (int mm = 0; mm < 3; mm++)
      if (mm != i) pa += ax[mm] * (a.size[mm] * signum(dot(ax[mm], n)));
    Vec3 pb = b.pos;
    for (int mm = 0; mm < 3; mm++)
      if (mm != j) pb -= bx[mm] * (b.size[mm] * signum(dot(bx[mm], n)));
    Vec3 x, y;
    closest_segments(pa - ax[i] * a.size[i], pa + ax[i] * a.size[i], pb - bx[j] * b.size[j], pb + bx[j] * b.size[j],
                     &x, &y);
    out.push_back(mkhit((x + y) * 0.5, n, overlap));
    return;
  }
  const GeomPose& rf = k < 3 ? a : b;
  const GeomPose& inc = k < 3 ? b : a;
  const Vec3* raxes = k < 3 ? ax : bx;
  const Vec3* iaxes = k < 3 ? bx : ax;
  Vec3 nref = k < 3 ? n : -n;
  int fi = k < 3 ? k : k - 3;
  Vec3 ref_center = rf.pos + nref * rf.size[fi];
  int u = (fi + 1) % 3, v = (fi + 2) % 3;
  int j = 0;
  Real bestdot = INFINITY;
  for (int mm = 0; mm < 3; mm++) {
    Real dt = dot(iaxes[mm], nref);
    if (-std::fabs(dt) < bestdot) {
      bestdot = -std::fabs(dt);
      j = mm;
    }
  }
  Real s = -signum(dot(iaxes[j], nref));
  Vec3 ic = inc.pos + iaxes[j] * (s * inc.size[j]);
  int ku = (j + 1) % 3, kv = (j + 2) % 3;
  Vec3 eu = iaxes[ku] * inc.size[ku], ev = iaxes[kv] * inc.size[kv];
  std::vector<Vec3> poly = {ic + eu + ev, ic - eu + ev, ic - eu - ev, ic + eu - ev};
  const std::pair<Vec3, Real> sides[2] = {{raxes[u], rf.size[u]}, {raxes[v], rf.size[v]}};
  for (auto& side : sides)
    for (Real sign : {1.0, -1.0}) {
      Vec3 pn = side.first * sign;
      Real off = dot(pn, ref_center) + side.second;
      poly = clip(poly, pn, off);
      if (poly.empty()) return;
    }
  std::vector<DistPt> pts;
  for (Vec3 p : poly) {
    Real sep = dot(p - ref_center, nref);
    if (sep < margin) pts.push_back({sep, p});
  }
  reduce_to_four(pts);
  for (auto& p : pts) out.push_back(mkhit(p.p - nref * (p.d * 0.5), n, -p.d));
}

// collision.rs:59-96: type-ordered dispatch; hits of a swapped call get their
// normals negated
void collide_pair(const GeomPose& a, const GeomPose& b, Real margin, std::vector<Hit>& out) {
  if (a.typ > b.typ) {
    size_t start = out.size();
    collide_pair(b, a, margin, out);
    for (size_t i = start; i < out.size(); i++) out[i].normal = -out[i].normal;
    return;
  }
  int ta = a.typ, tb = b.typ;
  if (ta == GEOM_PLANE && tb == GEOM_SPHERE) {
    plane_sphere(a, b.pos, b.size[0], margin, out);
  } else if (ta == GEOM_PLANE && tb == GEOM_CAPSULE) {
    Vec3 p0, p1;
    segment(b, &p0, &p1);
    size_t start = out.size();
    plane_sphere(a, p0, b.size[0], margin, out);
    plane_sphere(a, p1, b.size[0], margin, out);
    for (size_t i = start; i < out.size(); i++) out[i].tangent = col(b.mat, 2);
  } else if (ta == GEOM_PLANE && tb == GEOM_BOX) {
    plane_box(a, b, margin, out);
  } else if (ta == GEOM_PLANE && tb == GEOM_CYLINDER) {
    plane_cylinder(a, b, margin, out);
  } else if (ta == GEOM_SPHERE && tb == GEOM_SPHERE) {
    sphere_sphere(a.pos, a.size[0], b.pos, b.size[0], margin, out);
  } else if (ta == GEOM_SPHERE && tb == GEOM_CAPSULE) {
    Vec3 p0, p1;
    segment(b, &p0, &p1);
    Vec3 q = closest_on_segment(p0, p1, a.pos);
    sphere_sphere(a.pos, a.size[0], q, b.size[0], margin, out);
  } else if (ta == GEOM_SPHERE && tb == GEOM_BOX) {
    sphere_box(a.pos, a.size[0], b, margin, out);
  } else if (ta == GEOM_CAPSULE && tb == GEOM_CAPSULE) {
    capsule_capsule(a, b, margin, out);
  } else if (ta == GEOM_CAPSULE && tb == GEOM_BOX) {
    capsule_box(a, b, margin, out);
  } else if (ta == GEOM_BOX && tb == GEOM_BOX) {
    box_box(a, b, margin, out);
  }
  (void)pair_supported;
}

}  // namespace om
