// Narrow phase on the device: one lane per geom pair. Restates the primitive
// routines of crates/pippin/src/collision.rs:149-531 and their type-ordered
// dispatch (collision.rs:59-96): normals point from the first geom to the
// second, depth > 0 is penetration, at most 4 points per pair. Sorting and
// "first minimum / last maximum" tie-breaking follow the reference so the
// same points come out in the same order.
#pragma once
#include "pg_math.cuh"
#include "pg_model.h"

namespace pg {

constexpr int MAX_HITS = 4;

struct Hit {
  V3 pos, normal, tangent;
  double depth;
};
struct Hits {
  Hit h[MAX_HITS];
  int n;
  __device__ void push(V3 pos, V3 nrm, double depth) {
    if (n < MAX_HITS) h[n] = Hit{pos, nrm, V3{0, 0, 0}, depth};
    n++;
  }
};
struct GPose {
  int type;
  V3 pos;
  M3 mat;
  V3 size;
  int data;  // mesh id of a mesh geom
};

__device__ inline void segment(const GPose& g, V3* p0, V3* p1) {
  V3 ax = col(g.mat, 2) * g.size.y;
  *p0 = g.pos - ax;
  *p1 = g.pos + ax;
}

// collision.rs:154-162
__device__ inline V3 closest_on_segment(V3 a, V3 b, V3 p) {
  V3 d = b - a;
  double l2 = norm2(d);
  if (l2 < 1e-18) return a;
  double t = clampd(dot(p - a, d) / l2, 0.0, 1.0);
  return a + d * t;
}

// collision.rs:165-201
__device__ inline void closest_segments(V3 p0, V3 p1, V3 q0, V3 q1, V3* x, V3* y) {
  V3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
  double a = norm2(d1), e = norm2(d2), f = dot(d2, r);
  double s, t;
  if (a < 1e-18 && e < 1e-18) {
    *x = p0;
    *y = q0;
    return;
  }
  if (a < 1e-18) {
    s = 0.0;
    t = clampd(f / e, 0.0, 1.0);
  } else {
    double c = dot(d1, r);
    if (e < 1e-18) {
      t = 0.0;
      s = clampd(-c / a, 0.0, 1.0);
    } else {
      double b = dot(d1, d2);
      double denom = a * e - b * b;
      double s0 = denom > 1e-18 ? clampd((b * f - c * e) / denom, 0.0, 1.0) : 0.0;
      double t0 = (b * s0 + f) / e;
      if (t0 < 0.0) {
        t0 = 0.0;
        s0 = clampd(-c / a, 0.0, 1.0);
      } else if (t0 > 1.0) {
        t0 = 1.0;
        s0 = clampd((b - c) / a, 0.0, 1.0);
      }
      s = s0;
      t = t0;
    }
  }
  *x = p0 + d1 * s;
  *y = q0 + d2 * t;
}

// collision.rs:203-212
__device__ inline void plane_sphere(const GPose& pl, V3 c, double r, double margin, Hits& out) {
  V3 n = col(pl.mat, 2);
  double dist = dot(c - pl.pos, n);
  double depth = r - dist;
  if (depth > -margin) out.push(c - (n * (dist + r)) * 0.5, n, depth);
}

struct DP {
  double d;
  V3 p;
};
// stable insertion sort by distance (Rust's sort_by is stable)
__device__ inline void sort_dp(DP* a, int n) {
  for (int i = 1; i < n; i++) {
    DP x = a[i];
    int j = i - 1;
    while (j >= 0 && a[j].d > x.d) {
      a[j + 1] = a[j];
      j--;
    }
    a[j + 1] = x;
  }
}

// collision.rs:214-236
// The larger routines below stay out of line: one copy each keeps the
// step kernel's hot path small enough for the instruction cache.
__device__ __noinline__ void plane_box(const GPose& pl, const GPose& b, double margin, Hits& out) {
  V3 n = col(pl.mat, 2);
  DP hits[8];
  int k = 0;
  for (int i = 0; i < 8; i++) {
    V3 s{(i & 1) == 0 ? -1.0 : 1.0, (i & 2) == 0 ? -1.0 : 1.0, (i & 4) == 0 ? -1.0 : 1.0};
    V3 corner = b.pos + mv(b.mat, mul_elem(b.size, s));
    double dist = dot(corner - pl.pos, n);
    if (dist < margin) hits[k++] = DP{dist, corner};
  }
  sort_dp(hits, k);
  for (int i = 0; i < k && i < 4; i++) out.push(hits[i].p - n * (hits[i].d * 0.5), n, -hits[i].d);
}

// collision.rs:238-267
__device__ __noinline__ void plane_cylinder(const GPose& pl, const GPose& c, double margin, Hits& out) {
  V3 n = col(pl.mat, 2);
  V3 axis = col(c.mat, 2);
  double r = c.size.x, h = c.size.y;
  V3 radial = n - axis * dot(axis, n);
  double rl = norm(radial);
  V3 pts[8];
  int np = 0;
  for (int ci = 0; ci < 2; ci++) {
    double cap = ci == 0 ? -1.0 : 1.0;
    V3 cc = c.pos + axis * (h * cap);
    if (rl > 0.05) {
      V3 d = radial * (-1.0 / rl);
      pts[np++] = cc + d * r;
    } else {
      V3 t1, t2;
      tangents(axis, &t1, &t2);
      pts[np++] = cc + t1 * r;
      pts[np++] = cc + (-t1) * r;
      pts[np++] = cc + t2 * r;
      pts[np++] = cc + (-t2) * r;
    }
  }
  DP hits[8];
  int k = 0;
  for (int i = 0; i < np; i++) {
    double d = dot(pts[i] - pl.pos, n);
    if (d < margin) hits[k++] = DP{d, pts[i]};
  }
  sort_dp(hits, k);
  for (int i = 0; i < k && i < 4; i++) out.push(hits[i].p - n * (hits[i].d * 0.5), n, -hits[i].d);
}

// collision.rs:269-279
__device__ inline void sphere_sphere(V3 c1, double r1, V3 c2, double r2, double margin, Hits& out) {
  V3 d = c2 - c1;
  double dist = norm(d);
  double depth = r1 + r2 - dist;
  if (depth <= -margin) return;
  V3 n = dist > 1e-12 ? d * (1.0 / dist) : V3{0, 0, 1};
  out.push(c1 + n * (r1 - depth * 0.5), n, depth);
}

// collision.rs:282-316 (normal from sphere to box)
__device__ __noinline__ void sphere_box(V3 c, double r, const GPose& b, double margin, Hits& out) {
  V3 local = mtv(b.mat, c - b.pos);
  V3 h = b.size;
  V3 cl{clampd(local.x, -h.x, h.x), clampd(local.y, -h.y, h.y), clampd(local.z, -h.z, h.z)};
  V3 diff = local - cl;
  double dist = norm(diff);
  if (dist > 1e-12) {
    double depth = r - dist;
    if (depth <= -margin) return;
    V3 n = mv(b.mat, diff * (-1.0 / dist));
    V3 surf = b.pos + mv(b.mat, cl);
    out.push(surf - n * (depth * 0.5), n, depth);
  } else {
    double bd = INFINITY, bs = 1.0;
    int bi = 0;
    for (int i = 0; i < 3; i++)
      for (int si = 0; si < 2; si++) {
        double s = si == 0 ? -1.0 : 1.0;
        double d = comp(h, i) - s * comp(local, i);
        if (d < bd) {
          bd = d;
          bi = i;
          bs = s;
        }
      }
    V3 nl{0, 0, 0};
    set_comp(nl, bi, -bs);
    V3 n = mv(b.mat, nl);
    double depth = r + bd;
    out.push(c + n * (r - depth * 0.5), n, depth);
  }
}

// collision.rs:318-335
__device__ __noinline__ void capsule_capsule(const GPose& a, const GPose& b, double margin, Hits& out) {
  V3 p0, p1, q0, q1;
  segment(a, &p0, &p1);
  segment(b, &q0, &q1);
  double ra = a.size.x, rb = b.size.x;
  V3 x, y;
  closest_segments(p0, p1, q0, q1, &x, &y);
  sphere_sphere(x, ra, y, rb, margin, out);
  V3 da = normalized(p1 - p0), db = normalized(q1 - q0);
  if (norm(cross(da, db)) < 0.05) {
    for (int i = 0; i < 2; i++) {
      V3 p = i == 0 ? p0 : p1;
      V3 q = closest_on_segment(q0, q1, p);
      if (norm(q - y) > 0.25 * (ra + rb) || norm(p - x) > 0.25 * (ra + rb)) sphere_sphere(p, ra, q, rb, margin, out);
    }
  }
}

// collision.rs:338-344
__device__ inline double box_sdf(const GPose& b, V3 p) {
  V3 l = mtv(b.mat, p - b.pos);
  V3 q = vabs(l) - b.size;
  double outside = norm(vmax(q, V3{0, 0, 0}));
  double inside = fmin(fmax(fmax(q.x, q.y), q.z), 0.0);
  return outside + inside;
}

// collision.rs:346-380: golden-section minimum of the box SDF along the segment
__device__ __noinline__ void capsule_box(const GPose& a, const GPose& b, double margin, Hits& out) {
  V3 p0, p1;
  segment(a, &p0, &p1);
  double r = a.size.x;
  V3 d = p1 - p0;
  const double g = 0.61803398875;
  double lo = 0.0, hi = 1.0;
  double x1 = hi - g * (hi - lo), x2 = lo + g * (hi - lo);
  double f1 = box_sdf(b, p0 + d * x1), f2 = box_sdf(b, p0 + d * x2);
  for (int it = 0; it < 30; it++) {
    if (f1 < f2) {
      hi = x2;
      x2 = x1;
      f2 = f1;
      x1 = hi - g * (hi - lo);
      f1 = box_sdf(b, p0 + d * x1);
    } else {
      lo = x1;
      x1 = x2;
      f1 = f2;
      x2 = lo + g * (hi - lo);
      f2 = box_sdf(b, p0 + d * x2);
    }
  }
  double tmin = 0.5 * (lo + hi);
  double ts[3];
  int nt = 0;
  ts[nt++] = tmin;
  for (int i = 0; i < 2; i++) {
    double t = (double)i;
    if (fabs(t - tmin) > 0.1 && box_sdf(b, p0 + d * t) < r + margin) ts[nt++] = t;
  }
  for (int i = 0; i < nt; i++) sphere_box(p0 + d * ts[i], r, b, margin, out);
}

// collision.rs:496-511: Sutherland-Hodgman against pn.p <= off. A convex
// polygon gains at most one vertex per clip; `cap` bounds the output even
// if rounding produced more sign changes than that.
constexpr int CLIP_CAP = 16;
__device__ inline int clip_poly(const V3* in, int n, V3 pn, double off, V3* out) {
  int k = 0;
  for (int i = 0; i < n; i++) {
    V3 a = in[i], b = in[(i + 1) % n];
    double da = dot(pn, a) - off, db = dot(pn, b) - off;
    if (da <= 0.0 && k < CLIP_CAP) out[k++] = a;
    if ((da < 0.0) != (db < 0.0) && fabs(da - db) > 1e-15 && k < CLIP_CAP) out[k++] = a + (b - a) * (da / (da - db));
  }
  return k;
}

// collision.rs:514-531
__device__ inline int reduce_to_four(DP* pts, int n) {
  if (n <= 4) return n;
  DP keep[4];
  DP deepest = pts[0];
  for (int i = 1; i < n; i++)
    if (pts[i].d < deepest.d) deepest = pts[i];
  keep[0] = deepest;
  int bi = 0;
  double bv = norm2(pts[0].p - deepest.p);
  for (int i = 1; i < n; i++) {
    double v = norm2(pts[i].p - deepest.p);
    if (!(v < bv)) {
      bv = v;
      bi = i;
    }
  }
  keep[1] = pts[bi];
  bi = 0;
  bv = norm(cross(keep[1].p - keep[0].p, pts[0].p - keep[0].p));
  for (int i = 1; i < n; i++) {
    double v = norm(cross(keep[1].p - keep[0].p, pts[i].p - keep[0].p));
    if (!(v < bv)) {
      bv = v;
      bi = i;
    }
  }
  keep[2] = pts[bi];
  auto spread = [&](V3 p) {
    double s = INFINITY;
    for (int k = 0; k < 3; k++) s = fmin(s, norm(keep[k].p - p));
    return s;
  };
  bi = 0;
  bv = spread(pts[0].p);
  for (int i = 1; i < n; i++) {
    double v = spread(pts[i].p);
    if (!(v < bv)) {
      bv = v;
      bi = i;
    }
  }
  keep[3] = pts[bi];
  for (int k = 0; k < 4; k++) pts[k] = keep[k];
  return 4;
}

// collision.rs:383-493: separating axes, face clipping or edge-edge point
__device__ __noinline__ void box_box(const GPose& a, const GPose& b, double margin, Hits& out) {
  V3 d = b.pos - a.pos;
  V3 ax[3] = {col(a.mat, 0), col(a.mat, 1), col(a.mat, 2)};
  V3 bx[3] = {col(b.mat, 0), col(b.mat, 1), col(b.mat, 2)};
  bool have_best = false, have_face = false;
  double best_o = 0, face_o = 0;
  V3 best_l{0, 0, 0}, face_l{0, 0, 0};
  int best_k = 0, face_k = 0;
  for (int k = 0; k < 15; k++) {
    V3 l;
    if (k < 3) l = ax[k];
    else if (k < 6) l = bx[k - 3];
    else {
      V3 c = cross(ax[(k - 6) / 3], bx[(k - 6) % 3]);
      double n = norm(c);
      if (n < 1e-6) continue;
      l = c * (1.0 / n);
    }
    double pa = a.size.x * fabs(dot(ax[0], l)) + a.size.y * fabs(dot(ax[1], l)) + a.size.z * fabs(dot(ax[2], l));
    double pb = b.size.x * fabs(dot(bx[0], l)) + b.size.y * fabs(dot(bx[1], l)) + b.size.z * fabs(dot(bx[2], l));
    double overlap = pa + pb - fabs(dot(d, l));
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
  double overlap = best_o;
  V3 n = best_l;
  int k = best_k;
  if (k >= 6) {
    int i = (k - 6) / 3, j = (k - 6) % 3;
    V3 pa = a.pos;
    for (int t = 0; t < 3; t++)
      if (t != i) pa = pa + ax[t] * (comp(a.size, t) * signum(dot(ax[t], n)));
    V3 pb = b.pos;
    for (int t = 0; t < 3; t++)
      if (t != j) pb = pb - bx[t] * (comp(b.size, t) * signum(dot(bx[t], n)));
    V3 x, y;
    closest_segments(pa - ax[i] * comp(a.size, i), pa + ax[i] * comp(a.size, i), pb - bx[j] * comp(b.size, j),
                     pb + bx[j] * comp(b.size, j), &x, &y);
    out.push((x + y) * 0.5, n, overlap);
    return;
  }
  const GPose& rf = k < 3 ? a : b;
  const GPose& inc = k < 3 ? b : a;
  const V3* raxes = k < 3 ? ax : bx;
  const V3* iaxes = k < 3 ? bx : ax;
  V3 nref = k < 3 ? n : -n;
  int fi = k < 3 ? k : k - 3;
  V3 ref_center = rf.pos + nref * comp(rf.size, fi);
  int u = (fi + 1) % 3, v = (fi + 2) % 3;
  int j = 0;
  double bestdot = INFINITY;
  for (int t = 0; t < 3; t++) {
    double dt = dot(iaxes[t], nref);
    if (-fabs(dt) < bestdot) {
      bestdot = -fabs(dt);
      j = t;
    }
  }
  double s = -signum(dot(iaxes[j], nref));
  V3 ic = inc.pos + iaxes[j] * (s * comp(inc.size, j));
  int ku = (j + 1) % 3, kv = (j + 2) % 3;
  V3 eu = iaxes[ku] * comp(inc.size, ku), ev = iaxes[kv] * comp(inc.size, kv);
  V3 bufa[CLIP_CAP], bufb[CLIP_CAP];
  bufa[0] = ic + eu + ev;
  bufa[1] = ic - eu + ev;
  bufa[2] = ic - eu - ev;
  bufa[3] = ic + eu - ev;
  int np = 4;
  V3* cur = bufa;
  V3* nxt = bufb;
  for (int side = 0; side < 2; side++) {
    V3 axis = side == 0 ? raxes[u] : raxes[v];
    double ext = side == 0 ? comp(rf.size, u) : comp(rf.size, v);
    for (int sg = 0; sg < 2; sg++) {
      V3 pn = axis * (sg == 0 ? 1.0 : -1.0);
      double off = dot(pn, ref_center) + ext;
      np = clip_poly(cur, np, pn, off, nxt);
      V3* t = cur;
      cur = nxt;
      nxt = t;
      if (np == 0) return;
    }
  }
  DP pts[CLIP_CAP];
  int k2 = 0;
  for (int i = 0; i < np; i++) {
    double sep = dot(cur[i] - ref_center, nref);
    if (sep < margin) pts[k2++] = DP{sep, cur[i]};
  }
  k2 = reduce_to_four(pts, k2);
  for (int i = 0; i < k2; i++) out.push(pts[i].p - nref * (pts[i].d * 0.5), n, -pts[i].d);
}

// collision.rs:104-107: pairs the reference hands to its general convex path
__device__ inline bool needs_general(int a, int b) {
  return a == GEOM_MESH || b == GEOM_MESH || (a == GEOM_CYLINDER && b != GEOM_PLANE) ||
         (b == GEOM_CYLINDER && a != GEOM_PLANE);
}

// collision.rs:59-96: order by type, flip the normals of a swapped call
__device__ __noinline__ void collide_primitive(const GPose& a0, const GPose& b0, double margin, Hits& out) {
  bool swap = a0.type > b0.type;
  const GPose& a = swap ? b0 : a0;
  const GPose& b = swap ? a0 : b0;
  int ta = a.type, tb = b.type;
  if (ta == GEOM_PLANE && tb == GEOM_SPHERE) {
    plane_sphere(a, b.pos, b.size.x, margin, out);
  } else if (ta == GEOM_PLANE && tb == GEOM_CAPSULE) {
    V3 p0, p1;
    segment(b, &p0, &p1);
    int s = out.n;
    plane_sphere(a, p0, b.size.x, margin, out);
    plane_sphere(a, p1, b.size.x, margin, out);
    for (int i = s; i < out.n && i < MAX_HITS; i++) out.h[i].tangent = col(b.mat, 2);
  } else if (ta == GEOM_PLANE && tb == GEOM_BOX) {
    plane_box(a, b, margin, out);
  } else if (ta == GEOM_PLANE && tb == GEOM_CYLINDER) {
    plane_cylinder(a, b, margin, out);
  } else if (ta == GEOM_SPHERE && tb == GEOM_SPHERE) {
    sphere_sphere(a.pos, a.size.x, b.pos, b.size.x, margin, out);
  } else if (ta == GEOM_SPHERE && tb == GEOM_CAPSULE) {
    V3 p0, p1;
    segment(b, &p0, &p1);
    sphere_sphere(a.pos, a.size.x, closest_on_segment(p0, p1, a.pos), b.size.x, margin, out);
  } else if (ta == GEOM_SPHERE && tb == GEOM_BOX) {
    sphere_box(a.pos, a.size.x, b, margin, out);
  } else if (ta == GEOM_CAPSULE && tb == GEOM_CAPSULE) {
    capsule_capsule(a, b, margin, out);
  } else if (ta == GEOM_CAPSULE && tb == GEOM_BOX) {
    capsule_box(a, b, margin, out);
  } else if (ta == GEOM_BOX && tb == GEOM_BOX) {
    box_box(a, b, margin, out);
  }
  if (swap)
    for (int i = 0; i < out.n && i < MAX_HITS; i++) out.h[i].normal = -out.h[i].normal;
}

// collision.rs:47-55: friction frame honouring a preferred tangent
__device__ inline void contact_frame(V3 normal, V3 tangent, V3* t1, V3* t2) {
  V3 t = tangent - normal * dot(normal, tangent);
  if (norm2(t) > 1e-12) {
    *t1 = normalized(t);
    *t2 = cross(normal, *t1);
  } else {
    tangents(normal, t1, t2);
  }
}

}  // namespace pg
