// Oracle (test infrastructure only): general convex narrow phase for the pairs
// the reference hands to parry3d-f64 0.31.1 (collision.rs:102-147): mesh
// (convex hull) against anything, and cylinder against non-plane shapes.
// parry3d-f64 is an un-vendored dependency, so this path is this library's
// own algorithm, restated here for the CUDA backend's parity tests; its parity
// with the reference is unpinned (the reference's mesh.rs behaviour tests
// pin it instead).
//
// Every shape is a convex polytope with an optional rounding radius:
//   box        8 vertices, 6 faces
//   cylinder   a 16-sided prism (faces at distance r cos(pi/16) from the axis)
//   mesh       its convex hull (polygon faces and edges from the model)
//   sphere     a point of radius r;  capsule  a segment of radius r
// Polytope pairs use the separating-axis test of the reference's box-box
// routine (collision.rs:383-493) generalised: face normals of both shapes and
// the cross products of edge pairs that form a face of the Minkowski
// difference; a face axis is preferred unless an edge axis is clearly
// shallower; an edge axis gives one contact at the closest points of the
// two edges, a face axis clips the incident face against the reference
// face's side planes and keeps up to four points. Spheres and capsules
// against a polytope use the exact closest point (capsules at the deepest
// point along the segment and at the ends, as capsule-box does), and a plane
// against a hull takes the hull's four deepest vertices (as plane-box does).
#include <algorithm>

#include "om_model.h"

namespace om {

static const int CYL_SIDES = 16;

struct Polytope {
  std::vector<Vec3> v;
  std::vector<Vec3> fn;  // outward unit normals
  std::vector<Real> fd;  // n . x <= d inside
  std::vector<std::vector<int>> loop;
  std::vector<std::array<int, 2>> edge;  // vertex pairs
  std::vector<std::array<int, 2>> eface;  // the two faces of each edge
};

// faces adjacent to each edge, from the face loops
static void edge_faces(Polytope& p) {
  p.eface.assign(p.edge.size(), {-1, -1});
  for (size_t e = 0; e < p.edge.size(); e++) {
    int a = p.edge[e][0], b = p.edge[e][1];
    for (size_t f = 0; f < p.loop.size(); f++) {
      const auto& l = p.loop[f];
      for (size_t k = 0; k < l.size(); k++) {
        int x = l[k], y = l[(k + 1) % l.size()];
        if ((x == a && y == b) || (x == b && y == a)) {
          if (p.eface[e][0] == -1) p.eface[e][0] = (int)f;
          else if (p.eface[e][1] == -1) p.eface[e][1] = (int)f;
        }
      }
    }
  }
}

static Polytope make_polytope(const GeomPose& g) {
  Polytope p;
  auto add_face = [&](Vec3 nl, std::vector<int> loop) {
    Vec3 n = mul_vec(g.mat, nl);
    p.fn.push_back(n);
    p.fd.push_back(dot(n, p.v[loop[0]]));
    p.loop.push_back(loop);
  };
  if (g.typ == GEOM_BOX) {
    for (int i = 0; i < 8; i++) {
      Vec3 s = v3((i & 1) == 0 ? -1.0 : 1.0, (i & 2) == 0 ? -1.0 : 1.0, (i & 4) == 0 ? -1.0 : 1.0);
      p.v.push_back(g.pos + mul_vec(g.mat, mul_elem(g.size, s)));
    }
    add_face(v3(0, 0, -1), {0, 2, 3, 1});
    add_face(v3(1, 0, 0), {1, 3, 7, 5});
    add_face(v3(0, 1, 0), {2, 6, 7, 3});
    add_face(v3(0, -1, 0), {0, 1, 5, 4});
    add_face(v3(-1, 0, 0), {0, 4, 6, 2});
    add_face(v3(0, 0, 1), {4, 5, 7, 6});
    for (int i = 0; i < 8; i++)
      for (int bit = 1; bit < 8; bit <<= 1)
        if (!(i & bit)) p.edge.push_back({i, i | bit});
  } else if (g.typ == GEOM_CYLINDER) {
    const int K = CYL_SIDES;
    Real r = g.size[0], h = g.size[1];
    for (int cap = 0; cap < 2; cap++)
      for (int i = 0; i < K; i++) {
        Real th = 2.0 * M_PI * i / K;
        p.v.push_back(g.pos + mul_vec(g.mat, v3(r * std::cos(th), r * std::sin(th), cap ? h : -h)));
      }
    std::vector<int> bottom, top;
    for (int i = 0; i < K; i++) {
      bottom.push_back((K - i) % K);
      top.push_back(K + i);
    }
    add_face(v3(0, 0, -1), bottom);
    add_face(v3(0, 0, 1), top);
    for (int i = 0; i < K; i++) {
      Real th = 2.0 * M_PI * (i + 0.5) / K;
      add_face(v3(std::cos(th), std::sin(th), 0), {i, (i + 1) % K, K + (i + 1) % K, K + i});
    }
    for (int i = 0; i < K; i++) {
      p.edge.push_back({i, K + i});
      p.edge.push_back({i, (i + 1) % K});
      p.edge.push_back({K + i, K + (i + 1) % K});
    }
  } else {  // mesh: its hull
    const Hull& hl = *g.hull;
    for (const Vec3& x : hl.vert) p.v.push_back(g.pos + mul_vec(g.mat, x));
    for (size_t f = 0; f < hl.face_n.size(); f++) {
      Vec3 n = mul_vec(g.mat, hl.face_n[f]);
      p.fn.push_back(n);
      p.fd.push_back(hl.face_d[f] + dot(n, g.pos));
      p.loop.push_back(hl.face_loop[f]);
    }
    p.edge = hl.edge;
  }
  edge_faces(p);
  return p;
}

// point of the polytope closest to x: returns the signed distance (negative
// inside, then measured to the nearest face plane) and the point
static Real closest_point(const Polytope& p, Vec3 x, Vec3* q, int* inside_face) {
  Real best = -INFINITY;
  int bf = 0;
  for (size_t f = 0; f < p.fn.size(); f++) {
    Real s = dot(p.fn[f], x) - p.fd[f];
    if (s > best) {
      best = s;
      bf = (int)f;
    }
  }
  if (best <= 0.0) {
    *q = x - p.fn[bf] * best;
    *inside_face = bf;
    return best;
  }
  *inside_face = -1;
  Real bd = INFINITY;
  for (size_t f = 0; f < p.fn.size(); f++) {
    Real s = dot(p.fn[f], x) - p.fd[f];
    if (s <= 0.0) continue;
    Vec3 y = x - p.fn[f] * s;
    const auto& l = p.loop[f];
    bool in = true;
    for (size_t k = 0; k < l.size() && in; k++) {
      Vec3 a = p.v[l[k]], b = p.v[l[(k + 1) % l.size()]];
      Vec3 sn = cross(b - a, p.fn[f]);
      if (dot(sn, y - a) > 0.0) in = false;
    }
    if (in && s < bd) {
      bd = s;
      *q = y;
    }
  }
  for (const auto& e : p.edge) {
    Vec3 a = p.v[e[0]], b = p.v[e[1]];
    Vec3 ab = b - a;
    Real t = clampr(dot(x - a, ab) / rmax(dot(ab, ab), 1e-300), 0.0, 1.0);
    Vec3 y = a + ab * t;
    Real d = norm(x - y);
    if (d < bd) {
      bd = d;
      *q = y;
    }
  }
  return bd;
}

// Choices between candidates whose values tie up to rounding take the first
// one within TIE of the best, so that rounding-level differences between
// two implementations cannot change the contacts.
static const Real TIE = 1e-10;

// largest separation of b beyond a face of a: (separation, first face
// within TIE of it)
static Real face_query(const Polytope& a, const Polytope& b, int* face) {
  std::vector<Real> sep(a.fn.size());
  Real best = -INFINITY;
  for (size_t f = 0; f < a.fn.size(); f++) {
    Real mn = INFINITY;
    for (const Vec3& x : b.v) mn = rmin(mn, dot(a.fn[f], x));
    sep[f] = mn - a.fd[f];
    best = rmax(best, sep[f]);
  }
  *face = 0;
  while (*face + 1 < (int)sep.size() && sep[*face] < best - TIE) (*face)++;
  return best;
}

// arcs (a, b) and (c, d) of the Gauss map cross: the edges' cross product is
// a face normal of the Minkowski difference
static bool minkowski_face(Vec3 a, Vec3 b, Vec3 c, Vec3 d) {
  Vec3 bxa = cross(b, a), dxc = cross(d, c);
  Real cba = dot(c, bxa), dba = dot(d, bxa), adc = dot(a, dxc), bdc = dot(b, dxc);
  return cba * dba < 0.0 && adc * bdc < 0.0 && cba * bdc > 0.0;
}

// largest separation along the cross product of an edge of a and an edge of b
static Real edge_query(const Polytope& a, Vec3 ca, const Polytope& b, int* ea, int* eb, Vec3* axis) {
  Real best = -INFINITY;
  *ea = *eb = -1;
  for (size_t i = 0; i < a.edge.size(); i++) {
    if (a.eface[i][1] < 0) continue;
    Vec3 pa = a.v[a.edge[i][0]], da = a.v[a.edge[i][1]] - pa;
    Vec3 na1 = a.fn[a.eface[i][0]], na2 = a.fn[a.eface[i][1]];
    for (size_t j = 0; j < b.edge.size(); j++) {
      if (b.eface[j][1] < 0) continue;
      Vec3 nb1 = b.fn[b.eface[j][0]], nb2 = b.fn[b.eface[j][1]];
      if (!minkowski_face(na1, na2, -nb1, -nb2)) continue;
      Vec3 pb = b.v[b.edge[j][0]], db = b.v[b.edge[j][1]] - pb;
      Vec3 c = cross(da, db);
      Real l = norm(c);
      if (l < 1e-6 * norm(da) * norm(db)) continue;  // parallel edges: a face axis covers them
      Vec3 n = c * (1.0 / l);
      if (dot(n, pa - ca) < 0.0) n = -n;
      Real s = dot(n, pb - pa);
      if (s > best) {
        best = s;
        *ea = (int)i;
        *eb = (int)j;
        *axis = n;
      }
    }
  }
  return best;
}

// FastHull::support_vertex (fasthull.rs:52-120): hulls under 64 vertices
// are scanned (the first maximum); larger ones build each vertex's
// neighbours from the edges and the vertex extreme along each of the 26
// normalised directions (x, y, z) in {-1, 0, 1}^3 (Iterator::max_by keeps the
// last maximum), start from the better of vertex 0 (the hint, never written
// after construction) and the vertex of the seed direction closest to dir,
// then move to the neighbour with the largest projection while one improves.
int hull_support_walk(const std::vector<Vec3>& pts, const std::vector<std::array<int, 2>>& edges, Vec3 dir) {
  const int n = (int)pts.size();
  if (n < 64) {
    int v = 0;
    Real best = -INFINITY;
    for (int i = 0; i < n; i++) {
      Real d = dot(pts[i], dir);
      if (d > best) {
        best = d;
        v = i;
      }
    }
    return v;
  }
  std::vector<std::vector<int>> nb(n);
  for (const auto& e : edges) {
    nb[e[0]].push_back(e[1]);
    nb[e[1]].push_back(e[0]);
  }
  std::vector<std::pair<Vec3, int>> seeds;
  for (int x = -1; x <= 1; x++)
    for (int y = -1; y <= 1; y++)
      for (int z = -1; z <= 1; z++) {
        Vec3 d = v3(x, y, z);
        if (dot(d, d) <= 0.0) continue;
        d = normalized(d);
        int bi = 0;
        for (int i = 1; i < n; i++)
          if (!(dot(pts[i], d) < dot(pts[bi], d))) bi = i;
        seeds.push_back({d, bi});
      }
  int v = 0, seed = 0;
  Real seed_dot = -INFINITY;
  for (const auto& sd : seeds) {
    Real x = dot(sd.first, dir);
    if (x > seed_dot) {
      seed_dot = x;
      seed = sd.second;
    }
  }
  if (dot(pts[seed], dir) > dot(pts[v], dir)) v = seed;
  Real best = dot(pts[v], dir);
  for (;;) {
    int next = v;
    for (int w : nb[v]) {
      Real d = dot(pts[w], dir);
      if (d > best) {
        best = d;
        next = w;
      }
    }
    if (next == v) return v;
    v = next;
  }
}

static Vec3 centroid(const Polytope& p) {
  Vec3 c = v3zero();
  for (const Vec3& x : p.v) c += x;
  return c * (1.0 / (Real)p.v.size());
}

static Hit hit(Vec3 pos, Vec3 n, Real depth) { return Hit{pos, n, depth, v3zero()}; }

// reduce_to_four's choices (collision.rs:514-531: the deepest point, then
// the farthest from it, the farthest from their line, the most isolated),
// each taken within TIE: the first minimum, the last maximum. A clipped
// regular polygon (a cylinder cap) offers many exact ties.
static void reduce_to_four_tie(std::vector<DistPt>& pts) {
  if (pts.size() <= 4) return;
  auto last_max = [&](auto key) {
    Real mx = -INFINITY;
    for (auto& p : pts) mx = rmax(mx, key(p.p));
    size_t bi = 0;
    for (size_t i = 0; i < pts.size(); i++)
      if (key(pts[i].p) >= mx - TIE) bi = i;
    return pts[bi];
  };
  Real mn = INFINITY;
  for (auto& p : pts) mn = rmin(mn, p.d);
  size_t di = 0;
  while (pts[di].d > mn + TIE) di++;
  std::vector<DistPt> keep{pts[di]};
  keep.push_back(last_max([&](Vec3 p) { return norm2(p - keep[0].p); }));
  keep.push_back(last_max([&](Vec3 p) { return norm(cross(keep[1].p - keep[0].p, p - keep[0].p)); }));
  keep.push_back(last_max([&](Vec3 p) {
    Real s = INFINITY;
    for (auto& k : keep) s = rmin(s, norm(k.p - p));
    return s;
  }));
  pts = keep;
}

// reference face `rf` of polytope r (outward normal nref toward the other
// shape), incident polytope s: clip s's most anti-parallel face against the
// side planes of rf and keep the points within the margin (up to four);
// normals point along `n` (a to b)
static void clip_faces(const Polytope& r, int rf, const Polytope& s, Vec3 n, Real margin, std::vector<Hit>& out) {
  Vec3 nref = r.fn[rf];
  Real mn = INFINITY;
  for (size_t f = 0; f < s.fn.size(); f++) mn = rmin(mn, dot(s.fn[f], nref));
  int inc = 0;
  while (inc + 1 < (int)s.fn.size() && dot(s.fn[inc], nref) > mn + TIE) inc++;
  std::vector<Vec3> poly;
  for (int k : s.loop[inc]) poly.push_back(s.v[k]);
  const auto& l = r.loop[rf];
  for (size_t k = 0; k < l.size(); k++) {
    Vec3 a = r.v[l[k]], b = r.v[l[(k + 1) % l.size()]];
    Vec3 sn = normalized(cross(b - a, nref));
    poly = clip(poly, sn, dot(sn, a));
    if (poly.empty()) return;
  }
  std::vector<DistPt> pts;
  for (Vec3 p : poly) {
    Real sep = dot(p, nref) - r.fd[rf];
    if (sep < margin) pts.push_back({sep, p});
  }
  reduce_to_four_tie(pts);
  for (auto& p : pts) out.push_back(hit(p.p - nref * (p.d * 0.5), n, -p.d));
}

static void polytope_polytope(const Polytope& a, const Polytope& b, Real margin, std::vector<Hit>& out) {
  int fa, fb, ea, eb;
  Vec3 axis = v3zero();
  Real sa = face_query(a, b, &fa);
  if (sa > margin) return;
  Real sb = face_query(b, a, &fb);
  if (sb > margin) return;
  Real se = edge_query(a, centroid(a), b, &ea, &eb, &axis);
  if (se > margin) return;
  // overlaps; the shallowest axis wins, a face axis unless an edge axis is
  // clearly shallower (collision.rs:430-436)
  Real oa = -sa, ob = -sb, oe = -se;
  bool face_a = !(ob < oa - TIE);
  Real of = face_a ? oa : ob;
  if (ea >= 0 && oe < of && !(of < oe * 1.05 + 1e-4)) {
    Vec3 pa = a.v[a.edge[ea][0]], qa = a.v[a.edge[ea][1]];
    Vec3 pb = b.v[b.edge[eb][0]], qb = b.v[b.edge[eb][1]];
    Vec3 x, y;
    closest_segments(pa, qa, pb, qb, &x, &y);
    out.push_back(hit((x + y) * 0.5, axis, oe));
    return;
  }
  if (face_a) clip_faces(a, fa, b, a.fn[fa], margin, out);
  else clip_faces(b, fb, a, -b.fn[fb], margin, out);
}

// sphere (center c, radius r) against a polytope; normal from the sphere
static void sphere_polytope(Vec3 c, Real r, const Polytope& p, Real margin, std::vector<Hit>& out) {
  Vec3 q;
  int face;
  Real dist = closest_point(p, c, &q, &face);
  if (face < 0) {
    Real depth = r - dist;
    if (depth <= -margin || dist <= 1e-12) return;
    Vec3 n = (q - c) * (1.0 / dist);
    out.push_back(hit(q - n * (depth * 0.5), n, depth));
  } else {
    Vec3 n = -p.fn[face];
    Real depth = r - dist;
    out.push_back(hit(c + n * (r - depth * 0.5), n, depth));
  }
}

// capsule against a polytope: the deepest point along the axis (golden
// section on the signed distance) and the ends, as capsule-box does
static void capsule_polytope(const GeomPose& a, const Polytope& p, Real margin, std::vector<Hit>& out) {
  Vec3 ax = col(a.mat, 2) * a.size[1];
  Vec3 p0 = a.pos - ax, p1 = a.pos + ax;
  Real r = a.size[0];
  auto f = [&](Real t) {
    Vec3 q;
    int face;
    return closest_point(p, p0 + (p1 - p0) * t, &q, &face);
  };
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
  for (Real t : ts) sphere_polytope(p0 + (p1 - p0) * t, r, p, margin, out);
}

// plane against a hull: its four deepest vertices within the margin
static void plane_polytope(const GeomPose& plane, const Polytope& p, Real margin, std::vector<Hit>& out) {
  Vec3 n = col(plane.mat, 2);
  std::vector<DistPt> hits;
  for (const Vec3& x : p.v) {
    Real d = dot(x - plane.pos, n);
    if (d < margin) hits.push_back({d, x});
  }
  stable_sort_dist(hits);
  for (size_t k = 0; k < hits.size() && k < 4; k++) out.push_back(hit(hits[k].p - n * (hits[k].d * 0.5), n, -hits[k].d));
}

void collide_general(const GeomPose& a, const GeomPose& b, Real margin, std::vector<Hit>& out) {
  if (a.typ > b.typ) {  // type order, normals flipped back (collision.rs:59-67)
    size_t start = out.size();
    collide_general(b, a, margin, out);
    for (size_t i = start; i < out.size(); i++) out[i].normal = -out[i].normal;
    return;
  }
  Polytope pb = make_polytope(b);
  if (a.typ == GEOM_PLANE) {
    plane_polytope(a, pb, margin, out);
  } else if (a.typ == GEOM_SPHERE) {
    sphere_polytope(a.pos, a.size[0], pb, margin, out);
  } else if (a.typ == GEOM_CAPSULE) {
    capsule_polytope(a, pb, margin, out);
  } else {
    polytope_polytope(make_polytope(a), pb, margin, out);
  }
}

}  // namespace om
