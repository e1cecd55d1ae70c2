// General convex narrow phase on the device: the pairs the reference hands
// to parry3d-f64 (crates/pippin/src/collision.rs:102-147): mesh (convex hull)
// against anything, and cylinder against non-plane shapes. parry is an
// un-vendored dependency; this path is this library's own algorithm, the
// one the oracle restates (FP64; one pair at a time on a whole tile, whose
// lanes share out the polytope queries' candidates):
//   box        8 vertices, 6 faces
//   cylinder   a 16-sided prism (faces at distance r cos(pi/16) from the axis)
//   mesh       its convex hull: polygon faces (at most HULL_FACE_LIMIT long)
//              and edges from the model, with each edge's two faces
//   sphere     a point of radius r;  capsule  a segment of radius r
// Polytope pairs: separating axes over both shapes' face normals and the
// cross products of edge pairs that form a face of the Minkowski difference
// (the box-box test of collision.rs:383-493, generalised); a face axis wins
// unless an edge axis is clearly shallower; an edge axis gives one contact at
// the edges' closest points, a face axis clips the incident face against the
// reference face's side planes (up to four points kept as reduce_to_four
// picks them). Spheres and capsules against a polytope use its exact
// closest point; a plane against a hull takes the four deepest vertices.
// Two accelerations leave the results as they are: hulls of HULL_SCAN_BELOW
// vertices or more find support points by walking their vertex graph
// (fasthull.rs:76-120) instead of scanning, and the edge query skips every
// edge whose separation bound shows it cannot change the contacts.
#pragma once
#include "pg_collide.cuh"
#include "pg_tile.cuh"

namespace pg {

constexpr int GEN_CLIP_CAP = 2 * HULL_FACE_MAX;  // incident loop + one vertex per side plane

// A collide tile's shared scratch for general pairs: the polytope cache
// (poly_cache), clip buffers for faces longer than HULL_FACE_MAX, and the
// edge query's two survivor lists (GEN_SURV_CAP ints each). A pointer is
// nullptr when the model needs none.
struct GenScratch {
  double* cache;
  double* clip;
  int* surv;
};

// box faces (outward normals -z, +x, +y, -y, -x, +z), their loops, edges
// (vertex i to i | bit) and each edge's two faces; vertex i has coordinate
// signs (bit0, bit1, bit2) = (x, y, z) positive
__constant__ int c_box_loop[6][4] = {{0, 2, 3, 1}, {1, 3, 7, 5}, {2, 6, 7, 3}, {0, 1, 5, 4}, {0, 4, 6, 2}, {4, 5, 7, 6}};
__constant__ int c_box_edge[12][2] = {{0, 1}, {0, 2}, {0, 4}, {1, 3}, {1, 5}, {2, 3},
                                      {2, 6}, {3, 7}, {4, 5}, {4, 6}, {5, 7}, {6, 7}};
__constant__ int c_box_eface[12][2] = {{0, 3}, {0, 4}, {3, 4}, {0, 1}, {1, 3}, {0, 2},
                                       {2, 4}, {1, 2}, {3, 5}, {4, 5}, {1, 5}, {2, 5}};
__constant__ double c_box_normal[6][3] = {{0, 0, -1}, {1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {-1, 0, 0}, {0, 0, 1}};

// A box, cylinder prism or hull in the world frame, read on demand, or from
// vc / nc (its world vertices and face normals, 3 doubles each) once a tile
// has filled them (poly_cache).
struct Poly {
  int kind;
  V3 pos;
  M3 mat;
  V3 size;
  const DModel* m;
  int mesh;
  const double* vc = nullptr;
  const double* nc = nullptr;
};

__device__ inline int p_nv(const Poly& p) {
  return p.kind == GEOM_BOX ? 8 : p.kind == GEOM_CYLINDER ? 2 * CYL_SIDES : p.m->hull_vnum[p.mesh];
}
__device__ inline V3 p_v(const Poly& p, int i) {
  if (p.vc) return ld3(p.vc + 3 * i);
  if (p.kind == GEOM_BOX) {
    V3 s{(i & 1) == 0 ? -1.0 : 1.0, (i & 2) == 0 ? -1.0 : 1.0, (i & 4) == 0 ? -1.0 : 1.0};
    return p.pos + mv(p.mat, V3{p.size.x * s.x, p.size.y * s.y, p.size.z * s.z});
  }
  if (p.kind == GEOM_CYLINDER) {
    int cap = i / CYL_SIDES, k = i % CYL_SIDES;
    double th = 2.0 * M_PI * k / CYL_SIDES;
    double r = p.size.x, h = p.size.y;
    return p.pos + mv(p.mat, V3{r * cos(th), r * sin(th), cap ? h : -h});
  }
  return p.pos + mv(p.mat, ld3(p.m->hull_vert + 3 * (p.m->hull_vadr[p.mesh] + i)));
}
__device__ inline int p_nf(const Poly& p) {
  return p.kind == GEOM_BOX ? 6 : p.kind == GEOM_CYLINDER ? CYL_SIDES + 2 : p.m->hull_fnum[p.mesh];
}
__device__ inline int p_fvn(const Poly& p, int f) {
  if (p.kind == GEOM_BOX) return 4;
  if (p.kind == GEOM_CYLINDER) return f < 2 ? CYL_SIDES : 4;
  return p.m->hull_fvnum[p.m->hull_fadr[p.mesh] + f];
}
__device__ inline int p_fv(const Poly& p, int f, int k) {
  if (p.kind == GEOM_BOX) return c_box_loop[f][k];
  if (p.kind == GEOM_CYLINDER) {
    const int K = CYL_SIDES;
    if (f == 0) return (K - k) % K;
    if (f == 1) return K + k;
    int i = f - 2;
    return k == 0 ? i : k == 1 ? (i + 1) % K : k == 2 ? K + (i + 1) % K : K + i;
  }
  return p.m->hull_fv[p.m->hull_fvadr[p.m->hull_fadr[p.mesh] + f] + k];
}
__device__ inline V3 p_fn(const Poly& p, int f) {
  if (p.nc) return ld3(p.nc + 3 * f);
  if (p.kind == GEOM_BOX) return mv(p.mat, V3{c_box_normal[f][0], c_box_normal[f][1], c_box_normal[f][2]});
  if (p.kind == GEOM_CYLINDER) {
    if (f < 2) return mv(p.mat, V3{0.0, 0.0, f == 0 ? -1.0 : 1.0});
    double th = 2.0 * M_PI * ((f - 2) + 0.5) / CYL_SIDES;
    return mv(p.mat, V3{cos(th), sin(th), 0.0});
  }
  return mv(p.mat, ld3(p.m->hull_face + 4 * (p.m->hull_fadr[p.mesh] + f)));
}
__device__ inline double p_fd(const Poly& p, int f, V3 n) {
  if (p.kind == GEOM_MESH) return p.m->hull_face[4 * (p.m->hull_fadr[p.mesh] + f) + 3] + dot(n, p.pos);
  return dot(n, p_v(p, p_fv(p, f, 0)));
}
__device__ inline int p_ne(const Poly& p) {
  return p.kind == GEOM_BOX ? 12 : p.kind == GEOM_CYLINDER ? 3 * CYL_SIDES : p.m->hull_enum[p.mesh];
}
__device__ inline void p_edge(const Poly& p, int e, int* a, int* b) {
  if (p.kind == GEOM_BOX) {
    *a = c_box_edge[e][0];
    *b = c_box_edge[e][1];
  } else if (p.kind == GEOM_CYLINDER) {
    const int K = CYL_SIDES;
    int i = e / 3, t = e % 3;
    *a = t == 2 ? K + i : i;
    *b = t == 0 ? K + i : t == 1 ? (i + 1) % K : K + (i + 1) % K;
  } else {
    int g = p.m->hull_eadr[p.mesh] + e;
    *a = p.m->hull_edge[2 * g];
    *b = p.m->hull_edge[2 * g + 1];
  }
}
__device__ inline void p_eface(const Poly& p, int e, int* f1, int* f2) {
  if (p.kind == GEOM_BOX) {
    *f1 = c_box_eface[e][0];
    *f2 = c_box_eface[e][1];
  } else if (p.kind == GEOM_CYLINDER) {
    const int K = CYL_SIDES;
    int i = e / 3, t = e % 3;
    if (t == 0) {
      *f1 = i == 0 ? 2 : 2 + i - 1;
      *f2 = i == 0 ? 2 + K - 1 : 2 + i;
    } else {
      *f1 = t == 1 ? 0 : 1;
      *f2 = 2 + i;
    }
  } else {
    int g = p.m->hull_eadr[p.mesh] + e;
    *f1 = p.m->hull_eface[2 * g];
    *f2 = p.m->hull_eface[2 * g + 1];
  }
}

// Hull vertex extreme along dl (a direction in the hull's own frame), the
// support query of fasthull.rs:76-120: a hull under HULL_SCAN_BELOW
// vertices is scanned (the first maximum); a larger one starts from the
// better of vertex `hint` and the vertex extreme along the seed direction
// closest to dl, then moves to the neighbour with the largest projection
// while one beats the current vertex. On a convex hull that walk ends at a
// global maximum. Every step raises the projection, so no walk is longer
// than the hull's vertex count.
__device__ inline int hull_support(const DModel& m, int mesh, V3 dl, int hint) {
  const int nv = m.hull_vnum[mesh], base = m.hull_vadr[mesh];
  const double* vert = m.hull_vert + 3 * base;
  auto proj = [&](int i) { return dot(ld3(vert + 3 * i), dl); };
  if (nv < HULL_SCAN_BELOW) {
    int v = 0;
    double best = -INFINITY;
    for (int i = 0; i < nv; i++) {
      double d = proj(i);
      if (d > best) {
        best = d;
        v = i;
      }
    }
    return v;
  }
  // seed directions (x, y, z) / |(x, y, z)| in the order x, y, z from -1 to 1
  const double inv[4] = {0.0, 1.0, 0.70710678118654752440, 0.57735026918962576451};
  int seed = 0, k = 0;
  double sd = -INFINITY;
  for (int x = -1; x <= 1; x++)
    for (int y = -1; y <= 1; y++)
      for (int z = -1; z <= 1; z++) {
        if (!x && !y && !z) continue;
        double d = (x * dl.x + y * dl.y + z * dl.z) * inv[x * x + y * y + z * z];
        if (d > sd) {
          sd = d;
          seed = m.hull_seed[HULL_SEEDS * mesh + k];
        }
        k++;
      }
  int v = hint < 0 ? 0 : (hint >= nv ? nv - 1 : hint);
  double best = proj(v);
  double ds = proj(seed);
  if (ds > best) {
    best = ds;
    v = seed;
  }
  for (int step = 0; step < nv; step++) {
    int next = v;
    const int* nb = m.hull_nb + m.hull_nbadr[base + v];
    const int nn = m.hull_nbnum[base + v];
    for (int j = 0; j < nn; j++) {
      double d = proj(nb[j]);
      if (d > best) {
        best = d;
        next = nb[j];
      }
    }
    if (next == v) break;
    v = next;
  }
  return v;
}

__device__ inline bool p_walks(const Poly& p) { return p.kind == GEOM_MESH && p.m->hull_vnum[p.mesh] >= HULL_SCAN_BELOW; }

// Point of the polytope closest to x: the signed distance (negative inside,
// then to the nearest face plane), the point, and the face when inside (-1
// outside). Outside, the closest point lies on a face (projection inside
// its loop) or on an edge. The faces and edges are shared out over the
// tile's lanes; every choice is the one a loop over the faces, then the
// edges, in order with strict comparisons makes (the first maximum inside,
// the first minimum outside), and every lane returns the result.
template <int G>
__device__ __noinline__ double closest_point(const Tile<G>& T, const Poly& p, V3 x, V3* q, int* inside_face) {
  const int nf = p_nf(p), ne = p_ne(p);
  double best = -INFINITY;
  int bf = 0x7fffffff;
  for (int f = T.lane(); f < nf; f += G) {
    V3 n = p_fn(p, f);
    double s = dot(n, x) - p_fd(p, f, n);
    if (s > best) {
      best = s;
      bf = f;
    }
  }
  T.argmax(&best, &bf);
  if (bf == 0x7fffffff) bf = 0;
  if (best <= 0.0) {
    *q = x - p_fn(p, bf) * best;
    *inside_face = bf;
    return best;
  }
  *inside_face = -1;
  // candidates in the order faces (index f), then edges (index nf + e)
  double bd = INFINITY;
  int bk = 0x7fffffff;
  for (int f = T.lane(); f < nf; f += G) {
    V3 n = p_fn(p, f);
    double s = dot(n, x) - p_fd(p, f, n);
    if (s <= 0.0) continue;
    V3 y = x - n * s;
    int nl = p_fvn(p, f);
    bool in = true;
    for (int k = 0; k < nl && in; k++) {
      V3 a = p_v(p, p_fv(p, f, k)), b = p_v(p, p_fv(p, f, (k + 1) % nl));
      V3 sn = cross(b - a, n);
      if (dot(sn, y - a) > 0.0) in = false;
    }
    if (in && s < bd) {
      bd = s;
      bk = f;
    }
  }
  for (int e = T.lane(); e < ne; e += G) {
    int ia, ib;
    p_edge(p, e, &ia, &ib);
    V3 a = p_v(p, ia), b = p_v(p, ib);
    V3 ab = b - a;
    double t = clampd(dot(x - a, ab) / fmax(dot(ab, ab), 1e-300), 0.0, 1.0);
    double d = norm(x - (a + ab * t));
    if (d < bd) {
      bd = d;
      bk = nf + e;
    }
  }
  double nb = -bd;
  T.argmax(&nb, &bk);
  bd = -nb;
  if (bk < nf) {
    V3 n = p_fn(p, bk);
    *q = x - n * (dot(n, x) - p_fd(p, bk, n));
  } else if (bk != 0x7fffffff) {
    int ia, ib;
    p_edge(p, bk - nf, &ia, &ib);
    V3 a = p_v(p, ia), b = p_v(p, ib);
    V3 ab = b - a;
    double t = clampd(dot(x - a, ab) / fmax(dot(ab, ab), 1e-300), 0.0, 1.0);
    *q = a + ab * t;
  }
  return bd;
}

// Choices between candidates whose values tie up to rounding take the first
// one within GEN_TIE of the best, so that rounding-level differences (from
// the host's oracle, say) cannot change the contacts.
constexpr double GEN_TIE = 1e-10;

// largest separation of b beyond a face of a (first face within GEN_TIE),
// the faces shared out over the tile's lanes: the maximum, then the lowest
// face index within GEN_TIE of it, as a loop over the faces in order finds.
// b's vertex deepest below a face comes from a scan, or from the support
// walk when b is a hull of HULL_SCAN_BELOW vertices or more.
template <int G>
__device__ double face_query(const Tile<G>& T, const Poly& a, const Poly& b, int* face) {
  int nf = p_nf(a), nv = p_nv(b);
  const bool walk = p_walks(b);
  int hint = 0;  // a large hull's walks start from this lane's last answer
  auto sep = [&](int f) {
    V3 n = p_fn(a, f);
    double mn = INFINITY;
    if (walk) {
      hint = hull_support(*b.m, b.mesh, mtv(b.mat, -n), hint);
      mn = dot(n, p_v(b, hint));
    } else {
      for (int i = 0; i < nv; i++) mn = fmin(mn, dot(n, p_v(b, i)));
    }
    return mn - p_fd(a, f, n);
  };
  double best = -INFINITY;
  for (int f = T.lane(); f < nf; f += G) best = fmax(best, sep(f));
  best = T.fmax(best);
  int first = nf;
  for (int f = T.lane(); f < nf; f += G)
    if (!(sep(f) < best - GEN_TIE)) {
      first = f;
      break;
    }
  first = T.imin(first);
  *face = first < nf ? first : nf - 1;
  return best;
}

// arcs (a, b) and (c, d) of the Gauss map cross: the edges' cross product
// is a face normal of the Minkowski difference
__device__ inline bool minkowski_face(V3 a, V3 b, V3 c, V3 d) {
  V3 bxa = cross(b, a), dxc = cross(d, c);
  double cba = dot(c, bxa), dba = dot(d, bxa), adc = dot(a, dxc), bdc = dot(b, dxc);
  return cba * dba < 0.0 && adc * bdc < 0.0 && cba * bdc > 0.0;
}

// Largest u.w over the unit vectors u on the great-circle arc from n1 to n2
// (the outward normals of an edge's two faces, less than pi apart): the
// projection of w onto the arc's plane when it points between n1 and n2,
// else the better end.
__device__ inline double arc_max(V3 n1, V3 n2, V3 w) {
  double mx = fmax(dot(n1, w), dot(n2, w));
  V3 e = cross(n1, n2);
  double ee = dot(e, e);
  if (!(ee > 0.0)) return mx;
  V3 wp = w - e * (dot(e, w) / ee);
  if (dot(cross(n1, wp), e) > 0.0 && dot(cross(wp, n2), e) > 0.0) mx = fmax(mx, norm(wp));
  return mx;
}

// Index of p's vertex with the largest projection on dir: the walk for a
// large hull (every lane takes the same walk), else a scan shared out over
// the lanes.
template <int G>
__device__ int support_index(const Tile<G>& T, const Poly& p, V3 dir) {
  if (p_walks(p)) return hull_support(*p.m, p.mesh, mtv(p.mat, dir), 0);
  double best = -INFINITY;
  int bi = 0x7fffffff;
  for (int i = T.lane(); i < p_nv(p); i += G) {
    double d = dot(dir, p_v(p, i));
    if (d > best) {
      best = d;
      bi = i;
    }
  }
  T.argmax(&best, &bi);
  return bi == 0x7fffffff ? 0 : bi;
}

// Edge pruning. For an edge pair that forms a face of the Minkowski
// difference, its axis u lies on the arc of p's edge e, and the separation
// along it is -h_p(u) - h_q(-u) with h the support function. h_p(u) = u.x_e
// for any point x_e of the edge and h_q(-u) >= -u.y for any point y of q, so
// the separation is at most arc_max(n1, n2, y - x_e) for every y in q (with
// the roles of a and b swapped for b's edges). The witnesses y are q's
// vertices on its best face fq (up to eight, evenly spread) and q's vertex
// deepest below p's best face fp. An edge whose bound is below the pair's
// threshold cannot take part in the result, and is dropped with every pair
// it forms.
__device__ inline double edge_bound(const Poly& p, int e, const Poly& q, int fq, int yq) {
  int f1, f2, i0, i1;
  p_eface(p, e, &f1, &f2);
  if (f2 < 0) return -INFINITY;  // not between two faces: never a candidate
  p_edge(p, e, &i0, &i1);
  V3 xe = p_v(p, i0), n1 = p_fn(p, f1), n2 = p_fn(p, f2);
  double bd = arc_max(n1, n2, p_v(q, yq) - xe);
  int nl = p_fvn(q, fq), step = (nl + 7) / 8;
  for (int k = 0; k < nl; k += step) bd = fmin(bd, arc_max(n1, n2, p_v(q, p_fv(q, fq, k)) - xe));
  return bd;
}

// Lists p's edges whose bound reaches thr (ascending) in out[0, GEN_SURV_CAP);
// returns how many there are (past the cap only counted).
template <int G>
__device__ int edge_survivors(const Tile<G>& T, const Poly& p, const Poly& q, int fq, int yq, double thr, int* out) {
  int ne = p_ne(p), cnt = 0;
  for (int base = 0; base < ne; base += G) {
    int e = base + T.lane();
    bool keep = e < ne && !(edge_bound(p, e, q, fq, yq) < thr);
    unsigned mask = T.ballot(keep);
    if (keep) {
      unsigned below = T.lane() == 0 ? 0u : (mask & (0xffffffffu >> (32 - T.lane())));
      int pos = cnt + __popc(below);
      if (pos < GEN_SURV_CAP) out[pos] = e;
    }
    cnt += __popc(mask);
  }
  return cnt;
}

// largest separation along the cross product of an edge of a and of b; the
// edge pairs (i, j), in the order i * (edges of b) + j, are shared out over
// the tile's lanes, and the first pair with the largest separation wins, as
// a loop over the pairs in order with a strict comparison finds. With
// `surv`, only pairs of edges whose bound (edge_bound) reaches thr are
// visited: fa / fb are a's and b's best faces, and thr lies below every
// separation that could change the contacts, so the pairs skipped could
// not have been the winner where the winner matters.
template <int G>
__device__ double edge_query(const Tile<G>& T, const Poly& a, V3 ca, const Poly& b, int fa, int fb, double thr,
                             int* surv, int* ea, int* eb, V3* axis) {
  int nea = p_ne(a), neb = p_ne(b);
  // separation along the pair's axis; false when the pair is not a candidate
  auto pair_sep = [&](int i, int j, double* s, V3* n) -> bool {
    int fa1, fa2, fb1, fb2, ia, ja, ib, jb;
    p_eface(a, i, &fa1, &fa2);
    p_eface(b, j, &fb1, &fb2);
    if (fa2 < 0 || fb2 < 0) return false;
    if (!minkowski_face(p_fn(a, fa1), p_fn(a, fa2), -p_fn(b, fb1), -p_fn(b, fb2))) return false;
    p_edge(a, i, &ia, &ja);
    p_edge(b, j, &ib, &jb);
    V3 pa = p_v(a, ia), da = p_v(a, ja) - pa;
    V3 pb = p_v(b, ib), db = p_v(b, jb) - pb;
    V3 c = cross(da, db);
    double l = norm(c);
    if (l < 1e-6 * norm(da) * norm(db)) return false;  // parallel edges: a face axis covers them
    V3 u = c * (1.0 / l);
    if (dot(u, pa - ca) < 0.0) u = -u;
    *s = dot(u, pb - pa);
    *n = u;
    return true;
  };
  double best = -INFINITY;
  int bidx = 0x7fffffff;
  int na = -1, nb = -1;
  if (surv) {
    int yb = support_index(T, b, -p_fn(a, fa));  // b's vertex deepest below a's best face
    int ya = support_index(T, a, -p_fn(b, fb));
    T.sync();  // the lists of the previous pair are read
    na = edge_survivors(T, a, b, fb, yb, thr, surv);
    nb = na > 0 ? edge_survivors(T, b, a, fa, ya, thr, surv + GEN_SURV_CAP) : 0;
    T.sync();
  }
  if (na >= 0 && na <= GEN_SURV_CAP && nb <= GEN_SURV_CAP) {
    for (int k = T.lane(); k < na * nb; k += G) {
      int i = surv[k / nb], j = surv[GEN_SURV_CAP + k % nb];
      double sk;
      V3 nk;
      if (pair_sep(i, j, &sk, &nk) && sk > best) {
        best = sk;
        bidx = i * neb + j;
      }
    }
  } else {
    for (int k = T.lane(); k < nea * neb; k += G) {
      double sk;
      V3 nk;
      if (pair_sep(k / neb, k % neb, &sk, &nk) && sk > best) {
        best = sk;
        bidx = k;
      }
    }
  }
  T.argmax(&best, &bidx);
  *ea = *eb = -1;
  if (bidx != 0x7fffffff) {
    double sk;
    pair_sep(bidx / neb, bidx % neb, &sk, axis);
    *ea = bidx / neb;
    *eb = bidx % neb;
  }
  return best;
}

__device__ inline V3 p_centroid(const Poly& p) {
  V3 c{0.0, 0.0, 0.0};
  int nv = p_nv(p);
  for (int i = 0; i < nv; i++) c = c + p_v(p, i);
  return c * (1.0 / (double)nv);
}

// reduce_to_four's choices (collision.rs:514-531: the deepest point, then
// the farthest from it, the farthest from their line, the most isolated),
// each taken within GEN_TIE: the first minimum, the last maximum. A clipped
// regular polygon (a cylinder cap) offers many exact ties.
__device__ __noinline__ int reduce_to_four_tie(DP* pts, int n) {
  if (n <= 4) return n;
  DP keep[4];
  double mn = INFINITY;
  for (int i = 0; i < n; i++) mn = fmin(mn, pts[i].d);
  int di = 0;
  while (pts[di].d > mn + GEN_TIE) di++;
  keep[0] = pts[di];
  for (int k = 1; k < 4; k++) {
    auto key = [&](V3 p) {
      if (k == 1) return norm2(p - keep[0].p);
      if (k == 2) return norm(cross(keep[1].p - keep[0].p, p - keep[0].p));
      double s = INFINITY;
      for (int j = 0; j < 3; j++) s = fmin(s, norm(keep[j].p - p));
      return s;
    };
    double mx = -INFINITY;
    for (int i = 0; i < n; i++) mx = fmax(mx, key(pts[i].p));
    int bi = 0;
    for (int i = 0; i < n; i++)
      if (key(pts[i].p) >= mx - GEN_TIE) bi = i;
    keep[k] = pts[bi];
  }
  for (int k = 0; k < 4; k++) pts[k] = keep[k];
  return 4;
}

// Sutherland-Hodgman against pn.p <= off into at most `cap` vertices
__device__ inline int clip_poly_cap(const V3* in, int n, V3 pn, double off, V3* out, int cap) {
  int k = 0;
  for (int i = 0; i < n; i++) {
    V3 a = in[i], b = in[(i + 1) % n];
    double da = dot(pn, a) - off, db = dot(pn, b) - off;
    if (da <= 0.0 && k < cap) out[k++] = a;
    if ((da < 0.0) != (db < 0.0) && fabs(da - db) > 1e-15 && k < cap) out[k++] = a + (b - a) * (da / (da - db));
  }
  return k;
}

// reference face rf of r (outward normal toward s), incident polytope s:
// clip s's most anti-parallel face against rf's side planes, keep the points
// within the margin (up to four); (first geom to second). The clip runs in `area` (10 cap
// doubles: two polygon buffers of cap vertices, then cap kept points) when
// given, else in the lane's own buffers of GEN_CLIP_CAP.
__device__ __noinline__ void clip_faces(const Poly& r, int rf, const Poly& s, V3 n, double margin, Hits& out,
                                        double* area, int cap) {
  V3 nref = p_fn(r, rf);
  double dref = p_fd(r, rf, nref);
  int nfs = p_nf(s), inc = 0;
  double mn = INFINITY;
  for (int f = 0; f < nfs; f++) mn = fmin(mn, dot(p_fn(s, f), nref));
  while (inc + 1 < nfs && dot(p_fn(s, inc), nref) > mn + GEN_TIE) inc++;
  V3 lbuf[2][GEN_CLIP_CAP];
  DP lpts[GEN_CLIP_CAP];
  V3* buf[2] = {lbuf[0], lbuf[1]};
  DP* pts = lpts;
  if (area) {
    buf[0] = reinterpret_cast<V3*>(area);
    buf[1] = buf[0] + cap;
    pts = reinterpret_cast<DP*>(area + 6 * cap);
  } else {
    cap = GEN_CLIP_CAP;
  }
  int np = p_fvn(s, inc), cur = 0;
  for (int k = 0; k < np && k < cap; k++) buf[0][k] = p_v(s, p_fv(s, inc, k));
  np = np < cap ? np : cap;
  int nl = p_fvn(r, rf);
  for (int k = 0; k < nl; k++) {
    V3 a = p_v(r, p_fv(r, rf, k)), b = p_v(r, p_fv(r, rf, (k + 1) % nl));
    V3 sn = normalized(cross(b - a, nref));
    np = clip_poly_cap(buf[cur], np, sn, dot(sn, a), buf[cur ^ 1], cap);
    cur ^= 1;
    if (np == 0) return;
  }
  int n_pts = 0;
  for (int k = 0; k < np; k++) {
    double sep = dot(buf[cur][k], nref) - dref;
    if (sep < margin) pts[n_pts++] = DP{sep, buf[cur][k]};
  }
  n_pts = reduce_to_four_tie(pts, n_pts);
  for (int k = 0; k < n_pts; k++) out.push(pts[k].p - nref * (pts[k].d * 0.5), n, -pts[k].d);
}

template <int G>
__device__ void polytope_polytope(const Tile<G>& T, const Poly& a, const Poly& b, double margin, Hits& out,
                                  int owner, const GenScratch& gs) {
  int fa, fb, ea, eb;
  V3 axis{0.0, 0.0, 0.0};
  double sa = face_query(T, a, b, &fa);
  if (sa > margin) return;
  double sb = face_query(T, b, a, &fb);
  if (sb > margin) return;
  // An edge axis changes the contacts only when its separation is above
  // the margin (no contact) or wins over the face axis below (the edge
  // contact); the face separation used there is at least max(sa, sb) -
  // GEN_TIE. Edges bounded below thr are skipped (edge_query); 1e-9 covers
  // the rounding of the bounds.
  double sfl = fmax(sa, sb) - GEN_TIE;
  double thr = fmin(margin, fmax(sfl, (sfl + 1e-4) / 1.05)) - 1e-9;
  double se = edge_query(T, a, p_centroid(a), b, fa, fb, thr, gs.surv, &ea, &eb, &axis);
  if (se > margin) return;
  double oa = -sa, ob = -sb, oe = -se;
  bool face_a = !(ob < oa - GEN_TIE);
  double of = face_a ? oa : ob;
  if (T.lane() != owner) return;  // the contact points: on the owning lane only
  if (ea >= 0 && oe < of && !(of < oe * 1.05 + 1e-4)) {
    int i0, i1, j0, j1;
    p_edge(a, ea, &i0, &i1);
    p_edge(b, eb, &j0, &j1);
    V3 x, y;
    closest_segments(p_v(a, i0), p_v(a, i1), p_v(b, j0), p_v(b, j1), &x, &y);
    out.push((x + y) * 0.5, axis, oe);
    return;
  }
  const int cap = 2 * a.m->gen_lmax;
  if (face_a) clip_faces(a, fa, b, p_fn(a, fa), margin, out, gs.clip, cap);
  else clip_faces(b, fb, a, -p_fn(b, fb), margin, out, gs.clip, cap);
}

// sphere (center c, radius r) against a polytope; normal from the sphere;
// the contact on lane `owner`
template <int G>
__device__ void sphere_polytope(const Tile<G>& T, V3 c, double r, const Poly& p, double margin, Hits& out, int owner) {
  V3 q{0.0, 0.0, 0.0};
  int face;
  double dist = closest_point(T, p, c, &q, &face);
  if (T.lane() != owner) return;
  if (face < 0) {
    double depth = r - dist;
    if (depth <= -margin || dist <= 1e-12) return;
    V3 n = (q - c) * (1.0 / dist);
    out.push(q - n * (depth * 0.5), n, depth);
  } else {
    V3 n = -p_fn(p, face);
    double depth = r - dist;
    out.push(c + n * (r - depth * 0.5), n, depth);
  }
}

// capsule against a polytope: the deepest point along the axis (golden
// section on the signed distance) and the ends, as capsule-box does
template <int G>
__device__ void capsule_polytope(const Tile<G>& T, const GPose& a, const Poly& p, double margin, Hits& out, int owner) {
  V3 ax = col(a.mat, 2) * a.size.y;
  V3 p0 = a.pos - ax, p1 = a.pos + ax;
  double r = a.size.x;
  auto f = [&](double t) {
    V3 q;
    int face;
    return closest_point(T, p, p0 + (p1 - p0) * t, &q, &face);
  };
  const double g = 0.61803398875;
  double lo = 0.0, hi = 1.0;
  double x1 = hi - g * (hi - lo), x2 = lo + g * (hi - lo);
  double f1 = f(x1), f2 = f(x2);
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
  double tmin = 0.5 * (lo + hi);
  sphere_polytope(T, p0 + (p1 - p0) * tmin, r, p, margin, out, owner);
  for (int e = 0; e < 2; e++) {
    double t = e == 0 ? 0.0 : 1.0;
    if (fabs(t - tmin) > 0.1 && f(t) < r + margin) sphere_polytope(T, p0 + (p1 - p0) * t, r, p, margin, out, owner);
  }
}

// plane against a hull: the four deepest vertices within the margin, in
// the order a stable sort by depth gives (equal depths by vertex index).
// Each lane keeps the four best of its share of the vertices by (depth,
// index); four tile-wide minima then pick the result, which lane `owner`
// records.
template <int G>
__device__ void plane_polytope(const Tile<G>& T, const GPose& pl, const Poly& p, double margin, Hits& out, int owner) {
  V3 n = col(pl.mat, 2);
  double kd[4];
  int ki[4];
  int nk = 0;
  int nv = p_nv(p);
  for (int i = T.lane(); i < nv; i += G) {
    double d = dot(p_v(p, i) - pl.pos, n);
    if (!(d < margin)) continue;
    if (nk == 4 && !(d < kd[3])) continue;
    int j = nk < 4 ? nk++ : 3;
    while (j > 0 && kd[j - 1] > d) {
      kd[j] = kd[j - 1];
      ki[j] = ki[j - 1];
      j--;
    }
    kd[j] = d;
    ki[j] = i;
  }
  int head = 0, ns = 0, sel[4];
  for (int r = 0; r < 4; r++) {
    double v = head < nk ? -kd[head] : -INFINITY;
    int idx = head < nk ? ki[head] : 0x7fffffff;
    T.argmax(&v, &idx);
    if (idx == 0x7fffffff) break;
    sel[ns++] = idx;
    if (head < nk && ki[head] == idx) head++;
  }
  if (T.lane() != owner) return;
  for (int k = 0; k < ns; k++) {
    V3 x = p_v(p, sel[k]);
    double d = dot(x - pl.pos, n);
    out.push(x - n * (d * 0.5), n, -d);
  }
}

// Fills buf with p's world vertices, then its world face normals (the values
// p_v and p_fn give), shared out over the tile's lanes, and points p at them.
// buf holds 3 (nv + nf) doubles.
template <int G>
__device__ void poly_cache(const Tile<G>& T, Poly& p, double* buf) {
  int nv = p_nv(p), nf = p_nf(p);
  T.sync();  // every lane is done with the previous pair's cache
  for (int i = T.lane(); i < nv; i += G) st3(buf + 3 * i, p_v(p, i));
  for (int f = T.lane(); f < nf; f += G) st3(buf + 3 * (nv + f), p_fn(p, f));
  T.sync();
  p.vc = buf;
  p.nc = buf + 3 * nv;
}

// One pair on the whole tile: every lane passes the same pair; the polytope
// queries, closest-point searches and deepest-vertex picks share their
// candidates out over the lanes, and the contacts are formed (the clipping
// included) on lane `owner` alone, whose `out` gets them (the other lanes'
// stays as it was: their clip and point buffers stay untouched, so the
// tile's local-memory footprint is one lane's). With
// gs.cache (6 (gen_vmax + gen_fmax) doubles of the tile's shared memory) the
// polytopes' world vertices and normals are formed once instead of at every
// use.
template <int G>
__device__ __noinline__ void collide_general(const Tile<G>& T, const DModel& m, const GPose& a0, const GPose& b0,
                                             double margin, Hits& out, const GenScratch& gs, int owner) {
  double* cache = gs.cache;
  bool swap = a0.type > b0.type;  // type order, normals flipped back (collision.rs:59-67)
  const GPose& a = swap ? b0 : a0;
  const GPose& b = swap ? a0 : b0;
  int start = out.n;
  Poly pb{b.type, b.pos, b.mat, b.size, &m, b.data};
  if (cache) poly_cache(T, pb, cache);
  const bool own = T.lane() == owner;
  if (a.type == GEOM_PLANE) {
    plane_polytope(T, a, pb, margin, out, owner);
  } else if (a.type == GEOM_SPHERE) {
    sphere_polytope(T, a.pos, a.size.x, pb, margin, out, owner);
  } else if (a.type == GEOM_CAPSULE) {
    capsule_polytope(T, a, pb, margin, out, owner);
  } else {
    Poly pa{a.type, a.pos, a.mat, a.size, &m, a.data};
    if (cache) poly_cache(T, pa, cache + 3 * (m.gen_vmax + m.gen_fmax));
    polytope_polytope(T, pa, pb, margin, out, owner, gs);
  }
  if (swap && own)
    for (int k = start; k < out.n && k < MAX_HITS; k++) out.h[k].normal = -out.h[k].normal;
}

}  // namespace pg
