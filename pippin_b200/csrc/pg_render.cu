// Batched rasteriser: every (environment, view) image is cut into tiles of
// 64 x 64 or 128 x 128 pixels and one block renders one tile at a time (persistent grid,
// work items handed out in order). A block keeps a visibility buffer for its
// tile in shared memory: per pixel the 64-bit minimum of (depth bits << 32 |
// 2 * triangle + sub-triangle), so the nearest fragment wins and equal depths
// go to the earlier triangle, as a depth test `Less` over triangles drawn in
// order does. Triangles are transformed, clipped at the near plane and set
// up one per thread; small ones are scanned by their thread, large ones are
// queued and scanned once every triangle is set up (no thread waits for
// another while drawing): planes by the whole block, thin sides a warp each.
// A resolve pass then recomputes the winning triangle at each pixel,
// interpolates its attributes with perspective correction and shades it
// (render.metal:67-128), writing RGBA8, linear depth and segmentation in
// (image, y, x) order (:130-145).
//
// The file is compiled without FMA contraction: every product and sum is
// rounded on its own, in the order written, so that a CPU evaluation of the
// same expressions in IEEE single precision gives the same bits.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pippin_b200.h"
#include "../../include/pippin_b200_render.h"

namespace pg {
void internal_set_error(const std::string& msg);
}

namespace {

// Tiles of RT x RT pixels with NT threads: 64 x 64 with 256 threads (three
// blocks an SM) for images up to 64 pixels, else 128 x 128 with 512 threads
// (one block an SM). Each tile first culls the geoms whose bounding spheres
// cannot reach it.
constexpr int BIG_PIX = 64;       // bounding boxes above this many pixels are queued (scanned by a warp or the block)
constexpr int QWORDS = 14;        // x[3], y[3], z[3], id, x0, y0, x1, y1
constexpr unsigned long long EMPTY = ~0ull;

struct RArgs {
  const float* verts;
  const float* radius;  // per geom: the largest vertex distance from its origin, at unit scale
  const uint32_t* tris;
  int ntri, ngeom, ncam, nview;
  const float* views;
  int W, H, tiles_x, tiles_y;
  float near_, far_, A, An, L0, L1, L2;
  const float* geoms;
  const float* cams;
  const float* app;
  int nenv;
  uint8_t* rgba;
  float* depth;
  int32_t* seg;
};

// one polygon vertex: camera-space position, camera-space normal, local xy
struct PV {
  float a[8];
};

__device__ __forceinline__ void cam_xform(const float* v, const float* g, const float* ap, const float* c, float* pc) {
  float p0 = v[0] * ap[4], p1 = v[1] * ap[5], p2 = v[2] * ap[6];
  float w[3];
#pragma unroll
  for (int i = 0; i < 3; i++) w[i] = ((g[3 + 3 * i] * p0 + g[4 + 3 * i] * p1) + g[5 + 3 * i] * p2) + g[i];
  float d0 = w[0] - c[0], d1 = w[1] - c[1], d2 = w[2] - c[2];
#pragma unroll
  for (int i = 0; i < 3; i++) pc[i] = (c[3 + i] * d0 + c[6 + i] * d1) + c[9 + i] * d2;
}

// is[k] = 1 / max(scale[k], 1e-6): the inverse transpose of the geom's scale
__device__ __forceinline__ void cam_normal(const float* v, const float* g, const float* is, const float* c, float* nc) {
  float n0 = v[4] * is[0], n1 = v[5] * is[1], n2 = v[6] * is[2];
  const float il = 1.0f / sqrtf((n0 * n0 + n1 * n1) + n2 * n2);
  n0 = n0 * il;
  n1 = n1 * il;
  n2 = n2 * il;
  float w[3];
#pragma unroll
  for (int i = 0; i < 3; i++) w[i] = (g[3 + 3 * i] * n0 + g[4 + 3 * i] * n1) + g[5 + 3 * i] * n2;
#pragma unroll
  for (int i = 0; i < 3; i++) nc[i] = (c[3 + i] * w[0] + c[6 + i] * w[1]) + c[9 + i] * w[2];
}

// Sutherland-Hodgman against the near plane (-z >= near) over the edges
// v0->v1, v1->v2, v2->v0; `K` attributes per vertex are carried along.
template <int K>
__device__ __forceinline__ int clip_near(const PV* in, PV* out, float near_) {
  int n = 0;
#pragma unroll
  for (int e = 0; e < 3; e++) {
    const PV& a = in[e];
    const PV& b = in[e == 2 ? 0 : e + 1];
    float da = (-a.a[2]) - near_, db = (-b.a[2]) - near_;
    bool ia = da >= 0.0f, ib = db >= 0.0f;
    if (ia) out[n++] = a;
    if (ia != ib) {
      float t = da / (da - db);
#pragma unroll
      for (int k = 0; k < K; k++) out[n].a[k] = a.a[k] + t * (b.a[k] - a.a[k]);
      n++;
    }
  }
  return n;
}

struct SV {  // screen-space vertex
  float x, y, z, w;
};

__device__ __forceinline__ SV project(const PV& p, float fx, float fy, const RArgs& A) {
  SV s;
  s.w = -p.a[2];
  const float iw = 1.0f / s.w;
  float nx = (fx * p.a[0]) * iw, ny = (fy * p.a[1]) * iw;
  s.z = (A.A * p.a[2] + A.An) * iw;
  s.x = (nx + 1.0f) * (0.5f * (float)A.W);
  s.y = (1.0f - ny) * (0.5f * (float)A.H);
  return s;
}

__device__ __forceinline__ float edge(float ax, float ay, float bx, float by, float px, float py) {
  return (bx - ax) * (py - ay) - (by - ay) * (px - ax);
}

// a pixel centre exactly on an edge belongs to one of the two triangles sharing it
__device__ __forceinline__ bool owns(float e, float ax, float ay, float bx, float by) {
  if (e != 0.0f) return e > 0.0f;
  float dy = by - ay, dx = bx - ax;
  return dy < 0.0f || (dy == 0.0f && dx > 0.0f);
}

// orient counter-clockwise in (x right, y down) so that area > 0; returns area (NaN or <= 0: nothing to draw)
__device__ __forceinline__ float orient(SV* s, int* ord) {
  float area = edge(s[0].x, s[0].y, s[1].x, s[1].y, s[2].x, s[2].y);
  if (area < 0.0f) {
    SV t = s[1];
    s[1] = s[2];
    s[2] = t;
    int o = ord[1];
    ord[1] = ord[2];
    ord[2] = o;
    area = edge(s[0].x, s[0].y, s[1].x, s[1].y, s[2].x, s[2].y);
  }
  return area;
}

// edge functions of pixel (px, py); false when its centre is not covered
__device__ __forceinline__ bool cover(const SV* s, int px, int py, float* e) {
  float X = (float)px + 0.5f, Y = (float)py + 0.5f;
  e[0] = edge(s[1].x, s[1].y, s[2].x, s[2].y, X, Y);
  e[1] = edge(s[2].x, s[2].y, s[0].x, s[0].y, X, Y);
  e[2] = edge(s[0].x, s[0].y, s[1].x, s[1].y, X, Y);
  return owns(e[0], s[1].x, s[1].y, s[2].x, s[2].y) && owns(e[1], s[2].x, s[2].y, s[0].x, s[0].y) &&
         owns(e[2], s[0].x, s[0].y, s[1].x, s[1].y);
}

// NDC depth of a covered pixel, interpolated linearly in screen space (ia:
// the reciprocal of the sub-triangle's doubled area)
__device__ __forceinline__ float ndc_depth(const SV* s, float ia, const float* e) {
  return ((e[0] * s[0].z + e[1] * s[1].z) + e[2] * s[2].z) * ia;
}

// visibility key of pixel (px, py), or EMPTY
__device__ __forceinline__ unsigned long long frag_key(const SV* s, float ia, int px, int py, unsigned id) {
  float e[3];
  if (!cover(s, px, py, e)) return EMPTY;
  const float z = ndc_depth(s, ia, e);
  if (!(z >= 0.0f && z <= 1.0f)) return EMPTY;
  return ((unsigned long long)__float_as_uint(z) << 32) | id;
}

__device__ __forceinline__ void bbox(const SV* s, int tx0, int ty0, int tx1, int ty1, int* b) {
  float mnx = fminf(fminf(s[0].x, s[1].x), s[2].x), mxx = fmaxf(fmaxf(s[0].x, s[1].x), s[2].x);
  float mny = fminf(fminf(s[0].y, s[1].y), s[2].y), mxy = fmaxf(fmaxf(s[0].y, s[1].y), s[2].y);
  // pixel centres x + 0.5 in [mnx, mxx]: x in [ceil(mnx - 0.5), floor(mxx - 0.5)], widened by a quarter
  // pixel on each side, far more than the rounding of the edge functions can move an edge
  b[0] = max(tx0, (int)ceilf(fmaxf(mnx, -2.0f) - 0.75f));
  b[1] = max(ty0, (int)ceilf(fmaxf(mny, -2.0f) - 0.75f));
  b[2] = min(tx1 - 1, (int)floorf(fminf(mxx, 1.0e6f) - 0.25f));
  b[3] = min(ty1 - 1, (int)floorf(fminf(mxy, 1.0e6f) - 0.25f));
}

// Blocks of BLK x BLK pixels that a queued sub-triangle cannot cover are
// skipped as a whole. An edge function as `edge` evaluates it,
// fl(fl(A * fl(Y - ay)) - fl(B * fl(X - ax))) with A = fl(bx - ax) and
// B = fl(by - ay), is monotonic in X along a row (non-increasing for B > 0)
// and in Y along a column (non-decreasing for A > 0), since every rounding
// in it is monotonic; `owns` is a threshold on it. So over a rectangle of
// pixel centres the edge is largest at one corner picked by the signs of A
// and B, and a rectangle whose corner fails an edge has no centre that
// passes it: the test drops exactly pixels the per-pixel test rejects. It
// is applied only when every coordinate is below 1e18 in magnitude, where no
// product overflows.
constexpr int BLK = 4;  // blocks of 4 x 4 pixels: a half warp scans one

__device__ __forceinline__ bool edge_may_own(const SV& a, const SV& b, int x0, int x1, int y0, int y1) {
  const int x = (b.y - a.y) > 0.0f ? x0 : x1;
  const int y = (b.x - a.x) > 0.0f ? y1 : y0;
  return owns(edge(a.x, a.y, b.x, b.y, (float)x + 0.5f, (float)y + 0.5f), a.x, a.y, b.x, b.y);
}

// false when no pixel centre of [x0, x1] x [y0, y1] is covered (edges in `cover`'s order)
__device__ __forceinline__ bool rect_may_cover(const SV* s, bool tame, int x0, int x1, int y0, int y1) {
  return !tame || (edge_may_own(s[1], s[2], x0, x1, y0, y1) && edge_may_own(s[2], s[0], x0, x1, y0, y1) &&
                   edge_may_own(s[0], s[1], x0, x1, y0, y1));
}

__device__ __forceinline__ bool tame_coords(const SV* s) {
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 3; k++) ok = ok && fabsf(s[k].x) < 1e18f && fabsf(s[k].y) < 1e18f;
  return ok;
}

// triangle t's vertices in camera space (K = 3: position only; K = 8: with
// normal and local xy); false when its geom is hidden in this environment
template <int K>
__device__ __forceinline__ bool tri_verts(const RArgs& A, int t, const float* sg, const float* sa, const float* cp,
                                          PV* v, int* geom, const float* seen = nullptr) {
  const uint32_t* ix = A.tris + 3 * (size_t)t;
  const float* v0 = A.verts + 8 * (size_t)ix[0];
  int g = (int)__float_as_uint(v0[3]);
  *geom = g;
  const float* gp = sg + 12 * g;
  const float* ap = sa + 8 * g;
  if (!(ap[3] > 0.0f)) return false;
  if (seen && seen[g] == 0.0f) return false;
  float is[3];
  if (K == 8) {
#pragma unroll
    for (int k = 0; k < 3; k++) is[k] = 1.0f / fmaxf(ap[4 + k], 1e-6f);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float* vv = A.verts + 8 * (size_t)ix[k];
    cam_xform(vv, gp, ap, cp, v[k].a);
    if (K == 8) {
      cam_normal(vv, gp, is, cp, v[k].a + 3);
      v[k].a[6] = vv[0];
      v[k].a[7] = vv[1];
    }
  }
  return true;
}

// 1 when geom g's bounding sphere may reach pixels of the tile [tx0, tx1) x
// [ty0, ty1), else 0: a camera-space box around the sphere is projected
// through its corners (x / w is monotonic in x and in w on each side) and
// widened by two pixels; a sphere reaching the near plane is always kept.
// Only skips work: a kept geom is drawn exactly as without the test.
__device__ __forceinline__ float geom_seen(const RArgs& A, int g, const float* sg, const float* sa, const float* cp,
                                           float fx, float fy, int tx0, int ty0, int tx1, int ty1) {
  const float* gp = sg + 12 * g;
  const float* ap = sa + 8 * g;
  const float sc = fmaxf(fmaxf(fabsf(ap[4]), fabsf(ap[5])), fabsf(ap[6]));
  const float r = A.radius[g] * sc * 1.001f + 1e-5f;
  const float d0 = gp[0] - cp[0], d1 = gp[1] - cp[1], d2 = gp[2] - cp[2];
  const float x = (cp[3] * d0 + cp[6] * d1) + cp[9] * d2;
  const float y = (cp[4] * d0 + cp[7] * d1) + cp[10] * d2;
  const float w = -((cp[5] * d0 + cp[8] * d1) + cp[11] * d2);
  if (!(w - r > 2.0f * A.near_)) return 1.0f;
  const float w0 = w - r, w1 = w + r;
  const float nx0 = fminf(fx * (x - r) / w0, fx * (x - r) / w1), nx1 = fmaxf(fx * (x + r) / w0, fx * (x + r) / w1);
  const float ny0 = fminf(fy * (y - r) / w0, fy * (y - r) / w1), ny1 = fmaxf(fy * (y + r) / w0, fy * (y + r) / w1);
  const float sx0 = (nx0 + 1.0f) * (0.5f * (float)A.W) - 2.0f, sx1 = (nx1 + 1.0f) * (0.5f * (float)A.W) + 2.0f;
  const float sy0 = (1.0f - ny1) * (0.5f * (float)A.H) - 2.0f, sy1 = (1.0f - ny0) * (0.5f * (float)A.H) + 2.0f;
  if (!(sx0 == sx0 && sx1 == sx1 && sy0 == sy0 && sy1 == sy1)) return 1.0f;  // NaN: keep
  const bool out = sx1 < (float)tx0 || sx0 > (float)tx1 || sy1 < (float)ty0 || sy0 > (float)ty1;
  return out ? 0.0f : 1.0f;
}

// true when all three vertices lie on the visible side of the near plane:
// clipping then returns the triangle itself, in the same order
__device__ __forceinline__ bool in_front(const PV* v, float near_) {
  return (-v[0].a[2]) - near_ >= 0.0f && (-v[1].a[2]) - near_ >= 0.0f && (-v[2].a[2]) - near_ >= 0.0f;
}

// A large sub-triangle that found the block's queue full: its warp scans it
// (warp_scan) instead of its thread alone.
struct Pend {
  float x[3], y[3], z[3];
  unsigned id;
  int b[4];
  bool on;
};

// one sub-triangle into the tile's visibility buffer: scanned by its own
// thread when its bounding box is small, else queued for the whole block to
// scan after every triangle has been set up, or, with the queue of qcap
// entries full, left in *pend for the thread's warp
template <int RT>
__device__ __forceinline__ void raster_sub(SV s0, SV s1, SV s2, unsigned id, int tx0, int ty0, int tx1, int ty1,
                                           unsigned long long* keys, float* queue, int* qn, int qcap, Pend* pend) {
  SV s[3] = {s0, s1, s2};
  int ord[3] = {0, 1, 2};
  const float area = orient(s, ord);
  if (!(area > 0.0f)) return;
  int b[4];
  bbox(s, tx0, ty0, tx1, ty1, b);
  if (b[0] > b[2] || b[1] > b[3]) return;
  const int bw = b[2] - b[0] + 1, npix = bw * (b[3] - b[1] + 1);
  if (npix > BIG_PIX) {
    const int slot = atomicAdd(qn, 1);
    float* q = queue + QWORDS * (slot < qcap ? slot : 0);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      if (slot < qcap) {
        q[k] = s[k].x;
        q[3 + k] = s[k].y;
        q[6 + k] = s[k].z;
      }
      pend->x[k] = s[k].x;
      pend->y[k] = s[k].y;
      pend->z[k] = s[k].z;
    }
    if (slot < qcap) {
      q[9] = __uint_as_float(id);
#pragma unroll
      for (int k = 0; k < 4; k++) q[10 + k] = __int_as_float(b[k]);
      return;
    }
    pend->id = id;
#pragma unroll
    for (int k = 0; k < 4; k++) pend->b[k] = b[k];
    pend->on = true;
    return;
  }
  const float ia = 1.0f / area;
  for (int py = b[1]; py <= b[3]; py++)
    for (int px = b[0]; px <= b[2]; px++) {
      const unsigned long long k = frag_key(s, ia, px, py, id);
      if (k != EMPTY) atomicMin(&keys[(py - ty0) * RT + (px - tx0)], k);
    }
}

// every lane of the warp calls it: the lanes' pending sub-triangles, one
// after another, each scanned by the 32 lanes together
template <int RT>
__device__ __forceinline__ void warp_scan(const Pend& pd, int ty0, int tx0, unsigned long long* keys) {
  unsigned m = __ballot_sync(0xffffffffu, pd.on);
  const int lane = threadIdx.x & 31;
  while (m) {
    const int src = __ffs(m) - 1;
    m &= m - 1;
    SV s[3];
#pragma unroll
    for (int k = 0; k < 3; k++)
      s[k] = SV{__shfl_sync(0xffffffffu, pd.x[k], src), __shfl_sync(0xffffffffu, pd.y[k], src),
                __shfl_sync(0xffffffffu, pd.z[k], src), 0.0f};
    const unsigned id = __shfl_sync(0xffffffffu, pd.id, src);
    int b[4];
#pragma unroll
    for (int k = 0; k < 4; k++) b[k] = __shfl_sync(0xffffffffu, pd.b[k], src);
    const float ia = 1.0f / edge(s[0].x, s[0].y, s[1].x, s[1].y, s[2].x, s[2].y);
    const int bw = b[2] - b[0] + 1, npix = bw * (b[3] - b[1] + 1);
    for (int p = lane; p < npix; p += 32) {
      const int px = b[0] + p % bw, py = b[1] + p / bw;
      const unsigned long long k = frag_key(s, ia, px, py, id);
      if (k != EMPTY) atomicMin(&keys[(py - ty0) * RT + (px - tx0)], k);
    }
  }
}

// A queued sub-triangle whose box has at most HUGE_PIX pixels, scanned by
// one warp (every lane calls it): the lanes first test the box's 4 x 4
// blocks, 32 at a time, with rect_may_cover, then scan the blocks kept, two
// at a time, a half warp each.
constexpr int HUGE_PIX = 1024;

template <int RT>
__device__ __forceinline__ void warp_blocks(const float* q, int tx0, int ty0, unsigned long long* keys) {
  const int bx0 = __float_as_int(q[10]), by0 = __float_as_int(q[11]);
  const int bx1 = __float_as_int(q[12]), by1 = __float_as_int(q[13]);
  if ((bx1 - bx0 + 1) * (by1 - by0 + 1) > HUGE_PIX) return;
  SV s[3];
#pragma unroll
  for (int k = 0; k < 3; k++) s[k] = SV{q[k], q[3 + k], q[6 + k], 0.0f};
  const float ia = 1.0f / edge(s[0].x, s[0].y, s[1].x, s[1].y, s[2].x, s[2].y);
  const unsigned id = __float_as_uint(q[9]);
  const bool tame = tame_coords(s);
  const int lane = threadIdx.x & 31;
  const int ncx = (bx1 - bx0) / BLK + 1, nb = ncx * ((by1 - by0) / BLK + 1);
  for (int base = 0; base < nb; base += 32) {
    const int j = base + lane;
    bool keep = false;
    if (j < nb) {
      const int x0 = bx0 + BLK * (j % ncx), y0 = by0 + BLK * (j / ncx);
      keep = rect_may_cover(s, tame, x0, min(x0 + BLK - 1, bx1), y0, min(y0 + BLK - 1, by1));
    }
    unsigned m = __ballot_sync(0xffffffffu, keep);
    while (m) {
      const int a = __ffs(m) - 1;
      m &= m - 1;
      const int b = m ? __ffs(m) - 1 : -1;
      if (m) m &= m - 1;
      const int mine = lane < 16 ? a : b;
      if (mine >= 0) {
        const int jj = base + mine;
        const int px = bx0 + BLK * (jj % ncx) + (lane & 3), py = by0 + BLK * (jj / ncx) + ((lane >> 2) & 3);
        if (px <= bx1 && py <= by1) {
          const unsigned long long k = frag_key(s, ia, px, py, id);
          if (k != EMPTY) atomicMin(&keys[(py - ty0) * RT + (px - tx0)], k);
        }
      }
    }
  }
}

// what the resolve needs of the sub-triangle that won a pixel: its screen
// vertices in the orientation the visibility pass used, their normal and
// local xy, the weights c[k] = (1 / doubled area) * (1 / w[k]) that turn edge
// functions into perspective-correct barycentric weights, its geom and flags
struct Resolved {
  float x[3], y[3], w[3], c[3], at[15];
  int geom;
  uint32_t flags;
};

__device__ __forceinline__ void resolve_setup(const RArgs& A, unsigned id, const float* sg, const float* sa,
                                              const float* cp, float fx, float fy, Resolved& R) {
  const int t = (int)(id >> 1), sub = (int)(id & 1u);
  PV v[3];
  tri_verts<8>(A, t, sg, sa, cp, v, &R.geom);
  PV a0, a1, a2;
  if (in_front(v, A.near_)) {
    a0 = v[0];
    a1 = v[1];
    a2 = v[2];
  } else {
    PV poly[4];
    clip_near<8>(v, poly, A.near_);
    a0 = poly[0];
    a1 = sub ? poly[2] : poly[1];
    a2 = sub ? poly[3] : poly[2];
  }
  SV s[3] = {project(a0, fx, fy, A), project(a1, fx, fy, A), project(a2, fx, fy, A)};
  float area = edge(s[0].x, s[0].y, s[1].x, s[1].y, s[2].x, s[2].y);
  if (area < 0.0f) {  // the orientation the visibility pass used
    const SV ts = s[1];
    s[1] = s[2];
    s[2] = ts;
    const PV ta = a1;
    a1 = a2;
    a2 = ta;
    area = edge(s[0].x, s[0].y, s[1].x, s[1].y, s[2].x, s[2].y);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    R.x[k] = s[k].x;
    R.y[k] = s[k].y;
    R.w[k] = s[k].w;
  }
#pragma unroll
  for (int j = 0; j < 5; j++) {
    R.at[j] = a0.a[3 + j];
    R.at[5 + j] = a1.a[3 + j];
    R.at[10 + j] = a2.a[3 + j];
  }
  const float ia = 1.0f / area;
#pragma unroll
  for (int k = 0; k < 3; k++) R.c[k] = ia * (1.0f / s[k].w);
  R.flags = __float_as_uint(A.verts[8 * (size_t)A.tris[3 * (size_t)t] + 7]);
}

template <int RT, int NT>
__global__ void __launch_bounds__(NT, RT == 64 ? 3 : 1) render_kernel(RArgs A) {
  constexpr int QCAP = 2 * NT;  // queue entries for the image's large sub-triangles
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* keys = (unsigned long long*)smem;
  float* queue = (float*)(keys + RT * RT);
  float* sg = queue + QCAP * QWORDS;  // this env's geom poses
  float* sa = sg + 12 * A.ngeom;      // and appearance
  float* cp = sa + 8 * A.ngeom;       // the view's camera pose
  float* seen = cp + 12;              // per geom: may reach this tile
  __shared__ int qn, tri_next, q_next;  // queue length; next triangle and next queue entry to hand out
  const int tid = threadIdx.x;
  const int tiles = A.tiles_x * A.tiles_y;
  const long long items = (long long)A.nenv * A.nview * tiles;

  for (long long item = blockIdx.x; item < items; item += gridDim.x) {
    const int img = (int)(item / tiles), tile = (int)(item % tiles);
    const int env = img / A.nview, view = img % A.nview;
    const int tx0 = (tile % A.tiles_x) * RT, ty0 = (tile / A.tiles_x) * RT;
    const int tx1 = min(tx0 + RT, A.W), ty1 = min(ty0 + RT, A.H);
    const float* vw = A.views + 16 * view;
    const int cam = (int)vw[0];
    const float fx = vw[1], fy = vw[2];
    for (int i = tid; i < 12 * A.ngeom; i += NT) sg[i] = A.geoms[(size_t)env * A.ngeom * 12 + i];
    for (int i = tid; i < 8 * A.ngeom; i += NT) sa[i] = A.app[(size_t)env * A.ngeom * 8 + i];
    if (tid < 12) cp[tid] = cam >= 0 ? A.cams[((size_t)env * A.ncam + cam) * 12 + tid] : vw[4 + tid];
    for (int i = tid; i < RT * RT; i += NT) keys[i] = EMPTY;
    if (tid == 0) {
      qn = 0;
      tri_next = 0;
      q_next = 0;
    }
    __syncthreads();
    for (int g = tid; g < A.ngeom; g += NT) seen[g] = geom_seen(A, g, sg, sa, cp, fx, fy, tx0, ty0, tx1, ty1);
    __syncthreads();

    // ---- visibility: no thread waits for another while the triangles are
    // set up and the small ones scanned; the large ones, queued meanwhile,
    // are scanned afterwards (the visibility keys are a minimum: the order of
    // the updates does not matter). Warps take 32 consecutive triangles at a
    // time, so that none waits at the barrier below while others still have
    // triangles left.
    const int lane = tid & 31;
    for (;;) {
      int base = 0;
      if (lane == 0) base = atomicAdd(&tri_next, 32);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= A.ntri) break;
      const int t = base + lane;
      // the triangle's one or two sub-triangles (two when the near plane clips it to a quad)
      SV a[3], c[3];
      int nsub = 0;
      PV v[3];
      int geom;
      if (t < A.ntri && tri_verts<3>(A, t, sg, sa, cp, v, &geom, seen)) {
        if (in_front(v, A.near_)) {
#pragma unroll
          for (int k = 0; k < 3; k++) a[k] = project(v[k], fx, fy, A);
          nsub = 1;
        } else {
          PV poly[4];
          const int n = clip_near<3>(v, poly, A.near_);
          if (n >= 3) {
            a[0] = project(poly[0], fx, fy, A);
            a[1] = project(poly[1], fx, fy, A);
            a[2] = project(poly[2], fx, fy, A);
            nsub = 1;
            if (n == 4) {
              c[0] = a[0];
              c[1] = a[2];
              c[2] = project(poly[3], fx, fy, A);
              nsub = 2;
            }
          }
        }
      }
      Pend pd;
      pd.on = false;
      if (nsub >= 1) raster_sub<RT>(a[0], a[1], a[2], 2u * t, tx0, ty0, tx1, ty1, keys, queue, &qn, QCAP, &pd);
      warp_scan<RT>(pd, ty0, tx0, keys);
      pd.on = false;
      if (nsub >= 2) raster_sub<RT>(c[0], c[1], c[2], 2u * t + 1u, tx0, ty0, tx1, ty1, keys, queue, &qn, QCAP, &pd);
      warp_scan<RT>(pd, ty0, tx0, keys);
    }
    __syncthreads();
    // the queued sub-triangles: those with boxes over HUGE_PIX pixels (a plane
    // crossing the view) by the whole block, pixel p of the box to thread
    // p mod NT, stepping coordinates by NT pixels at a time; the others (long
    // thin sides of capsules and cylinders, mostly) a warp each (warp_blocks)
    const int nq = min(qn, QCAP);
    for (int e = 0; e < nq; e++) {
      const float* q = queue + QWORDS * e;
      const int bx0 = __float_as_int(q[10]), by0 = __float_as_int(q[11]);
      const int bx1 = __float_as_int(q[12]), by1 = __float_as_int(q[13]);
      const int bw = bx1 - bx0 + 1;
      if (bw * (by1 - by0 + 1) <= HUGE_PIX) continue;
      SV s[3];
      for (int k = 0; k < 3; k++) s[k] = SV{q[k], q[3 + k], q[6 + k], 0.0f};
      const float ia = 1.0f / edge(s[0].x, s[0].y, s[1].x, s[1].y, s[2].x, s[2].y);
      const unsigned id = __float_as_uint(q[9]);
      const int dy = NT / bw, dx = NT - dy * bw;
      int py = by0 + tid / bw, px = bx0 + (tid - (tid / bw) * bw);
      while (py <= by1) {
        const unsigned long long k = frag_key(s, ia, px, py, id);
        if (k != EMPTY) atomicMin(&keys[(py - ty0) * RT + (px - tx0)], k);
        px += dx;
        py += dy;
        if (px > bx1) {
          px -= bw;
          py++;
        }
      }
    }
    for (;;) {  // the other entries, a warp each, handed out one at a time
      int e = 0;
      if (lane == 0) e = atomicAdd(&q_next, 1);
      e = __shfl_sync(0xffffffffu, e, 0);
      if (e >= nq) break;
      warp_blocks<RT>(queue + QWORDS * e, tx0, ty0, keys);
    }
    __syncthreads();  // every fragment is in before the resolve reads the keys

    // ---- resolve and shade: a thread keeps the set-up of the last triangle
    // it resolved, which the next pixels it visits mostly share (128 x 128
    // tiles; the 64 x 64 kernel, held to 80 registers for three blocks an SM,
    // sets up every pixel's triangle afresh: 2.89 against 3.14 ms a 4096-image
    // frame, keeping the set-up across pixels cost it spills)
    Resolved R;
    unsigned rid = ~0u;  // no sub-triangle id: ids are 2 * triangle + sub with fewer than 2^30 triangles
    const int tw = tx1 - tx0, npx = tw * (ty1 - ty0);
    for (int p = tid; p < npx; p += NT) {
      const int px = tx0 + p % tw, py = ty0 + p / tw;
      const unsigned long long key = keys[(py - ty0) * RT + (px - tx0)];
      const size_t o = ((size_t)img * A.H + py) * A.W + px;
      uchar4 c = make_uchar4(184, 199, 219, 255);  // the clear colour (0.72, 0.78, 0.86) in RGBA8
      float d = A.far_;
      int sgid = -1;
      if (key != EMPTY) {
        const unsigned id = (unsigned)(key & 0xffffffffu);
        if (RT == 64 || id != rid) {
          rid = id;
          resolve_setup(A, id, sg, sa, cp, fx, fy, R);
        }
        const SV s[3] = {{R.x[0], R.y[0], 0.0f, R.w[0]}, {R.x[1], R.y[1], 0.0f, R.w[1]},
                         {R.x[2], R.y[2], 0.0f, R.w[2]}};
        float e[3];
        cover(s, px, py, e);
        float q[3];
#pragma unroll
        for (int k = 0; k < 3; k++) q[k] = e[k] * R.c[k];
        const float iQ = 1.0f / ((q[0] + q[1]) + q[2]);
        float at[6];  // normal xyz, local xy, linear depth
#pragma unroll
        for (int j = 0; j < 5; j++) at[j] = ((q[0] * R.at[j] + q[1] * R.at[5 + j]) + q[2] * R.at[10 + j]) * iQ;
        at[5] = ((q[0] * s[0].w + q[1] * s[1].w) + q[2] * s[2].w) * iQ;
        const float il = 1.0f / sqrtf((at[0] * at[0] + at[1] * at[1]) + at[2] * at[2]);
        const float n0 = at[0] * il, n1 = at[1] * il, n2 = at[2] * il;
        const float head = fabsf(n2);
        const float keyl = fmaxf((n0 * A.L0 + n1 * A.L1) + n2 * A.L2, 0.0f);
        float shade = (0.25f + 0.5f * head) + 0.35f * keyl;
        if (R.flags & 1u) {
          const int cx = (int)floorf(at[3] * 4.0f), cy = (int)floorf(at[4] * 4.0f);  // checker squares of 0.25
          shade = shade * (((cx + cy) & 1) ? 0.8f : 1.05f);
        }
        const int geom = R.geom;
        const float* ap = sa + 8 * geom;
        unsigned char u[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const float x = fminf(fmaxf(ap[k] * shade, 0.0f), 1.0f);
          u[k] = (unsigned char)(x * 255.0f + 0.5f);
        }
        c = make_uchar4(u[0], u[1], u[2], 255);
        d = at[5];
        sgid = geom;
      }
      ((uchar4*)A.rgba)[o] = c;
      A.depth[o] = d;
      A.seg[o] = sgid;
    }
    __syncthreads();
  }
}

size_t render_smem(int rt, int nt, int ngeom) {
  return sizeof(unsigned long long) * rt * rt + sizeof(float) * (2 * (size_t)nt * QWORDS + 21 * (size_t)ngeom + 12);
}

int rfail(int code, const std::string& msg) {
  pg::internal_set_error(msg);
  return code;
}

#define RCK(x)                                                                                      \
  do {                                                                                              \
    cudaError_t _e = (x);                                                                           \
    if (_e != cudaSuccess) return rfail(PG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); \
  } while (0)

}  // namespace

constexpr int MAX_VIEWS = 4096;  // views per env (the kernel indexes images as 32-bit ints)
constexpr int RCHUNKS = 8;  // host-buffer frames: at most this many chunks, whose copies back overlap the next chunk's rendering

struct pg_renderer {
  int device = 0;
  cudaStream_t stream = nullptr, copy_stream = nullptr;
  cudaEvent_t done[RCHUNKS] = {};
  int nvert = 0, ntri = 0, ngeom = 0, ncam = 0, nview = 0, W = 0, H = 0, sms = 0, per_sm = 0;
  int rt = 64, nt = 256;  // tile edge and threads per block
  float uni[8] = {};
  float *verts = nullptr, *views = nullptr, *radius = nullptr;
  uint32_t* tris = nullptr;
  std::vector<float> base_app;
  // per-call staging, grown on demand
  size_t cap_env = 0;
  float *d_geoms = nullptr, *d_cams = nullptr, *d_app = nullptr;
  uint8_t* d_rgba = nullptr;
  float* d_depth = nullptr;
  int32_t* d_seg = nullptr;
  size_t default_app_env = 0;  // envs the default appearance in d_app covers
};

namespace {

void free_staging(pg_renderer* r) {
  for (void* p : {(void*)r->d_geoms, (void*)r->d_cams, (void*)r->d_app, (void*)r->d_rgba, (void*)r->d_depth,
                  (void*)r->d_seg})
    if (p) cudaFree(p);
  r->d_geoms = r->d_cams = r->d_app = r->d_depth = nullptr;
  r->d_rgba = nullptr;
  r->d_seg = nullptr;
  r->cap_env = 0;
  r->default_app_env = 0;
}

int launch(pg_renderer* r, int64_t nenv, const float* geoms, const float* cams, const float* app, uint8_t* rgba,
           float* depth, int32_t* seg) {
  if (nenv == 0) return PG_OK;
  RArgs a;
  a.verts = r->verts;
  a.radius = r->radius;
  a.tris = r->tris;
  a.ntri = r->ntri;
  a.ngeom = r->ngeom;
  a.ncam = r->ncam;
  a.nview = r->nview;
  a.views = r->views;
  a.W = r->W;
  a.H = r->H;
  a.tiles_x = (r->W + r->rt - 1) / r->rt;
  a.tiles_y = (r->H + r->rt - 1) / r->rt;
  a.near_ = r->uni[0];
  a.far_ = r->uni[1];
  a.A = r->uni[2];
  a.An = r->uni[3];
  a.L0 = r->uni[4];
  a.L1 = r->uni[5];
  a.L2 = r->uni[6];
  a.geoms = geoms;
  a.cams = cams;
  a.app = app;
  a.nenv = (int)nenv;
  a.rgba = rgba;
  a.depth = depth;
  a.seg = seg;
  long long items = nenv * r->nview * (long long)a.tiles_x * a.tiles_y;
  long long blocks = std::min<long long>(items, (long long)r->sms * r->per_sm);
  const size_t smem = render_smem(r->rt, r->nt, r->ngeom);
  if (r->rt == 128)
    render_kernel<128, 512><<<(unsigned)blocks, 512, smem, r->stream>>>(a);
  else
    render_kernel<64, 256><<<(unsigned)blocks, 256, smem, r->stream>>>(a);
  RCK(cudaGetLastError());
  return PG_OK;
}

}  // namespace

extern "C" {

int pg_render_create(const float* vertices, int64_t nvert, const uint32_t* triangles, int64_t ntri, int64_t ngeom,
                     int64_t ncam, const float* views, int64_t nview, const float* base_appearance, int64_t width,
                     int64_t height, const float* uniforms, int device, pg_renderer** out) {
  if (!out || !views || !base_appearance || !uniforms) return rfail(PG_ERR_INVALID, "NULL argument");
  *out = nullptr;
  if (nvert < 0 || ntri < 0 || ngeom < 0 || ncam < 0 || nview < 1 || width < 1 || height < 1)
    return rfail(PG_ERR_INVALID, "renderer sizes out of range");
  if ((nvert > 0 && !vertices) || (ntri > 0 && !triangles)) return rfail(PG_ERR_INVALID, "NULL mesh");
  if (ntri >= (1ll << 30) || nvert >= (1ll << 31) || width > 16384 || height > 16384 || ngeom >= (1 << 20) ||
      nview > MAX_VIEWS)
    return rfail(PG_ERR_UNSUPPORTED, "scene or image too large");
  for (int64_t i = 0; i < 3 * ntri; i++)
    if ((int64_t)triangles[i] >= nvert) return rfail(PG_ERR_INVALID, "triangle index out of range");
  for (int64_t i = 0; i < nvert; i++) {
    uint32_t g;
    std::memcpy(&g, vertices + 8 * i + 3, 4);
    if ((int64_t)g >= ngeom) return rfail(PG_ERR_INVALID, "vertex geom id out of range");
  }
  for (int64_t v = 0; v < nview; v++) {
    float c = views[16 * v];
    if (!(c == -1.0f || (c >= 0.0f && c < (float)ncam && c == (float)(int)c)))
      return rfail(PG_ERR_INVALID, "view refers to a camera the scene does not have");
  }
  if (!(uniforms[0] > 0.0f) || !(uniforms[1] > uniforms[0])) return rfail(PG_ERR_INVALID, "need 0 < near < far");
  const size_t smem_limit = 227 * 1024;
  // 128 x 128 tiles for images above 64 pixels (fewer tiles set up the same
  // triangles: Ant at 256 x 256, 139k frames/s against 117k with 64 x 64
  // tiles), 64 x 64 tiles, three blocks an SM, for images up to 64 pixels.
  // PIPPIN_RENDER_TILE=64 or 128 overrides the choice.
  const char* tile_env = std::getenv("PIPPIN_RENDER_TILE");
  const int want = tile_env ? std::atoi(tile_env) : (width > 64 || height > 64 ? 128 : 64);
  const bool large = want == 128 && render_smem(128, 512, (int)ngeom) <= smem_limit;
  const size_t smem = large ? render_smem(128, 512, (int)ngeom) : render_smem(64, 256, (int)ngeom);
  if (smem > smem_limit) return rfail(PG_ERR_UNSUPPORTED, "too many geoms for the renderer's shared memory");
  pg_renderer* r = new pg_renderer();
  r->device = device;
  r->nvert = (int)nvert;
  r->ntri = (int)ntri;
  r->ngeom = (int)ngeom;
  r->ncam = (int)ncam;
  r->nview = (int)nview;
  r->W = (int)width;
  r->H = (int)height;
  r->rt = large ? 128 : 64;
  r->nt = large ? 512 : 256;
  std::memcpy(r->uni, uniforms, sizeof(r->uni));
  r->base_app.assign(base_appearance, base_appearance + 8 * ngeom);
  auto bail = [&](int rc) {
    pg_render_destroy(r);
    return rc;
  };
#define RCKB(x)                                                                                   \
  do {                                                                                            \
    cudaError_t _e = (x);                                                                         \
    if (_e != cudaSuccess) return bail(rfail(PG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e))); \
  } while (0)
  RCKB(cudaSetDevice(device));
  RCKB(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking));
  RCKB(cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking));
  for (cudaEvent_t& e : r->done) RCKB(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  RCKB(cudaMalloc(&r->verts, sizeof(float) * 8 * std::max<int64_t>(nvert, 1)));
  RCKB(cudaMalloc(&r->tris, sizeof(uint32_t) * 3 * std::max<int64_t>(ntri, 1)));
  RCKB(cudaMalloc(&r->views, sizeof(float) * 16 * nview));
  if (nvert) RCKB(cudaMemcpy(r->verts, vertices, sizeof(float) * 8 * nvert, cudaMemcpyHostToDevice));
  if (ntri) RCKB(cudaMemcpy(r->tris, triangles, sizeof(uint32_t) * 3 * ntri, cudaMemcpyHostToDevice));
  RCKB(cudaMemcpy(r->views, views, sizeof(float) * 16 * nview, cudaMemcpyHostToDevice));
  {
    std::vector<float> rad(std::max<int64_t>(ngeom, 1), 0.0f);
    for (int64_t i = 0; i < nvert; i++) {
      uint32_t g;
      std::memcpy(&g, vertices + 8 * i + 3, 4);
      const float* p = vertices + 8 * i;
      rad[g] = std::max(rad[g], std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]));
    }
    RCKB(cudaMalloc(&r->radius, sizeof(float) * rad.size()));
    RCKB(cudaMemcpy(r->radius, rad.data(), sizeof(float) * rad.size(), cudaMemcpyHostToDevice));
  }
  RCKB(cudaDeviceGetAttribute(&r->sms, cudaDevAttrMultiProcessorCount, device));
  if (large) {
    RCKB(cudaFuncSetAttribute(render_kernel<128, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    RCKB(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r->per_sm, render_kernel<128, 512>, 512, smem));
  } else {
    RCKB(cudaFuncSetAttribute(render_kernel<64, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    RCKB(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r->per_sm, render_kernel<64, 256>, 256, smem));
  }
  if (r->per_sm < 1) return bail(rfail(PG_ERR_UNSUPPORTED, "renderer block does not fit on an SM"));
#undef RCKB
  *out = r;
  return PG_OK;
}

int pg_render_destroy(pg_renderer* r) {
  if (!r) return PG_OK;
  cudaSetDevice(r->device);
  if (r->stream) cudaStreamSynchronize(r->stream);
  free_staging(r);
  if (r->verts) cudaFree(r->verts);
  if (r->tris) cudaFree(r->tris);
  if (r->views) cudaFree(r->views);
  if (r->radius) cudaFree(r->radius);
  if (r->copy_stream) cudaStreamSynchronize(r->copy_stream);
  for (cudaEvent_t& e : r->done)
    if (e) cudaEventDestroy(e);
  if (r->copy_stream) cudaStreamDestroy(r->copy_stream);
  if (r->stream) cudaStreamDestroy(r->stream);
  delete r;
  return PG_OK;
}

int pg_render_frames(pg_renderer* r, int64_t nenv, const float* geoms, size_t geoms_len, const float* cams,
                     size_t cams_len, const float* appearance, size_t appearance_len, uint8_t* rgba, float* depth,
                     int32_t* seg) {
  if (!r) return rfail(PG_ERR_INVALID, "NULL renderer");
  if (nenv < 0 || nenv > (1 << 24)) return rfail(PG_ERR_INVALID, "nenv out of range");
  if (nenv * r->nview >= (1ll << 31)) return rfail(PG_ERR_INVALID, "nenv x views must stay below 2^31 images");
  const size_t ne = (size_t)nenv;
  if (geoms_len != ne * r->ngeom * 12 || cams_len != ne * r->ncam * 12)
    return rfail(PG_ERR_LENGTH, "expected " + std::to_string(ne * r->ngeom) + " geom and " +
                                    std::to_string(ne * r->ncam) + " camera poses");
  if (appearance && appearance_len != ne * r->ngeom * 8)
    return rfail(PG_ERR_LENGTH, "expected " + std::to_string(ne * r->ngeom) + " appearance entries");
  if (nenv == 0) return PG_OK;
  if ((r->ngeom && !geoms) || (r->ncam && !cams) || !rgba || !depth || !seg) return rfail(PG_ERR_INVALID, "NULL buffer");
  RCK(cudaSetDevice(r->device));
  const size_t px = ne * r->nview * (size_t)r->W * r->H;
  if (ne > r->cap_env) {
    free_staging(r);
    RCK(cudaMalloc(&r->d_geoms, sizeof(float) * 12 * std::max<size_t>(ne * r->ngeom, 1)));
    RCK(cudaMalloc(&r->d_cams, sizeof(float) * 12 * std::max<size_t>(ne * r->ncam, 1)));
    RCK(cudaMalloc(&r->d_app, sizeof(float) * 8 * std::max<size_t>(ne * r->ngeom, 1)));
    RCK(cudaMalloc(&r->d_rgba, 4 * px));
    RCK(cudaMalloc(&r->d_depth, 4 * px));
    RCK(cudaMalloc(&r->d_seg, 4 * px));
    r->cap_env = ne;
  }
  cudaStream_t s = r->stream;
  if (r->ngeom) RCK(cudaMemcpyAsync(r->d_geoms, geoms, sizeof(float) * 12 * ne * r->ngeom, cudaMemcpyHostToDevice, s));
  if (r->ncam) RCK(cudaMemcpyAsync(r->d_cams, cams, sizeof(float) * 12 * ne * r->ncam, cudaMemcpyHostToDevice, s));
  if (appearance) {
    RCK(cudaMemcpyAsync(r->d_app, appearance, sizeof(float) * 8 * ne * r->ngeom, cudaMemcpyHostToDevice, s));
    r->default_app_env = 0;
  } else if (r->default_app_env < ne && r->ngeom) {
    std::vector<float> def(8 * ne * r->ngeom);
    for (size_t e = 0; e < ne; e++) std::copy(r->base_app.begin(), r->base_app.end(), def.begin() + 8 * e * r->ngeom);
    RCK(cudaMemcpyAsync(r->d_app, def.data(), sizeof(float) * def.size(), cudaMemcpyHostToDevice, s));
    RCK(cudaStreamSynchronize(s));  // `def` is pageable and about to go
    r->default_app_env = ne;
  }
  // every chunk's kernel is queued first, then each chunk's images go back on
  // the copy stream once its kernel is done, overlapping the later chunks
  const size_t per_env = (size_t)r->nview * r->W * r->H;
  // as many chunks as keep at least two full waves of blocks in each (fewer
  // leave a chunk's last wave part-empty: 64 x 64 Ant frames lost 12% at 8)
  const long long tiles = (long long)((r->W + r->rt - 1) / r->rt) * ((r->H + r->rt - 1) / r->rt);
  const long long wave = (long long)r->sms * r->per_sm;
  const int nch = (int)std::max<long long>(1, std::min<long long>(RCHUNKS, (long long)ne * r->nview * tiles / (2 * wave)));
  size_t bounds[RCHUNKS + 1];
  for (int k = 0; k <= RCHUNKS; k++) bounds[k] = k <= nch ? ne * k / nch : ne;
  for (int k = 0; k < RCHUNKS; k++) {
    const size_t e0 = bounds[k], e1 = bounds[k + 1];
    if (e1 == e0) continue;
    int rc = launch(r, (int64_t)(e1 - e0), r->d_geoms + 12 * e0 * r->ngeom, r->d_cams + 12 * e0 * r->ncam,
                    r->d_app + 8 * e0 * r->ngeom, r->d_rgba + 4 * e0 * per_env, r->d_depth + e0 * per_env,
                    r->d_seg + e0 * per_env);
    if (rc) return rc;
    RCK(cudaEventRecord(r->done[k], s));
  }
  cudaStream_t cs = r->copy_stream;
  for (int k = 0; k < RCHUNKS; k++) {
    const size_t e0 = bounds[k], e1 = bounds[k + 1];
    if (e1 == e0) continue;
    const size_t o = e0 * per_env, cnt = (e1 - e0) * per_env;
    RCK(cudaStreamWaitEvent(cs, r->done[k], 0));
    RCK(cudaMemcpyAsync(rgba + 4 * o, r->d_rgba + 4 * o, 4 * cnt, cudaMemcpyDeviceToHost, cs));
    RCK(cudaMemcpyAsync(depth + o, r->d_depth + o, 4 * cnt, cudaMemcpyDeviceToHost, cs));
    RCK(cudaMemcpyAsync(seg + o, r->d_seg + o, 4 * cnt, cudaMemcpyDeviceToHost, cs));
  }
  RCK(cudaStreamSynchronize(cs));
  RCK(cudaStreamSynchronize(s));
  return PG_OK;
}

int pg_render_frames_device(pg_renderer* r, int64_t nenv, const float* geoms, const float* cams,
                            const float* appearance, uint8_t* rgba, float* depth, int32_t* seg) {
  if (!r) return rfail(PG_ERR_INVALID, "NULL renderer");
  if (nenv < 0 || nenv > (1 << 24)) return rfail(PG_ERR_INVALID, "nenv out of range");
  if (nenv * r->nview >= (1ll << 31)) return rfail(PG_ERR_INVALID, "nenv x views must stay below 2^31 images");
  if (nenv == 0) return PG_OK;
  if ((r->ngeom && (!geoms || !appearance)) || (r->ncam && !cams) || !rgba || !depth || !seg)
    return rfail(PG_ERR_INVALID, "NULL buffer");
  RCK(cudaSetDevice(r->device));
  return launch(r, nenv, geoms, cams, appearance, rgba, depth, seg);
}

void* pg_render_stream(const pg_renderer* r) { return r ? (void*)r->stream : nullptr; }

int pg_render_synchronize(pg_renderer* r) {
  if (!r) return rfail(PG_ERR_INVALID, "NULL renderer");
  RCK(cudaSetDevice(r->device));
  RCK(cudaStreamSynchronize(r->stream));
  return PG_OK;
}

}  // extern "C"
