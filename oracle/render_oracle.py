"""Oracle (test infrastructure only): numpy restatement of the batched
rasteriser, evaluated in IEEE single precision with every product and sum
rounded on its own, in the same order as the CUDA kernel.

Only tests/ and ``__graft_entry__.smoke()`` use this module, as the checker;
the product package never imports it.

What it restates:
- the vertex stage of crates/pippin-render/src/render.metal:67-109: geom
  scale, geom pose, camera pose (scene camera or fixed view), the projection
  (f / aspect, f, A = far / (near - far)) and the normal transform;
- the fixed-function stages Metal runs between the two shaders, which the
  reference does not spell out and this restatement defines: clipping at the
  near plane (Sutherland-Hodgman, fan-triangulated), the viewport transform,
  coverage at pixel centres by edge functions with a top-left ownership rule
  for centres on an edge, the depth test `Less` with depth cleared to 1
  (crates/pippin-render/src/lib.rs:133-136, 286-290) over triangles in draw
  order, and perspective-correct interpolation;
- the fragment stage (render.metal:111-128: headlight, key light, checker
  on planes) and the readback to RGBA8 / linear depth / segmentation
  (render.metal:130-145) with the clear values of lib.rs:275-279.

Parity with the reference's own images is unpinned: Metal's rasteriser and
its interpolation are hardware behaviour that cannot run here. The
reference's analytic tests (crates/pippin-render/tests/geometry.rs) pin
silhouettes, depths and per-env appearance instead.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32
EMPTY = np.uint64(0xFFFFFFFFFFFFFFFF)
CLEAR = np.array([184, 199, 219, 255], np.uint8)


def _vertex_stage(V, geom_pose, app, cam):
    """Camera-space position, normal and local xy of vertices V (n, 8) under
    per-vertex geom poses (n, 12) and appearance (n, 8); cam (12,)."""
    g, a, c = geom_pose, app, cam
    p = [V[:, k] * a[:, 4 + k] for k in range(3)]
    w = [((g[:, 3 + 3 * i] * p[0] + g[:, 4 + 3 * i] * p[1]) + g[:, 5 + 3 * i] * p[2]) + g[:, i] for i in range(3)]
    d = [w[i] - c[i] for i in range(3)]
    pc = [(c[3 + i] * d[0] + c[6 + i] * d[1]) + c[9 + i] * d[2] for i in range(3)]
    # normals: times the reciprocal scale (the inverse transpose of a diagonal scale), then unit length
    n = [V[:, 4 + k] * (f32(1) / np.fmax(a[:, 4 + k], f32(1e-6))) for k in range(3)]
    il = f32(1) / np.sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2])
    n = [n[k] * il for k in range(3)]
    nw = [(g[:, 3 + 3 * i] * n[0] + g[:, 4 + 3 * i] * n[1]) + g[:, 5 + 3 * i] * n[2] for i in range(3)]
    nc = [(c[3 + i] * nw[0] + c[6 + i] * nw[1]) + c[9 + i] * nw[2] for i in range(3)]
    return np.stack(pc + nc + [V[:, 0], V[:, 1]], axis=1).astype(f32)


def _clip_near(P, near):
    """P (T, 3, 8) -> polygons (T, 4, 8) and vertex counts, clipped to
    -z >= near over the edges v0->v1, v1->v2, v2->v0."""
    T = P.shape[0]
    out = np.zeros((T, 4, 8), f32)
    cnt = np.zeros(T, np.int64)
    rows = np.arange(T)
    for e in range(3):
        a, b = P[:, e], P[:, (e + 1) % 3]
        da = (-a[:, 2]) - near
        db = (-b[:, 2]) - near
        ia, ib = da >= 0, db >= 0
        r = rows[ia]
        out[r, cnt[r]] = a[r]
        cnt[r] += 1
        r = rows[ia != ib]
        t = da[r] / (da[r] - db[r])
        out[r, cnt[r]] = a[r] + t[:, None] * (b[r] - a[r])
        cnt[r] += 1
    return out, cnt


def _project(p, fx, fy, A, An, W, H):
    w = -p[..., 2]
    iw = f32(1) / w
    nx = (fx * p[..., 0]) * iw
    ny = (fy * p[..., 1]) * iw
    z = (A * p[..., 2] + An) * iw
    x = (nx + f32(1)) * (f32(0.5) * f32(W))
    y = (f32(1) - ny) * (f32(0.5) * f32(H))
    return x, y, z, w


def _edge(ax, ay, bx, by, px, py):
    return (bx - ax) * (py - ay) - (by - ay) * (px - ax)


def _owns(e, ax, ay, bx, by):
    dy, dx = by - ay, bx - ax
    return np.where(e != 0, e > 0, (dy < 0) | ((dy == 0) & (dx > 0)))


def render_image(verts, tris, view, uni, W, H, geoms, app, cams):
    """One image. verts (n, 8) float32 (geom, flags as u32 bits), tris (m, 3),
    view (16,), uni (8,), geoms (ngeom, 12), app (ngeom, 8), cams (ncam, 12).
    Returns rgba (H, W, 4) u8, depth (H, W) f32, seg (H, W) i32."""
    verts = np.asarray(verts, f32)
    vb = verts.view(np.uint32)
    near, far, A, An, L0, L1, L2 = (f32(x) for x in uni[:7])
    cam_i = int(view[0])
    cam = (cams[cam_i] if cam_i >= 0 else view[4:16]).astype(f32)
    fx, fy = f32(view[1]), f32(view[2])
    rgba = np.tile(CLEAR, (H, W, 1))
    depth = np.full((H, W), far, f32)
    seg = np.full((H, W), -1, np.int32)
    if len(tris) == 0:
        return rgba, depth, seg
    tg = vb[tris[:, 0], 3].astype(np.int64)  # each triangle's geom
    shown = app[tg, 3] > 0
    tid = np.nonzero(shown)[0]
    if len(tid) == 0:
        return rgba, depth, seg
    idx = tris[tid].reshape(-1)
    gv = np.repeat(tg[tid], 3)
    P = _vertex_stage(verts[idx], geoms[gv].astype(f32), app[gv].astype(f32), cam).reshape(-1, 3, 8)
    poly, cnt = _clip_near(P, near)
    # sub-triangles (poly[0], poly[1 + sub], poly[2 + sub]), oriented so that area > 0
    subs = []
    for sub in (0, 1):
        ok = cnt >= 3 + sub
        order = np.tile(np.array([0, 1 + sub, 2 + sub]), (len(tid), 1))
        with np.errstate(all="ignore"):  # unused polygon slots hold zeros
            x, y, z, w = _project(poly, fx, fy, A, An, W, H)  # (T, 4)
        sel = lambda arr: np.take_along_axis(arr, order, axis=1)  # noqa: E731
        sx, sy = sel(x), sel(y)
        area = _edge(sx[:, 0], sy[:, 0], sx[:, 1], sy[:, 1], sx[:, 2], sy[:, 2])
        flip = area < 0
        order[flip] = order[flip][:, [0, 2, 1]]
        sx, sy, sz, sw = sel(x), sel(y), sel(z), sel(w)
        area = _edge(sx[:, 0], sy[:, 0], sx[:, 1], sy[:, 1], sx[:, 2], sy[:, 2])
        ok &= area > 0
        subs.append(dict(ok=ok, order=order, x=sx, y=sy, z=sz, w=sw, area=area))
    # visibility: per pixel the minimum of (depth bits << 32 | 2 * triangle + sub)
    PY, PX = np.mgrid[0:H, 0:W]
    X = PX.reshape(-1).astype(f32) + f32(0.5)
    Y = PY.reshape(-1).astype(f32) + f32(0.5)
    best = np.full(H * W, EMPTY, np.uint64)
    for sub, S in enumerate(subs):
        rows = np.nonzero(S["ok"])[0]
        for c0 in range(0, len(rows), max(1, 4_000_000 // (H * W))):
            r = rows[c0:c0 + max(1, 4_000_000 // (H * W))]
            x, y, z = S["x"][r][:, :, None], S["y"][r][:, :, None], S["z"][r][:, :, None]
            area = S["area"][r][:, None]
            e0 = _edge(x[:, 1], y[:, 1], x[:, 2], y[:, 2], X, Y)
            e1 = _edge(x[:, 2], y[:, 2], x[:, 0], y[:, 0], X, Y)
            e2 = _edge(x[:, 0], y[:, 0], x[:, 1], y[:, 1], X, Y)
            inside = (_owns(e0, x[:, 1], y[:, 1], x[:, 2], y[:, 2]) & _owns(e1, x[:, 2], y[:, 2], x[:, 0], y[:, 0])
                      & _owns(e2, x[:, 0], y[:, 0], x[:, 1], y[:, 1]))
            with np.errstate(all="ignore"):
                zz = ((e0 * z[:, 0] + e1 * z[:, 1]) + e2 * z[:, 2]) * (f32(1) / area)
            inside &= (zz >= 0) & (zz <= 1)
            ids = (2 * tid[r] + sub).astype(np.uint64)[:, None]
            key = (zz.astype(f32).view(np.uint32).astype(np.uint64) << np.uint64(32)) | ids
            key = np.where(inside, key, EMPTY)
            best = np.minimum(best, key.min(axis=0))
    hit = np.nonzero(best != EMPTY)[0]
    if len(hit) == 0:
        return rgba, depth, seg
    ids = (best[hit] & np.uint64(0xFFFFFFFF)).astype(np.int64)
    t_glob, sub = ids >> 1, ids & 1
    row = np.searchsorted(tid, t_glob)
    Xh, Yh = X[hit], Y[hit]
    out_d = np.zeros(len(hit), f32)
    out_c = np.zeros((len(hit), 3), np.uint8)
    for s_ in (0, 1):
        m = sub == s_
        if not m.any():
            continue
        S, r = subs[s_], row[m]
        x, y, w, area = S["x"][r], S["y"][r], S["w"][r], S["area"][r]
        e0 = _edge(x[:, 1], y[:, 1], x[:, 2], y[:, 2], Xh[m], Yh[m])
        e1 = _edge(x[:, 2], y[:, 2], x[:, 0], y[:, 0], Xh[m], Yh[m])
        e2 = _edge(x[:, 0], y[:, 0], x[:, 1], y[:, 1], Xh[m], Yh[m])
        # perspective-correct weights: e_k * (1 / area) * (1 / w_k), normalised by their sum
        ia = f32(1) / area
        q = [(e0, e1, e2)[k] * (ia * (f32(1) / w[:, k])) for k in range(3)]
        iQ = f32(1) / ((q[0] + q[1]) + q[2])
        att = np.take_along_axis(poly[r], S["order"][r][:, :, None], axis=1)  # (n, 3, 8)
        at = [((q[0] * att[:, 0, 3 + j] + q[1] * att[:, 1, 3 + j]) + q[2] * att[:, 2, 3 + j]) * iQ for j in range(5)]
        d = ((q[0] * w[:, 0] + q[1] * w[:, 1]) + q[2] * w[:, 2]) * iQ
        il = f32(1) / np.sqrt((at[0] * at[0] + at[1] * at[1]) + at[2] * at[2])
        n0, n1, n2 = at[0] * il, at[1] * il, at[2] * il
        head = np.abs(n2)
        keyl = np.fmax((n0 * L0 + n1 * L1) + n2 * L2, f32(0))
        shade = (f32(0.25) + f32(0.5) * head) + f32(0.35) * keyl
        tg_hit = tg[t_glob[m]]
        flags = vb[tris[t_glob[m], 0], 7]
        cx = np.floor(at[3] * f32(4)).astype(np.int64)  # checker squares of 0.25
        cy = np.floor(at[4] * f32(4)).astype(np.int64)
        checker = np.where(((cx + cy) & 1) == 1, f32(0.8), f32(1.05))
        shade = np.where((flags & 1) == 1, shade * checker, shade)
        col = np.fmin(np.fmax(app[tg_hit, 0:3].astype(f32) * shade[:, None], f32(0)), f32(1))
        out_c[m] = (col * f32(255) + f32(0.5)).astype(np.uint8)
        out_d[m] = d
        seg.reshape(-1)[hit[m]] = tg_hit
    rgba.reshape(-1, 4)[hit, 0:3] = out_c
    depth.reshape(-1)[hit] = out_d
    return rgba, depth, seg


def render(verts, tris, views, uni, W, H, geoms, cams, app):
    """All images of nenv environments: geoms (nenv, ngeom, 12), cams
    (nenv, ncam, 12), app (nenv, ngeom, 8). Shapes (nenv, nview, H, W[, 4])."""
    nenv, nview = geoms.shape[0], len(views)
    rgba = np.zeros((nenv, nview, H, W, 4), np.uint8)
    depth = np.zeros((nenv, nview, H, W), f32)
    seg = np.zeros((nenv, nview, H, W), np.int32)
    for e in range(nenv):
        for v in range(nview):
            rgba[e, v], depth[e, v], seg[e, v] = render_image(verts, tris, views[v], uni, W, H, geoms[e], app[e],
                                                              cams[e] if cams is not None and len(cams) else None)
    return rgba, depth, seg
