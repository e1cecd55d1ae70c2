"""The batched rasteriser: mesh building and the oracle on CPU (the oracle
pinned by the reference's analytic render tests,
crates/pippin-render/tests/geometry.rs), and on the GPU the CUDA kernel
against the oracle bit for bit plus the same analytic tests through the
C-ABI."""
import math
import os
import sys

import numpy as np
import pytest

from pippin_b200 import render as R
from pippin_b200.physics import CameraDesc, GeomVisual, Mesh, Scene, Shape

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import render_oracle as O  # noqa: E402

W = H = 128
FOVY = 60.0
f32 = np.float32


def geom(shape, size, rgba=(0.8, 0.2, 0.2, 1.0), group=0, mesh=None):
    return GeomVisual("g", shape, mesh, tuple(size), tuple(rgba), 1, group)


def one_geom(shape, size, dist, w=W, h=H):
    sc = Scene([], [geom(shape, size)], [], [])
    cfg = R.RenderConfig(w, h, [R.ViewSource.look_at([0.0, 0.0, dist], [0.0, 0.0, 0.0], FOVY)], 0.01, 100.0)
    return sc, cfg


def oracle_frames(sc, cfg, geoms, cams=None, app=None):
    v, t = R.build_mesh(sc)
    nenv = geoms.shape[0]
    if app is None:
        app = np.broadcast_to(R.base_appearance(sc), (nenv, len(sc.geoms), 8))
    if cams is None:
        cams = np.zeros((nenv, len(sc.cameras), 12), f32)
    return O.render(v, t, R.view_table(cfg, sc), R.uniforms(cfg), cfg.width, cfg.height, geoms, cams, app)


def px_per_unit(z):
    f = 1.0 / math.tan(0.5 * math.radians(FOVY))
    return f / z * (H / 2.0)


def pose(mat=(1, 0, 0, 0, 1, 0, 0, 0, 1), pos=(0, 0, 0)):
    return np.array(list(pos) + list(mat), f32)


LIE = (0, 0, 1, 0, 1, 0, -1, 0, 0)  # the z axis onto x
C45 = math.sqrt(0.5)


# ------------------------------------------------------------ analytic checks
def check_sphere(render):
    r, d = 0.2, 2.0
    rgba, depth, seg = render(*one_geom(Shape.SPHERE, (r, 0, 0), d), pose()[None, None])
    depth, seg = depth[0, 0], seg[0, 0]
    assert seg[H // 2, W // 2] == 0
    assert abs(depth[H // 2, W // 2] - (d - r)) < 2e-3
    rad_px = r / math.sqrt(d * d - r * r) * (1 / math.tan(0.5 * math.radians(FOVY))) * (H / 2)
    expect = math.pi * rad_px * rad_px
    assert abs((seg == 0).sum() - expect) / expect < 0.05
    assert seg[0, 0] == -1 and abs(depth[0, 0] - 100.0) < 1e-3
    assert tuple(rgba[0, 0, 0, 0]) == R.CLEAR_RGBA


def check_boxes(render):
    h, d = 0.1, 1.5
    _, depth, seg = render(*one_geom(Shape.BOX, (h, h, h), d), pose()[None, None])
    side = 2 * h * px_per_unit(d - h)
    assert abs((seg[0, 0] == 0).sum() - side * side) / (side * side) < 0.05
    assert abs(depth[0, 0, H // 2, W // 2] - (d - h)) < 2e-3
    _, _, seg = render(*one_geom(Shape.BOX, (h, h, h), d), pose((C45, -C45, 0, C45, C45, 0, 0, 0, 1))[None, None])
    seg = seg[0, 0]
    assert abs((seg == 0).sum() - side * side) / (side * side) < 0.06
    assert abs((seg[H // 2] == 0).sum() - side * math.sqrt(2)) < 3.0
    t = math.radians(30)
    c, s = math.cos(t), math.sin(t)
    _, _, seg = render(*one_geom(Shape.BOX, (h, h, h), d), pose((1, 0, 0, 0, c, -s, 0, s, c))[None, None])
    seg = seg[0, 0]
    assert (seg[:, W // 2] == 0).sum() > 2 * h * (c + s) * px_per_unit(d) * 0.9
    assert (seg[H // 2] == 0).sum() > 2 * h * px_per_unit(d) * 0.9


def check_lying(render):
    r, hl, d = 0.05, 0.2, 2.0
    s = px_per_unit(d - r)
    _, _, seg = render(*one_geom(Shape.CAPSULE, (r, hl, 0), d), pose(LIE)[None, None])
    expect = (2 * r * 2 * hl + math.pi * r * r) * s * s
    assert abs((seg == 0).sum() - expect) / expect < 0.08
    _, _, seg = render(*one_geom(Shape.CYLINDER, (r, hl, 0), d), pose(LIE)[None, None])
    expect = 2 * r * 2 * hl * s * s
    assert abs((seg == 0).sum() - expect) / expect < 0.08


def check_appearance(render):
    sc = Scene([], [geom(Shape.SPHERE, (0.1, 0, 0))], [], [])
    cfg = R.RenderConfig(W, H, [R.ViewSource.look_at([0, 0, 3.0], [0, 0, 0], FOVY)], 0.01, 100.0)
    app = np.array([[[1, 0, 0, 1, 1, 1, 1, 0]], [[0, 0, 1, 1, 2, 2, 2, 0]]], f32)
    rgba, _, seg = render(sc, cfg, np.stack([pose()[None]] * 2), app=app)
    a, b = (seg[0] == 0).sum(), (seg[1] == 0).sum()
    assert abs(b / a - 4.0) < 0.3
    c0, c1 = rgba[0, 0, H // 2, W // 2], rgba[1, 0, H // 2, W // 2]
    assert c0[0] > 100 and c0[2] < 30 and c1[2] > 100 and c1[0] < 30


ANALYTIC = [check_sphere, check_boxes, check_lying, check_appearance]


@pytest.mark.parametrize("check", ANALYTIC, ids=lambda f: f.__name__)
def test_oracle_matches_the_reference_analytic_tests(check):
    check(lambda sc, cfg, geoms, app=None: oracle_frames(sc, cfg, geoms, app=app))


# ------------------------------------------------------------- host side
def test_block_corner_test_never_drops_a_covered_pixel():
    """The renderer skips a 4 x 4 block of a queued sub-triangle when, for some
    edge, the ownership test fails at one corner of the block chosen by the
    signs of A = bx - ax and B = by - ay (pg_render.cu: edge_may_own). That is
    exact because the IEEE single-precision edge function
    fl(fl(A * fl(Y - ay)) - fl(B * fl(X - ax))) is monotonic in X along a row
    and in Y along a column. Checked here with the oracle's own float32 edge
    and ownership functions on random triangles, small and huge, thin and
    axis-aligned: no skipped block holds a pixel centre the per-pixel test
    accepts."""
    rng = np.random.default_rng(11)
    px, py = np.meshgrid(np.arange(64), np.arange(64))
    X, Y = px.astype(f32) + f32(0.5), py.astype(f32) + f32(0.5)
    checked = skipped = 0
    for trial in range(600):
        scale = f32(10.0 ** rng.uniform(-0.5, 7))
        c = rng.uniform(0, 64, 2)
        v = (rng.uniform(-1, 1, (3, 2)) * scale + c).astype(f32)
        if trial % 5 == 0:
            v[1] = v[0] + (v[1] - v[0]) * f32(1e-3)  # a sliver
        if trial % 7 == 0:
            v[2, 1] = v[1, 1]  # a horizontal edge
        area = O._edge(v[0, 0], v[0, 1], v[1, 0], v[1, 1], v[2, 0], v[2, 1])
        if not area > 0:
            v = v[[0, 2, 1]]
            area = O._edge(v[0, 0], v[0, 1], v[1, 0], v[1, 1], v[2, 0], v[2, 1])
        if not area > 0 or np.abs(v).max() >= 1e18:
            continue
        edges = [(v[1], v[2]), (v[2], v[0]), (v[0], v[1])]  # cover()'s order
        inside = np.ones_like(X, dtype=bool)
        for a, b in edges:
            inside &= O._owns(O._edge(a[0], a[1], b[0], b[1], X, Y), a[0], a[1], b[0], b[1])
        for by in range(0, 64, 4):
            for bx in range(0, 64, 4):
                keep = True
                for a, b in edges:
                    x = bx if (b[1] - a[1]) > 0 else bx + 3
                    y = by + 3 if (b[0] - a[0]) > 0 else by
                    e = O._edge(a[0], a[1], b[0], b[1], f32(x) + f32(0.5), f32(y) + f32(0.5))
                    keep &= bool(O._owns(e, a[0], a[1], b[0], b[1]))
                checked += 1
                if not keep:
                    skipped += 1
                    assert not inside[by:by + 4, bx:bx + 4].any(), (trial, bx, by, v.tolist())
    assert checked > 50000 and skipped > checked // 4


def test_mesh_triangle_counts_and_welding():
    sc = Scene([], [geom(Shape.PLANE, (0, 0, 0.1)), geom(Shape.SPHERE, (0.1, 0, 0)), geom(Shape.CAPSULE, (0.05, 0.2, 0)),
                    geom(Shape.CYLINDER, (0.05, 0.1, 0)), geom(Shape.BOX, (0.1, 0.2, 0.3)),
                    geom(Shape.BOX, (1, 1, 1), group=3), geom(Shape.SPHERE, (1, 0, 0), rgba=(1, 1, 1, 0))], [], [])
    v, t = R.build_mesh(sc)
    g = v.view(np.uint32)[:, 3][t[:, 0]]
    counts = np.bincount(g, minlength=7)
    # plane 2, sphere 12 stacks x 24 slices x 2, capsule 26-sample profile, cylinder 3 rings, box 12; hidden 0
    assert list(counts) == [2, 576, 1200, 144, 12, 0, 0]
    assert len(v) < 3 * len(t)  # welded
    assert np.allclose(np.linalg.norm(v[:, 4:7], axis=1), 1, atol=1e-6)
    assert (v.view(np.uint32)[:, 7][t[:, 0]] == (g == 0)).all()  # checker flag on the plane only
    # the box's faces point outwards
    box = t[g == 4]
    cen = v[box][:, :, 0:3].mean(axis=1)
    assert (np.einsum("ij,ij->i", cen, v[box[:, 0], 4:7]) > 0).all()


def test_mesh_geom_gets_smooth_normals():
    cube = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], f32) * 0.1
    tris = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                     [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.uint32)
    sc = Scene([], [geom(Shape.MESH, (1, 1, 1), mesh=0)], [Mesh("cube", cube, tris)], [])
    v, t = R.build_mesh(sc)
    assert len(v) == 8 and len(t) == 12
    assert np.allclose(np.linalg.norm(v[:, 4:7], axis=1), 1, atol=1e-6)


def test_look_at_and_views():
    vs = R.ViewSource.look_at([1.5, -1.5, 1.2], [0, 0, 0.3], 45.0)
    m = np.array(vs.mat).reshape(3, 3)
    assert np.allclose(m.T @ m, np.eye(3), atol=1e-6)
    fwd = -m[:, 2]  # the camera looks along its local -z
    to = np.array([0, 0, 0.3]) - np.array([1.5, -1.5, 1.2])
    assert np.allclose(fwd, to / np.linalg.norm(to), atol=1e-6)
    sc = Scene([], [], [], [CameraDesc("c", 90.0)])
    cfg = R.RenderConfig(64, 32, [vs, R.ViewSource.scene(0)], 0.01, 20.0)
    tab = R.view_table(cfg, sc)
    assert tab[0, 0] == -1 and tab[1, 0] == 0
    assert abs(tab[1, 2] - 1.0) < 1e-6 and abs(tab[1, 1] - 0.5) < 1e-6  # fovy 90, aspect 2
    u = R.uniforms(cfg)
    assert abs(u[2] - 20.0 / (0.01 - 20.0)) < 1e-6 and abs(np.linalg.norm(u[4:7]) - 1) < 1e-6


def test_renderer_rejects_bad_configs():
    sc = Scene([], [geom(Shape.SPHERE, (0.1, 0, 0))], [], [])
    with pytest.raises(R.RenderError, match="at least one view"):
        R.CudaRenderer(sc, R.RenderConfig(8, 8, []))
    with pytest.raises(R.RenderError, match="scene camera 2"):
        R.CudaRenderer(sc, R.RenderConfig(8, 8, [R.ViewSource.scene(2)]))


# ------------------------------------------------------------------ GPU
def random_scene(rng, with_mesh=True):
    gs = [geom(Shape.PLANE, (0, 0, 0.1), rgba=(0.9, 0.9, 0.9, 1))]
    for k in range(5):
        sh = [Shape.SPHERE, Shape.CAPSULE, Shape.CYLINDER, Shape.BOX, Shape.BOX][k]
        gs.append(geom(sh, rng.uniform(0.05, 0.2, 3), rgba=tuple(rng.uniform(0.1, 1, 3)) + (1.0,)))
    meshes = []
    if with_mesh:
        from pippin_b200 import mjcf
        pts = rng.normal(size=(12, 3))
        pts /= np.linalg.norm(pts, axis=1, keepdims=True) * 8
        hv, ht = mjcf.convex_hull([tuple(float(x) for x in p) for p in pts])
        meshes.append(Mesh("hull", np.asarray(hv, f32), np.asarray(ht, np.uint32)))
        gs.append(geom(Shape.MESH, (1, 1, 1), rgba=(0.2, 0.7, 0.3, 1), mesh=0))
    return Scene([], gs, meshes, [CameraDesc("track", 50.0)])


def random_poses(rng, nenv, ngeom):
    out = np.zeros((nenv, ngeom, 12), f32)
    for e in range(nenv):
        out[e, 0] = pose()
        for g in range(1, ngeom):
            q = rng.normal(size=4)
            q /= np.linalg.norm(q)
            w, x, y, z = q
            m = [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                 2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                 2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]
            out[e, g] = pose(m, rng.uniform([-0.5, -0.5, 0.0], [0.5, 0.5, 0.5]))
    return out


def gpu_frames(sc, cfg, geoms, cams=None, app=None):
    r = R.CudaRenderer(sc, cfg)
    try:
        nenv = geoms.shape[0]
        f = r.render(0, nenv, geoms, cams, app)
        return f.rgba.copy(), f.depth.copy(), f.segmentation.copy()
    finally:
        r.close()


@pytest.mark.gpu
@pytest.mark.parametrize("check", ANALYTIC, ids=lambda f: f.__name__)
def test_cuda_renderer_passes_the_reference_analytic_tests(check):
    check(lambda sc, cfg, geoms, app=None: gpu_frames(sc, cfg, geoms, app=app))


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,seed,tile", [(48, 40, 0, None), (96, 80, 1, None), (130, 70, 2, None), (200, 150, 3, None),
                                          (48, 40, 0, "128"), (130, 70, 2, "64"), (200, 150, 3, "64")])
def test_cuda_renderer_matches_the_oracle_bit_for_bit(w, h, seed, tile, monkeypatch):
    # tile: the renderer's tile edge when not its default (64 up to 64 pixels, else 128)
    if tile is not None:
        monkeypatch.setenv("PIPPIN_RENDER_TILE", tile)
    rng = np.random.default_rng(seed)
    sc = random_scene(rng)
    nenv, ng = 3, len(sc.geoms)
    geoms = random_poses(rng, nenv, ng)
    cams = np.stack([pose(R.ViewSource.look_at([0.8, -0.9, 0.6], [0, 0, 0.1], 50.0).mat, (0.8, -0.9, 0.6))[None]
                     for _ in range(nenv)])
    app = np.broadcast_to(R.base_appearance(sc), (nenv, ng, 8)).copy()
    app[1, 2, 3] = 0.0                   # hidden in env 1
    app[2, 1:, 4:7] = rng.uniform(0.5, 1.5, (ng - 1, 3))  # per-env scale
    views = [R.ViewSource.look_at([1.2, 1.0, 0.9], [0, 0, 0.1], 55.0), R.ViewSource.scene(0),
             R.ViewSource.look_at([0.3, -0.2, 0.05], [0, 0.5, 0.05], 80.0)]  # low: the plane crosses the near plane
    cfg = R.RenderConfig(w, h, views, 0.01, 20.0)
    want = oracle_frames(sc, cfg, geoms, cams, app)
    got = gpu_frames(sc, cfg, geoms, cams, app)
    for a, b, name in zip(got, want, ("rgba", "depth", "seg")):
        bad = np.argwhere(a.view(np.uint8) != b.view(np.uint8))
        assert len(bad) == 0, f"{name}: {len(bad)} bytes differ, first at {bad[:3].tolist()}"
    assert (got[2] >= 0).mean() > 0.3 and (got[2][1, :, :, :] == 2).sum() == 0


@pytest.mark.gpu
def test_cuda_renderer_on_ant_poses_matches_the_oracle():
    from pippin_b200 import CudaPhysics, Field, mjcf, scenes
    m = mjcf.load_string(scenes.ant_xml())
    n = 2
    phys = CudaPhysics(mjcf.to_blob(m), n)
    rng = np.random.default_rng(3)
    q = np.tile(np.asarray(m.qpos0), (n, 1)) + rng.uniform(-0.1, 0.1, (n, len(m.qpos0)))
    phys.set(Field.QPOS, range(n), q)
    phys.step(range(n), 20)
    g, c = phys.poses(range(n))
    sc = phys.scene()
    cfg = R.RenderConfig(40, 40, [R.ViewSource.look_at([1.5, -1.5, 1.2], [0, 0, 0.3], 45.0)], 0.01, 20.0)
    want = oracle_frames(sc, cfg, g, c)
    got = gpu_frames(sc, cfg, g, c)
    for a, b in zip(got, want):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    assert len(set(np.unique(got[2])) - {-1}) >= 5  # the floor and several body parts
    phys.close()


@pytest.mark.gpu
def test_cuda_renderer_length_errors_and_slots():
    sc, cfg = one_geom(Shape.SPHERE, (0.2, 0, 0), 2.0, 16, 16)
    r = R.CudaRenderer(sc, cfg)
    with pytest.raises(R.RenderError, match="expected 2 geom and 0 camera poses"):
        r.render(0, 2, np.zeros((1, 12), f32))
    with pytest.raises(R.RenderError, match="expected 1 appearance entries"):
        r.render(0, 1, pose()[None], None, np.zeros((2, 8), f32))
    a = r.render(0, 1, pose()[None])
    b = r.render(1, 1, pose((1, 0, 0, 0, 1, 0, 0, 0, 1), (5, 0, 0))[None])
    assert (a.segmentation == 0).sum() > 0 and (b.segmentation == 0).sum() == 0  # slot 0 kept
    r.close()



@pytest.mark.gpu
@pytest.mark.parametrize("nenv", [5003, 7919])
def test_host_buffer_frames_in_chunks_match_device_frames(nenv):
    """Host-buffer frames of thousands of small images render in several
    chunks (each chunk's copies back overlap the next chunk's kernel). The
    chunk count comes from the work, and the env counts here do not divide
    evenly by it. The images must equal the device-buffer path's bit for bit,
    and a sample of envs the oracle's."""
    import torch
    rng = np.random.default_rng(nenv)
    sc = random_scene(rng)
    ng = len(sc.geoms)
    geoms = random_poses(rng, nenv, ng)
    cams = np.tile(pose(R.ViewSource.look_at([0.8, -0.9, 0.6], [0, 0, 0.1], 50.0).mat, (0.8, -0.9, 0.6)),
                   (nenv, 1, 1)).astype(f32)
    app = np.broadcast_to(R.base_appearance(sc), (nenv, ng, 8)).copy()
    app[::7, 3, 3] = 0.0  # some geoms hidden
    cfg = R.RenderConfig(16, 16, [R.ViewSource.look_at([1.2, 1.0, 0.9], [0, 0, 0.1], 55.0)], 0.01, 20.0)
    r = R.CudaRenderer(sc, cfg)
    try:
        host = r.render(0, nenv, geoms, cams, app)
        dev = torch.device("cuda", 0)
        gd, cd, ad = (torch.from_numpy(np.ascontiguousarray(x).reshape(-1)).to(dev) for x in (geoms, cams, app))
        px = nenv * 16 * 16
        rgba = torch.empty(px * 4, dtype=torch.uint8, device=dev)
        depth = torch.empty(px, dtype=torch.float32, device=dev)
        seg = torch.empty(px, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        r.render_device(nenv, gd.data_ptr(), cd.data_ptr(), ad.data_ptr(), rgba.data_ptr(), depth.data_ptr(),
                        seg.data_ptr())
        r.synchronize()
        got_dev = (rgba.cpu().numpy(), depth.cpu().numpy(), seg.cpu().numpy())
        for a, b, name in zip((host.rgba, host.depth, host.segmentation), got_dev, ("rgba", "depth", "seg")):
            assert np.array_equal(a.reshape(-1).view(np.uint8), b.reshape(-1).view(np.uint8)), name
        assert (host.segmentation >= 0).mean() > 0.2
        # chunk edges and a few envs in between against the oracle
        sample = sorted({0, 1, nenv // 3, nenv // 2, nenv - 2, nenv - 1})
        want = oracle_frames(sc, cfg, geoms[sample], cams[sample], app[sample])
        for a, b in zip((host.rgba[sample], host.depth[sample], host.segmentation[sample]), want):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
    finally:
        r.close()

def test_c_abi_rejects_bad_scenes_before_touching_the_gpu():
    """pg_render_create checks its arguments before any CUDA call, so the
    errors come back (with pg_last_error set) on a machine without a GPU."""
    import ctypes as C

    from pippin_b200 import _native
    L = _native.load()
    sc = Scene([], [geom(Shape.BOX, (0.1, 0.1, 0.1))], [], [CameraDesc("c", 45.0)])
    cfg = R.RenderConfig(8, 8, [R.ViewSource.scene(0)], 0.01, 10.0)
    v, t = R.build_mesh(sc)
    views, uni, app = R.view_table(cfg, sc), R.uniforms(cfg), R.base_appearance(sc)

    def create(verts=v, tris=t, ngeom=1, ncam=1, views=views, uni=uni):
        h = C.c_void_p()
        pf = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
        rc = L.pg_render_create(pf(verts), len(verts), tris.ctypes.data_as(C.POINTER(C.c_uint32)), len(tris), ngeom,
                                ncam, pf(views), len(views), pf(app), 8, 8, pf(uni), 0, C.byref(h))
        return rc, _native.last_error()

    bad = t.copy()
    bad[0, 0] = len(v)
    assert create(tris=bad) == (_native.PG_ERR_INVALID, "triangle index out of range")
    assert create(ncam=0) == (_native.PG_ERR_INVALID, "view refers to a camera the scene does not have")
    far_first = uni.copy()
    far_first[1] = far_first[0]
    assert create(uni=far_first) == (_native.PG_ERR_INVALID, "need 0 < near < far")
    vb = v.copy()
    vb.view(np.uint32)[0, 3] = 5
    assert create(verts=vb) == (_native.PG_ERR_INVALID, "vertex geom id out of range")
