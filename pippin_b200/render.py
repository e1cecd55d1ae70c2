"""Batched renderer of environment poses: the host side of
include/pippin_b200_render.h.

Mirrors the reference's `Renderer` trait and its Metal implementation:
`RenderConfig`, `ViewSource` and `Frames` (crates/pippin-env/src/lib.rs:173-238),
the per-geom triangle meshes (crates/pippin-render/src/mesh.rs) and
`MetalRenderer::new` / `render` (crates/pippin-render/src/lib.rs:95-355) as
`CudaRenderer`. Images are rendered by the CUDA rasteriser in
csrc/pg_render.cu; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native
from .physics import Scene, Shape

f32 = np.float32
SLICES = 24
STACKS = 12
PLANE_EXTENT = 20.0  # visual half-extent of planes declared infinite (size 0)
CLEAR_RGBA = (184, 199, 219, 255)  # the clear colour (0.72, 0.78, 0.86, 1) in RGBA8


class RenderError(ValueError):
    pass


@dataclass
class ViewSource:
    """A scene camera (`camera` >= 0) or a fixed world pose with its own
    vertical field of view in degrees (lib.rs:173-199)."""
    camera: int = -1
    pos: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    mat: Tuple[float, ...] = (1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0)
    fovy: float = 0.0

    @staticmethod
    def scene(camera: int) -> "ViewSource":
        return ViewSource(camera=int(camera))

    @staticmethod
    def fixed(pos, mat, fovy: float) -> "ViewSource":
        return ViewSource(-1, tuple(float(x) for x in pos), tuple(float(x) for x in mat), float(fovy))

    @staticmethod
    def look_at(eye, target, fovy: float) -> "ViewSource":
        """Fixed camera at `eye` looking at `target` with +z up; the camera
        looks along its local -z (lib.rs:182-199), in single precision."""
        eye = np.asarray(eye, f32)
        target = np.asarray(target, f32)

        def norm(a):
            n = max(float(np.sqrt(f32(a[0] * a[0] + a[1] * a[1]) + a[2] * a[2])), 1e-12)
            return (a / f32(n)).astype(f32)

        def cross(a, b):
            return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]], f32)

        z = norm(eye - target)
        up = np.array([0, 1, 0] if abs(z[2]) > 0.99 else [0, 0, 1], f32)
        x = norm(cross(up, z))
        y = cross(z, x)
        mat = [x[0], y[0], z[0], x[1], y[1], z[1], x[2], y[2], z[2]]
        return ViewSource(-1, tuple(float(v) for v in eye), tuple(float(v) for v in mat), float(fovy))


@dataclass
class RenderConfig:
    width: int
    height: int
    views: List[ViewSource] = field(default_factory=list)
    near: float = 0.01
    far: float = 100.0


@dataclass
class Frames:
    """Images shaped (envs, views, height, width[, 4])."""
    rgba: np.ndarray
    depth: np.ndarray
    segmentation: np.ndarray


# ------------------------------------------------------------------ meshes
def _normalize(a):
    a = np.asarray(a, f32)
    n = max(f32(np.sqrt(f32(a[0] * a[0] + a[1] * a[1]) + a[2] * a[2])), f32(1e-12))
    return a / n


class _Builder:
    def __init__(self):
        self.pos: List[np.ndarray] = []
        self.nrm: List[np.ndarray] = []
        self.geom: List[int] = []
        self.flags: List[int] = []
        self.g = 0
        self.f = 0

    def tri(self, p, n):
        for i in range(3):
            self.pos.append(np.asarray(p[i], f32))
            self.nrm.append(np.asarray(n[i], f32))
            self.geom.append(self.g)
            self.flags.append(self.f)

    def flat(self, a, b, c):
        a, b, c = (np.asarray(x, f32) for x in (a, b, c))
        n = _normalize(np.cross(b - a, c - a).astype(f32))
        self.tri([a, b, c], [n, n, n])


def _revolve(b: _Builder, profile):
    """Surface of revolution around z from (radius, z, normal_r, normal_z)
    samples (mesh.rs:46-67)."""
    ring = [(f32(math.cos(2 * math.pi * k / SLICES)), f32(math.sin(2 * math.pi * k / SLICES))) for k in range(SLICES)]
    for (r0, z0, nr0, nz0), (r1, z1, nr1, nz1) in zip(profile[:-1], profile[1:]):
        for k in range(SLICES):
            c0, s0 = ring[k]
            c1, s1 = ring[(k + 1) % SLICES]

            def p(r, z, c, s):
                return [f32(r) * c, f32(r) * s, f32(z)]

            def n(nr, nz, c, s):
                return _normalize([f32(nr) * c, f32(nr) * s, f32(nz)])

            a, bb, cc, d = p(r0, z0, c0, s0), p(r0, z0, c1, s1), p(r1, z1, c1, s1), p(r1, z1, c0, s0)
            na, nb, nc, nd = n(nr0, nz0, c0, s0), n(nr0, nz0, c1, s1), n(nr1, nz1, c1, s1), n(nr1, nz1, c0, s0)
            b.tri([a, bb, cc], [na, nb, nc])
            b.tri([a, cc, d], [na, nc, nd])


def _sphere_profile(r, z_offset, start, stop):
    out = []
    for i in range(STACKS + 1):
        phi = start + (stop - start) * i / STACKS
        s, c = math.sin(phi), math.cos(phi)
        out.append((r * s, z_offset + r * c, s, c))
    return out


def _box(b: _Builder, h):
    for axis in range(3):
        for sign in (-1.0, 1.0):
            u, v = (axis + 1) % 3, (axis + 2) % 3

            def corner(su, sv):
                p = [0.0, 0.0, 0.0]
                p[axis] = sign * h[axis]
                p[u] = su * h[u]
                p[v] = sv * h[v]
                return p

            a, bb, c, d = corner(-1, -1), corner(1, -1), corner(1, 1), corner(-1, 1)
            if sign > 0:
                b.flat(a, bb, c)
                b.flat(a, c, d)
            else:
                b.flat(a, c, bb)
                b.flat(a, d, c)


def _visible(g) -> bool:
    """Groups 0-2 with a positive alpha are drawn (mesh.rs:122-125)."""
    return g.group <= 2 and g.rgba[3] > 0.0


def build_mesh(scene: Scene) -> Tuple[np.ndarray, np.ndarray]:
    """Triangulates every visible geom in its local frame with its size
    baked in (mesh.rs:172-236), then welds identical (position, normal,
    geom, flags) vertices (mesh.rs:100-118). Mesh geoms get area-weighted
    smooth normals (mesh.rs:128-171; no simplification). Returns
    (vertices (n, 8) float32 with geom and flags as u32 bits, triangles
    (m, 3) uint32) in draw order."""
    b = _Builder()
    mesh_tris = []
    for g, geom in enumerate(scene.geoms):
        if not _visible(geom):
            continue
        b.g, b.f = g, int(geom.shape == Shape.PLANE)
        s = [float(x) for x in geom.size]
        if geom.shape == Shape.PLANE:
            ex = s[0] if s[0] > 0 else PLANE_EXTENT
            ey = s[1] if s[1] > 0 else PLANE_EXTENT
            b.flat([-ex, -ey, 0.0], [ex, -ey, 0.0], [ex, ey, 0.0])
            b.flat([-ex, -ey, 0.0], [ex, ey, 0.0], [-ex, ey, 0.0])
        elif geom.shape == Shape.SPHERE:
            _revolve(b, _sphere_profile(s[0], 0.0, 0.0, math.pi))
        elif geom.shape == Shape.CAPSULE:
            prof = _sphere_profile(s[0], s[1], 0.0, math.pi / 2) + _sphere_profile(s[0], -s[1], math.pi / 2, math.pi)
            _revolve(b, prof)
        elif geom.shape == Shape.CYLINDER:
            r, h = s[0], s[1]
            _revolve(b, [(0.0, h, 0.0, 1.0), (r, h, 0.0, 1.0)])
            _revolve(b, [(r, h, 1.0, 0.0), (r, -h, 1.0, 0.0)])
            _revolve(b, [(r, -h, 0.0, -1.0), (0.0, -h, 0.0, -1.0)])
        elif geom.shape == Shape.BOX:
            _box(b, s)
        elif geom.shape == Shape.MESH and geom.mesh is not None and geom.mesh < len(scene.meshes):
            mesh_tris.append((g, scene.meshes[geom.mesh]))
    verts: List[Tuple] = []
    index: Dict[Tuple, int] = {}
    tris: List[int] = []
    for p, n, g, fl in zip(b.pos, b.nrm, b.geom, b.flags):
        key = (p.tobytes(), n.tobytes(), g, fl)
        k = index.get(key)
        if k is None:
            k = index[key] = len(verts)
            verts.append((p, n, g, fl))
        tris.append(k)
    for g, mesh in mesh_tris:
        wpos: List[np.ndarray] = []
        wmap: Dict[bytes, int] = {}
        idx = []
        for t in np.asarray(mesh.triangles, np.uint32).reshape(-1, 3):
            for i in t:
                p = np.asarray(mesh.vertices[i], f32)
                k = wmap.get(p.tobytes())
                if k is None:
                    k = wmap[p.tobytes()] = len(wpos)
                    wpos.append(p)
                idx.append(k)
        nrm = [np.zeros(3, f32) for _ in wpos]
        for t in range(0, len(idx), 3):
            a, bb, c = wpos[idx[t]], wpos[idx[t + 1]], wpos[idx[t + 2]]
            n = np.cross(bb - a, c - a).astype(f32)
            for i in idx[t:t + 3]:
                nrm[i] = (nrm[i] + n).astype(f32)
        base = len(verts)
        verts.extend((p, _normalize(n), g, 0) for p, n in zip(wpos, nrm))
        tris.extend(base + i for i in idx)
    out = np.zeros((len(verts), 8), f32)
    bits = out.view(np.uint32)
    for k, (p, n, g, fl) in enumerate(verts):
        out[k, 0:3] = p
        out[k, 4:7] = n
        bits[k, 3] = g
        bits[k, 7] = fl
    return out, np.asarray(tris, np.uint32).reshape(-1, 3)


def view_table(config: RenderConfig, scene: Scene) -> np.ndarray:
    """16 floats per view: camera index (-1 fixed), fx = f / aspect, fy = f,
    pad, fixed pose; f = 1 / tan(fovy / 2) with a view's own fovy, else its
    scene camera's, else 45 degrees (render.metal:91-97)."""
    aspect = f32(config.width) / f32(config.height)
    out = np.zeros((len(config.views), 16), f32)
    cam_fovy = [c.fovy for c in scene.cameras] or [45.0]
    for i, v in enumerate(config.views):
        fovy = v.fovy if v.fovy > 0 else cam_fovy[max(v.camera, 0)]
        f = f32(1.0 / math.tan(0.5 * float(f32(fovy)) * math.pi / 180.0))
        out[i, 0] = v.camera if v.camera >= 0 else -1
        out[i, 1] = f / aspect
        out[i, 2] = f
        out[i, 4:7] = v.pos
        out[i, 7:16] = v.mat
    return out


def uniforms(config: RenderConfig) -> np.ndarray:
    """near, far, A = far / (near - far), A * near, the key light direction
    normalize(-0.4, 0.8, 0.5) in camera space (render.metal:114-115), pad."""
    near, far = f32(config.near), f32(config.far)
    A = far / (near - far)
    L = np.array([-0.4, 0.8, 0.5], f32)
    L = L / np.sqrt(f32(L[0] * L[0] + L[1] * L[1]) + L[2] * L[2])
    return np.array([near, far, A, A * near, L[0], L[1], L[2], 0.0], f32)


def base_appearance(scene: Scene) -> np.ndarray:
    out = np.zeros((len(scene.geoms), 8), f32)
    for g, geom in enumerate(scene.geoms):
        out[g, 0:4] = geom.rgba
        out[g, 4:7] = 1.0
    return out


def _host(shape, dtype) -> np.ndarray:
    """A slot's output array, in page-locked memory when torch can provide
    it, so that the copies back from the device run at full speed."""
    try:
        import torch
        tdt = {np.uint8: torch.uint8, np.float32: torch.float32, np.int32: torch.int32}[np.dtype(dtype).type]
        return torch.empty(shape, dtype=tdt, pin_memory=True).numpy()
    except Exception:
        return np.empty(shape, dtype)


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class CudaRenderer:
    """`Renderer` (lib.rs:220-238) on the CUDA rasteriser. Output lives in
    numbered slots: a slot's frames stay valid until that slot is rendered
    again."""

    def __init__(self, scene: Scene, config: RenderConfig, device: int = 0):
        if not config.views:
            raise RenderError("RenderConfig needs at least one view")
        for v in config.views:
            if v.camera >= len(scene.cameras):
                raise RenderError(f"view refers to scene camera {v.camera}, scene has {len(scene.cameras)}")
        self._L = _native.load()
        self.config = config
        self.ngeom = len(scene.geoms)
        self.ncam = len(scene.cameras)
        self.vertices, self.triangles = build_mesh(scene)
        self.views = view_table(config, scene)
        self.uniforms = uniforms(config)
        self.base_appearance = base_appearance(scene)
        h = C.c_void_p()
        rc = self._L.pg_render_create(_fp(self.vertices), len(self.vertices),
                                      self.triangles.ctypes.data_as(C.POINTER(C.c_uint32)), len(self.triangles),
                                      self.ngeom, self.ncam, _fp(self.views), len(self.views), _fp(self.base_appearance),
                                      config.width, config.height, _fp(self.uniforms), device, C.byref(h))
        if rc:
            raise RenderError(_native.last_error())
        self._h = h
        self._slots: Dict[int, Frames] = {}

    def name(self) -> str:
        return "cuda-raster"

    def close(self):
        if getattr(self, "_h", None):
            self._L.pg_render_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc:
            raise RenderError(_native.last_error())

    def render(self, slot: int, nenv: int, geoms, cams=None, appearance=None) -> Frames:
        """geoms: (nenv * ngeom) poses as (…, 12) float32 [pos, row-major
        mat]; cams: (nenv * ncam) poses; appearance: (nenv * ngeom, 8) or
        None for the scene's colours at unit scale."""
        g = np.ascontiguousarray(np.asarray(geoms, f32).reshape(-1))
        c = np.ascontiguousarray(np.asarray(cams if cams is not None else np.zeros(0), f32).reshape(-1))
        a = None if appearance is None else np.ascontiguousarray(np.asarray(appearance, f32).reshape(-1))
        if g.size != nenv * self.ngeom * 12 or c.size != nenv * self.ncam * 12:
            raise RenderError(f"expected {nenv * self.ngeom} geom and {nenv * self.ncam} camera poses")
        if a is not None and a.size != nenv * self.ngeom * 8:
            raise RenderError(f"expected {nenv * self.ngeom} appearance entries")
        W, H, nv = self.config.width, self.config.height, len(self.config.views)
        fr = self._slots.get(slot)
        if fr is None or fr.depth.shape[0] != nenv:
            fr = Frames(_host((nenv, nv, H, W, 4), np.uint8), _host((nenv, nv, H, W), f32),
                        _host((nenv, nv, H, W), np.int32))
            self._slots[slot] = fr
        self._check(self._L.pg_render_frames(
            self._h, nenv, _fp(g), g.size, _fp(c), c.size, None if a is None else _fp(a), 0 if a is None else a.size,
            fr.rgba.ctypes.data_as(C.POINTER(C.c_uint8)), _fp(fr.depth),
            fr.segmentation.ctypes.data_as(C.POINTER(C.c_int32))))
        return fr

    def render_device(self, nenv: int, geoms_ptr: int, cams_ptr: int, appearance_ptr: int, rgba_ptr: int,
                      depth_ptr: int, seg_ptr: int):
        """Enqueues a frame from device buffers on the renderer's stream."""
        self._check(self._L.pg_render_frames_device(self._h, nenv, geoms_ptr or None, cams_ptr or None,
                                                    appearance_ptr or None, rgba_ptr, depth_ptr, seg_ptr))

    def stream(self) -> int:
        return self._L.pg_render_stream(self._h) or 0

    def synchronize(self):
        self._check(self._L.pg_render_synchronize(self._h))


def poses_to_array(geoms: np.ndarray) -> np.ndarray:
    """Physics.poses() output (…, 12) as the renderer's pose layout (the
    same [pos, row-major mat] floats)."""
    return np.ascontiguousarray(np.asarray(geoms, f32).reshape(-1, 12))


def identity_pose(pos: Sequence[float] = (0.0, 0.0, 0.0)) -> np.ndarray:
    return np.array(list(pos) + [1, 0, 0, 0, 1, 0, 0, 0, 1], f32)
