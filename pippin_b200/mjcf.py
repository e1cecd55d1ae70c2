"""MJCF subset -> model blob.

Compiles the MuJoCo-XML subset the reference loader accepts
(crates/pippin/src/mjcf.rs:211-395) into the flat model blob that
``pg_create`` consumes (format: include/pippin_b200.h). The arithmetic
follows the reference loader operation by operation (quaternion conventions
of crates/pippin/src/math.rs:214-301, geom mass properties of
mjcf.rs:684-716,774-808, inertia finalisation of mjcf.rs:829-850) and the
compile step of crates/pippin/src/model.rs:279-451 (dof tree, dof blocks,
weld ids, static collision filter). Everything derived from a configuration
(invweight0, bounding volumes) is recomputed by whoever loads the blob.
"""
from __future__ import annotations

import math
import struct
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

PI = math.pi

JNT_FREE, JNT_BALL, JNT_SLIDE, JNT_HINGE = 0, 1, 2, 3
GEOM_PLANE, GEOM_SPHERE, GEOM_CAPSULE, GEOM_BOX, GEOM_CYLINDER, GEOM_MESH = range(6)
GEOM_TYPES = {"plane": GEOM_PLANE, "sphere": GEOM_SPHERE, "capsule": GEOM_CAPSULE, "box": GEOM_BOX,
              "cylinder": GEOM_CYLINDER, "mesh": GEOM_MESH}


class MjcfError(ValueError):
    """Invalid or unsupported model (mjcf.rs:13-25)."""


# ----------------------------------------------------------------- math.rs restated on tuples
def vdot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def vcross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


def vadd(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def vsub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def vscale(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def vnorm(a):
    return math.sqrt(vdot(a, a))


def vnormalized(a):
    n = vnorm(a)
    if n > 1e-15:
        return vscale(a, 1.0 / n)
    return (0.0, 0.0, 0.0)


def m_mul(a, b):
    return tuple(a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j]
                 for i in range(3) for j in range(3))


def m_t(m):
    return (m[0], m[3], m[6], m[1], m[4], m[7], m[2], m[5], m[8])


def m_vec(m, v):
    return (m[0] * v[0] + m[1] * v[1] + m[2] * v[2], m[3] * v[0] + m[4] * v[1] + m[5] * v[2],
            m[6] * v[0] + m[7] * v[1] + m[8] * v[2])


def m_add(a, b):
    return tuple(x + y for x, y in zip(a, b))


def m_scale(m, s):
    return tuple(x * s for x in m)


def m_diag(d):
    return (d[0], 0.0, 0.0, 0.0, d[1], 0.0, 0.0, 0.0, d[2])


def m_skew(v):
    return (0.0, -v[2], v[1], v[2], 0.0, -v[0], -v[1], v[0], 0.0)


def m_rotate(inertia, r):
    """R * I * R^T (math.rs:209-211)."""
    return m_mul(m_mul(r, inertia), m_t(r))


def m_cols(a, b, c):
    return (a[0], b[0], c[0], a[1], b[1], c[1], a[2], b[2], c[2])


Q_ID = (1.0, 0.0, 0.0, 0.0)


def q_axis_angle(axis, angle):
    a = vnormalized(axis)
    s, c = math.sin(0.5 * angle), math.cos(0.5 * angle)
    return (c, a[0] * s, a[1] * s, a[2] * s)


def q_normalized(q):
    n = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    if n < 1e-15:
        return Q_ID
    return (q[0] / n, q[1] / n, q[2] / n, q[3] / n)


def q_mul(p, o):
    a, b, c, d = p
    e, f, g, h = o
    return (a * e - b * f - c * g - d * h, a * f + b * e + c * h - d * g,
            a * g - b * h + c * e + d * f, a * h + b * g - c * f + d * e)


def q_to_mat(q):
    w, x, y, z = q
    ww, xx, yy, zz = w * w, x * x, y * y, z * z
    xy, xz, yz, wx, wy, wz = x * y, x * z, y * z, w * x, w * y, w * z
    return (ww + xx - yy - zz, 2.0 * (xy - wz), 2.0 * (xz + wy),
            2.0 * (xy + wz), ww - xx + yy - zz, 2.0 * (yz - wx),
            2.0 * (xz - wy), 2.0 * (yz + wx), ww - xx - yy + zz)


def q_from_mat(m):
    """Shepperd's method (math.rs:271-291)."""
    tr = m[0] + m[4] + m[8]
    if tr > 0.0:
        s = math.sqrt(tr + 1.0) * 2.0
        q = (0.25 * s, (m[7] - m[5]) / s, (m[2] - m[6]) / s, (m[3] - m[1]) / s)
    elif m[0] > m[4] and m[0] > m[8]:
        s = math.sqrt(1.0 + m[0] - m[4] - m[8]) * 2.0
        q = ((m[7] - m[5]) / s, 0.25 * s, (m[1] + m[3]) / s, (m[2] + m[6]) / s)
    elif m[4] > m[8]:
        s = math.sqrt(1.0 + m[4] - m[0] - m[8]) * 2.0
        q = ((m[2] - m[6]) / s, (m[1] + m[3]) / s, 0.25 * s, (m[5] + m[7]) / s)
    else:
        s = math.sqrt(1.0 + m[8] - m[0] - m[4]) * 2.0
        q = ((m[3] - m[1]) / s, (m[2] + m[6]) / s, (m[5] + m[7]) / s, 0.25 * s)
    q = q_normalized(q)
    if q[0] < 0.0:
        return tuple(-v for v in q)
    return q


def q_from_z_to(direction):
    """Rotation taking +z onto `direction` (math.rs:293-302)."""
    d = vnormalized(direction)
    c = vdot((0.0, 0.0, 1.0), d)
    if c < -1.0 + 1e-12:
        return (0.0, 1.0, 0.0, 0.0)
    axis = vcross((0.0, 0.0, 1.0), d)
    return q_normalized((1.0 + c, axis[0], axis[1], axis[2]))


# ----------------------------------------------------------------- convex hull
def convex_hull(points: List[Tuple[float, float, float]]):
    """Incremental 3-D convex hull: (vertices, outward-wound triangles).

    Stands in for parry3d-f64's `transformation::convex_hull` (mesh.rs:63-67),
    an un-vendored dependency; only the hull's point set and an outward
    winding matter to the mass properties and the narrow phase.
    """
    import numpy as np

    pts = np.asarray(points, dtype=np.float64)
    n = len(pts)
    if n < 4:
        raise MjcfError("convex hull needs at least 4 points")
    scale = float(np.abs(pts).max()) or 1.0
    eps = 1e-10 * scale
    # initial tetrahedron from extreme points
    i0 = int(np.argmin(pts[:, 0]))
    i1 = int(np.argmax(np.linalg.norm(pts - pts[i0], axis=1)))
    d01 = pts[i1] - pts[i0]
    cr = np.cross(d01, pts - pts[i0])
    i2 = int(np.argmax(np.linalg.norm(cr, axis=1)))
    nrm = np.cross(d01, pts[i2] - pts[i0])
    vol = (pts - pts[i0]) @ nrm
    i3 = int(np.argmax(np.abs(vol)))
    if abs(vol[i3]) <= eps * scale * scale or np.linalg.norm(nrm) <= eps * scale:
        raise MjcfError("degenerate point set: no convex hull")
    faces = []

    def add_face(a, b, c, inside):
        nn = np.cross(pts[b] - pts[a], pts[c] - pts[a])
        if np.dot(nn, inside - pts[a]) > 0:
            b, c = c, b
        faces.append([a, b, c])

    tet = [i0, i1, i2, i3]
    centroid = pts[tet].mean(axis=0)
    for f in ((i0, i1, i2), (i0, i1, i3), (i0, i2, i3), (i1, i2, i3)):
        add_face(*f, centroid)
    for p in range(n):
        if p in tet:
            continue
        visible = []
        for fi, (a, b, c) in enumerate(faces):
            nn = np.cross(pts[b] - pts[a], pts[c] - pts[a])
            ln = np.linalg.norm(nn)
            if ln > 0 and np.dot(nn / ln, pts[p] - pts[a]) > eps:
                visible.append(fi)
        if not visible:
            continue
        edges = {}
        for fi in visible:
            a, b, c = faces[fi]
            for e in ((a, b), (b, c), (c, a)):
                edges[e] = edges.get(e, 0) + 1
        horizon = [e for e in edges if (e[1], e[0]) not in edges]
        vis = set(visible)
        faces = [f for i, f in enumerate(faces) if i not in vis]
        for a, b in horizon:
            faces.append([a, b, p])
    used = sorted({i for f in faces for i in f})
    remap = {old: new for new, old in enumerate(used)}
    verts = [tuple(float(x) for x in pts[i]) for i in used]
    tris = [tuple(remap[i] for i in f) for f in faces]
    return verts, tris


def hull_features(verts, tris):
    """Polygon faces and edges of a convex hull given as outward triangles.

    Coplanar triangles merge into one face: (outward unit normal, offset d
    with n . v <= d inside, vertex loop counter-clockwise seen from outside).
    Edges are the unique vertex pairs that bound two different faces. The
    general convex narrow phase clips against these polygons and tests their
    edge directions.
    """
    import numpy as np

    v = np.asarray(verts, dtype=np.float64)
    scale = float(np.abs(v).max()) if len(v) else 1.0
    tol = 1e-10 * max(scale, 1.0)
    planes = []
    for a, b, c in tris:
        n = np.cross(v[b] - v[a], v[c] - v[a])
        ln = float(np.linalg.norm(n))
        n = n / ln if ln > 0 else n
        planes.append((n, float(n @ v[a])))
    group = [-1] * len(tris)
    faces = []
    for t in range(len(tris)):
        if group[t] != -1:
            continue
        n0, d0 = planes[t]
        members = [u for u in range(len(tris)) if group[u] == -1 and
                   float(planes[u][0] @ n0) > 1.0 - 1e-10 and abs(planes[u][1] - d0) <= tol]
        for u in members:
            group[u] = len(faces)
        directed = set()
        for u in members:
            a, b, c = tris[u]
            directed.update(((a, b), (b, c), (c, a)))
        nxt = {a: b for a, b in directed if (b, a) not in directed}
        start = min(nxt)
        loop = [start]
        while nxt[loop[-1]] != start:
            loop.append(nxt[loop[-1]])
            if len(loop) > len(nxt):
                raise MjcfError("hull face boundary is not a single loop")
        faces.append((tuple(float(x) for x in n0), d0, loop))
    edges = sorted({(min(a, b), max(a, b)) for _, _, loop in faces
                    for a, b in zip(loop, loop[1:] + loop[:1])})
    return faces, edges


def mesh_mass_properties(verts, tris):
    """Volume, com, inertia about com per unit density (mesh.rs:71-105)."""
    vol = 0.0
    first = (0.0, 0.0, 0.0)
    c = [[0.0] * 3 for _ in range(3)]
    for t in tris:
        a, b, d = verts[t[0]], verts[t[1]], verts[t[2]]
        v6 = vdot(a, vcross(b, d))
        vol += v6 / 6.0
        first = vadd(first, vscale(vadd(vadd(a, b), d), v6 / 24.0))
        for i in range(3):
            for j in range(3):
                s = a[i] * a[j] + b[i] * b[j] + d[i] * d[j]
                p = (a[i] + b[i] + d[i]) * (a[j] + b[j] + d[j])
                c[i][j] += v6 / 120.0 * (s + p)
    if abs(vol) < 1e-18:
        return 0.0, (0.0, 0.0, 0.0), (0.0,) * 9
    com = vscale(first, 1.0 / vol)
    tr = c[0][0] + c[1][1] + c[2][2]
    io = tuple((tr if i == j else 0.0) - c[i][j] for i in range(3) for j in range(3))
    cx = m_skew(com)
    icom = m_add(io, m_scale(m_mul(cx, m_t(cx)), -vol))
    return vol, com, icom


# ----------------------------------------------------------------- model
@dataclass
class Model:
    """Raw compiled model (the fields of model.rs:103-249 the step path reads)."""
    timestep: float = 0.002
    gravity: Tuple[float, float, float] = (0.0, 0.0, -9.81)
    integrator: int = 0
    solver: int = 0
    iterations: int = 30
    tolerance: float = 1e-8
    margin: float = 1e-3
    solref: Tuple[float, float] = (0.02, 1.0)
    solimp: Tuple[float, ...] = (0.9, 0.95, 0.001, 0.5, 2.0)
    impratio: float = 1.0
    hertz: float = 0.0
    dampratio: float = 1.0
    slop: float = 5e-4
    nq: int = 0
    nv: int = 0
    nu: int = 0
    body_names: List[str] = field(default_factory=list)
    body_parent: List[int] = field(default_factory=list)
    body_pos: List[tuple] = field(default_factory=list)
    body_quat: List[tuple] = field(default_factory=list)
    body_jntadr: List[int] = field(default_factory=list)
    body_jntnum: List[int] = field(default_factory=list)
    body_dofadr: List[int] = field(default_factory=list)
    body_dofnum: List[int] = field(default_factory=list)
    body_mass: List[float] = field(default_factory=list)
    body_ipos: List[tuple] = field(default_factory=list)
    body_inertia: List[tuple] = field(default_factory=list)
    body_lastdof: List[int] = field(default_factory=list)
    body_weldid: List[int] = field(default_factory=list)
    jnt_names: List[str] = field(default_factory=list)
    jnt_type: List[int] = field(default_factory=list)
    jnt_body: List[int] = field(default_factory=list)
    jnt_qposadr: List[int] = field(default_factory=list)
    jnt_dofadr: List[int] = field(default_factory=list)
    jnt_pos: List[tuple] = field(default_factory=list)
    jnt_axis: List[tuple] = field(default_factory=list)
    jnt_limited: List[int] = field(default_factory=list)
    jnt_range: List[tuple] = field(default_factory=list)
    jnt_stiffness: List[float] = field(default_factory=list)
    jnt_springref: List[float] = field(default_factory=list)
    dof_body: List[int] = field(default_factory=list)
    dof_jnt: List[int] = field(default_factory=list)
    dof_parent: List[int] = field(default_factory=list)
    dof_damping: List[float] = field(default_factory=list)
    dof_armature: List[float] = field(default_factory=list)
    geom_names: List[str] = field(default_factory=list)
    geom_type: List[int] = field(default_factory=list)
    geom_body: List[int] = field(default_factory=list)
    geom_pos: List[tuple] = field(default_factory=list)
    geom_quat: List[tuple] = field(default_factory=list)
    geom_size: List[tuple] = field(default_factory=list)
    geom_friction: List[float] = field(default_factory=list)
    geom_contype: List[int] = field(default_factory=list)
    geom_conaffinity: List[int] = field(default_factory=list)
    geom_rgba: List[tuple] = field(default_factory=list)
    geom_dataid: List[int] = field(default_factory=list)
    geom_group: List[int] = field(default_factory=list)
    mesh_names: List[str] = field(default_factory=list)
    mesh_vert: List[list] = field(default_factory=list)     # visual vertices per mesh
    mesh_tri: List[list] = field(default_factory=list)
    hull_vert: List[list] = field(default_factory=list)     # convex hull per mesh
    hull_tri: List[list] = field(default_factory=list)
    cam_names: List[str] = field(default_factory=list)
    cam_body: List[int] = field(default_factory=list)
    cam_pos: List[tuple] = field(default_factory=list)
    cam_quat: List[tuple] = field(default_factory=list)
    cam_fovy: List[float] = field(default_factory=list)
    actuator_names: List[str] = field(default_factory=list)
    actuator_joint: List[int] = field(default_factory=list)
    actuator_gear: List[float] = field(default_factory=list)
    actuator_gain: List[float] = field(default_factory=list)
    actuator_bias: List[tuple] = field(default_factory=list)
    actuator_ctrllimited: List[int] = field(default_factory=list)
    actuator_ctrlrange: List[tuple] = field(default_factory=list)
    actuator_forcelimited: List[int] = field(default_factory=list)
    actuator_forcerange: List[tuple] = field(default_factory=list)
    actuator_moment: List[list] = field(default_factory=list)
    tendon_names: List[str] = field(default_factory=list)
    tendon_joints: List[list] = field(default_factory=list)
    eq_names: List[str] = field(default_factory=list)
    eq_joint1: List[int] = field(default_factory=list)
    eq_joint2: List[int] = field(default_factory=list)
    eq_polycoef: List[tuple] = field(default_factory=list)
    eq_solref: List[tuple] = field(default_factory=list)
    eq_solimp: List[tuple] = field(default_factory=list)
    exclude_pairs: List[tuple] = field(default_factory=list)
    dof_blocks: List[tuple] = field(default_factory=list)
    qpos0: List[float] = field(default_factory=list)
    qpos_reset: List[float] = field(default_factory=list)
    pair_candidates: List[tuple] = field(default_factory=list)
    key_names: List[str] = field(default_factory=list)
    key_qpos: List[list] = field(default_factory=list)
    key_ctrl: List[list] = field(default_factory=list)
    warnings: List[str] = field(default_factory=list)

    @property
    def nbody(self):
        return len(self.body_parent)

    @property
    def njnt(self):
        return len(self.jnt_type)

    @property
    def ngeom(self):
        return len(self.geom_type)

    def body_id(self, name):
        return self.body_names.index(name)

    def geom_id(self, name):
        return self.geom_names.index(name)

    def joint_id(self, name):
        return self.jnt_names.index(name)


# ----------------------------------------------------------------- loader
def _floats(s: str) -> List[float]:
    try:
        return [float(t) for t in s.split()]
    except ValueError as e:
        raise MjcfError(f"bad number in '{s}'") from e


class _Ctx:
    def __init__(self):
        self.materials: Dict[str, tuple] = {}
        self.degrees = True
        self.eulerseq = "xyz"
        self.autolimits = True
        self.defaults: Dict[str, Dict[str, Dict[str, str]]] = {"main": {}}
        self.warnings: List[str] = []

    # mjcf.rs:45-62
    def get(self, node, cls, name):
        v = node.get(name)
        if v is not None:
            return v
        tag = node.tag
        cls = node.get("class", cls)
        dc = self.defaults.get(cls)
        if dc is None:
            return None
        v = dc.get(tag, {}).get(name)
        if v is not None:
            return v
        if tag in ("motor", "position", "velocity"):
            return dc.get("general", {}).get(name)
        return None

    def floats(self, node, cls, name):
        v = self.get(node, cls, name)
        return None if v is None else _floats(v)

    def float(self, node, cls, name, default):
        v = self.floats(node, cls, name)
        return v[0] if v else default

    def vec3(self, node, cls, name, default):
        v = self.floats(node, cls, name)
        if v is None:
            return default
        if len(v) < 3:
            raise MjcfError(f"attribute '{name}' needs 3 numbers")
        return (v[0], v[1], v[2])

    def angle(self, a):
        return a * PI / 180.0 if self.degrees else a

    # mjcf.rs:92-141
    def orientation(self, node, cls):
        q = self.floats(node, cls, "quat")
        if q is not None:
            if len(q) != 4:
                raise MjcfError("quat needs 4 numbers")
            return q_normalized(tuple(q))
        a = self.floats(node, cls, "axisangle")
        if a is not None:
            if len(a) != 4:
                raise MjcfError("axisangle needs 4 numbers")
            return q_axis_angle((a[0], a[1], a[2]), self.angle(a[3]))
        e = self.floats(node, cls, "euler")
        if e is not None:
            if len(e) != 3:
                raise MjcfError("euler needs 3 numbers")
            q = Q_ID
            for i in range(3):
                c = self.eulerseq[i]
                axis = {"x": (1.0, 0.0, 0.0), "y": (0.0, 1.0, 0.0), "z": (0.0, 0.0, 1.0)}.get(c.lower())
                if axis is None:
                    raise MjcfError("bad eulerseq")
                r = q_axis_angle(axis, self.angle(e[i]))
                q = q_mul(q, r) if c.islower() else q_mul(r, q)
            return q_normalized(q)
        x = self.floats(node, cls, "xyaxes")
        if x is not None:
            if len(x) != 6:
                raise MjcfError("xyaxes needs 6 numbers")
            xa = vnormalized((x[0], x[1], x[2]))
            ya = (x[3], x[4], x[5])
            ya = vnormalized(vsub(ya, vscale(xa, vdot(xa, ya))))
            za = vcross(xa, ya)
            return q_from_mat(m_cols(xa, ya, za))
        z = self.floats(node, cls, "zaxis")
        if z is not None:
            if len(z) != 3:
                raise MjcfError("zaxis needs 3 numbers")
            return q_from_z_to((z[0], z[1], z[2]))
        return Q_ID


def _parse_default(ctx: _Ctx, node, parent: str, is_top: bool):
    """mjcf.rs:397-411: each class holds its parents' attributes, overridden."""
    name = "main" if is_top else node.get("class", "main")
    dc = {tag: dict(attrs) for tag, attrs in ctx.defaults.get(parent, {}).items()}
    for c in node:
        if c.tag == "default":
            continue
        dc.setdefault(c.tag, {}).update(c.attrib)
    ctx.defaults[name] = dc
    for c in node:
        if c.tag == "default":
            _parse_default(ctx, c, name, False)


def _geom_volume_inertia(gt, s):
    """Volume and principal inertia per unit density (mjcf.rs:774-808)."""
    if gt in (GEOM_PLANE, GEOM_MESH):
        return 0.0, (0.0, 0.0, 0.0)
    if gt == GEOM_SPHERE:
        r = s[0]
        v = 4.0 / 3.0 * PI * r * r * r
        i = 0.4 * v * r * r
        return v, (i, i, i)
    if gt == GEOM_BOX:
        a, b, c = s
        v = 8.0 * a * b * c
        return v, (v * (b * b + c * c) / 3.0, v * (a * a + c * c) / 3.0, v * (a * a + b * b) / 3.0)
    if gt == GEOM_CYLINDER:
        r, h = s[0], s[1]
        v = PI * r * r * 2.0 * h
        ix = v * (3.0 * r * r + 4.0 * h * h) / 12.0
        return v, (ix, ix, 0.5 * v * r * r)
    # capsule: cylinder plus two hemispheres
    r, h = s[0], s[1]
    vc = PI * r * r * 2.0 * h
    vs = 4.0 / 3.0 * PI * r * r * r
    v = vc + vs
    hs = vs * 0.5
    d = h + 3.0 * r / 8.0
    hs_ix = hs * (83.0 / 320.0) * r * r
    ix = vc * (3.0 * r * r + 4.0 * h * h) / 12.0 + 2.0 * (hs_ix + hs * d * d)
    iz = 0.5 * vc * r * r + 0.4 * vs * r * r
    return v, (ix, ix, iz)


class _Builder:
    def __init__(self, ctx):
        self.ctx = ctx
        self.m = Model()
        self.geom_mass: List[list] = []
        self.explicit_inertial: List[bool] = []

    def add_body(self, name, parent, pos, quat):
        m = self.m
        m.body_names.append(name)
        m.body_parent.append(parent)
        m.body_pos.append(pos)
        m.body_quat.append(quat)
        m.body_jntadr.append(len(m.jnt_type))
        m.body_jntnum.append(0)
        m.body_dofadr.append(m.nv)
        m.body_dofnum.append(0)
        m.body_mass.append(0.0)
        m.body_ipos.append((0.0, 0.0, 0.0))
        m.body_inertia.append((0.0,) * 9)
        self.geom_mass.append([0.0, (0.0, 0.0, 0.0), (0.0,) * 9])
        self.explicit_inertial.append(False)
        return len(m.body_names) - 1

    # mjcf.rs:512-555
    def body_contents(self, node, body, cls):
        ctx, m = self.ctx, self.m
        for c in node:
            if not isinstance(c.tag, str):
                continue
            t = c.tag
            if t == "geom":
                self.geom(c, body, cls)
            elif t in ("joint", "freejoint"):
                if body == 0:
                    raise MjcfError("joints cannot be attached to the world body")
                self.joint(c, body, cls)
            elif t == "inertial":
                self.inertial(c, body, cls)
            elif t == "body":
                name = c.get("name", f"body{m.nbody}")
                pos = ctx.vec3(c, cls, "pos", (0.0, 0.0, 0.0))
                quat = ctx.orientation(c, cls)
                child_cls = c.get("childclass", cls)
                bid = self.add_body(name, body, pos, quat)
                self.body_contents(c, bid, child_cls)
            elif t == "camera":
                cid = len(m.cam_body)
                m.cam_names.append(c.get("name", f"camera{cid}"))
                m.cam_body.append(body)
                m.cam_pos.append(ctx.vec3(c, cls, "pos", (0.0, 0.0, 0.0)))
                m.cam_quat.append(ctx.orientation(c, cls))
                m.cam_fovy.append(ctx.float(c, cls, "fovy", 45.0))
            elif t in ("site", "light", "include"):
                pass
            else:
                ctx.warnings.append(f"<{t}> inside body is not supported")

    # mjcf.rs:559-633
    def joint(self, node, body, cls):
        ctx, m = self.ctx, self.m
        if node.tag == "freejoint":
            jt = JNT_FREE
        else:
            tname = ctx.get(node, cls, "type") or "hinge"
            jt = {"free": JNT_FREE, "ball": JNT_BALL, "slide": JNT_SLIDE, "hinge": JNT_HINGE}.get(tname)
            if jt is None:
                raise MjcfError(f"unknown joint type '{tname}'")
        jid = len(m.jnt_type)
        name = node.get("name", f"joint{jid}")
        pos = (0.0, 0.0, 0.0) if jt == JNT_FREE else ctx.vec3(node, cls, "pos", (0.0, 0.0, 0.0))
        axis = vnormalized(ctx.vec3(node, cls, "axis", (0.0, 0.0, 1.0)))
        rng = ctx.floats(node, cls, "range")
        lim = ctx.get(node, cls, "limited")
        if lim == "true":
            limited = True
        elif lim == "false":
            limited = False
        else:
            limited = ctx.autolimits and rng is not None
        limited = limited and jt in (JNT_HINGE, JNT_SLIDE)
        rng = (rng[0], rng[1]) if rng is not None else (0.0, 0.0)
        angular = jt == JNT_HINGE
        if angular:
            rng = (ctx.angle(rng[0]), ctx.angle(rng[1]))
        refv = ctx.float(node, cls, "ref", 0.0)
        springref = ctx.float(node, cls, "springref", 0.0)
        if angular:
            refv = ctx.angle(refv)
            springref = ctx.angle(springref)
        damping = ctx.float(node, cls, "damping", 0.0)
        armature = ctx.float(node, cls, "armature", 0.0)
        stiffness = ctx.float(node, cls, "stiffness", 0.0)
        m.jnt_names.append(name)
        m.jnt_type.append(jt)
        m.jnt_body.append(body)
        m.jnt_qposadr.append(m.nq)
        m.jnt_dofadr.append(m.nv)
        m.jnt_pos.append(pos)
        m.jnt_axis.append(axis)
        m.jnt_limited.append(1 if limited else 0)
        m.jnt_range.append(rng)
        m.jnt_stiffness.append(stiffness)
        m.jnt_springref.append(springref)
        if jt == JNT_FREE:
            p, q = m.body_pos[body], m.body_quat[body]
            m.qpos0.extend([p[0], p[1], p[2], q[0], q[1], q[2], q[3]])
        elif jt == JNT_BALL:
            m.qpos0.extend([1.0, 0.0, 0.0, 0.0])
        else:
            m.qpos0.append(refv)
        nvj = {JNT_FREE: 6, JNT_BALL: 3}.get(jt, 1)
        nqj = {JNT_FREE: 7, JNT_BALL: 4}.get(jt, 1)
        for _ in range(nvj):
            m.dof_body.append(body)
            m.dof_jnt.append(jid)
            m.dof_damping.append(damping)
            m.dof_armature.append(armature)
        m.nq += nqj
        m.nv += nvj
        m.body_jntnum[body] += 1
        m.body_dofnum[body] += nvj
        if m.body_jntnum[body] == 1:
            m.body_jntadr[body] = jid
            m.body_dofadr[body] = m.jnt_dofadr[jid]

    # mjcf.rs:635-738
    def geom(self, node, body, cls):
        ctx, m = self.ctx, self.m
        tname = ctx.get(node, cls, "type") or "sphere"
        gt = GEOM_TYPES.get(tname)
        if gt is None:
            ctx.warnings.append(f"geom type '{tname}' not supported yet; geom skipped")
            return
        sz = ctx.floats(node, cls, "size") or []

        def g(i):
            return sz[i] if i < len(sz) else 0.0

        size = (g(0), g(1), g(2))
        pos = ctx.vec3(node, cls, "pos", (0.0, 0.0, 0.0))
        quat = ctx.orientation(node, cls)
        ft = ctx.floats(node, cls, "fromto")
        if ft is not None:
            if len(ft) != 6:
                raise MjcfError("fromto needs 6 numbers")
            a, b = (ft[0], ft[1], ft[2]), (ft[3], ft[4], ft[5])
            d = vsub(b, a)
            pos = vscale(vadd(a, b), 0.5)
            quat = q_from_z_to(d)
            if gt in (GEOM_CAPSULE, GEOM_CYLINDER):
                size = (g(0), vnorm(d) * 0.5, 0.0)
            elif gt == GEOM_BOX:
                size = (g(0), g(1), vnorm(d) * 0.5)
            else:
                raise MjcfError("fromto only valid for capsule, cylinder, box")
        fr = ctx.floats(node, cls, "friction")
        friction = fr[0] if fr else 1.0
        contype = _as_u32(ctx.float(node, cls, "contype", 1.0))
        conaffinity = _as_u32(ctx.float(node, cls, "conaffinity", 1.0))
        rgba = ctx.floats(node, cls, "rgba")
        if rgba is not None and len(rgba) == 4:
            rgba = tuple(_f32(x) for x in rgba)
        else:
            mat = ctx.get(node, cls, "material")
            rgba = ctx.materials.get(mat) if mat is not None else None
        group = int(ctx.float(node, cls, "group", 0.0))
        dataid = -1
        if gt == GEOM_MESH:
            mname = ctx.get(node, cls, "mesh")
            if mname is None:
                raise MjcfError("mesh geom needs a 'mesh' attribute")
            if mname not in m.mesh_names:
                raise MjcfError(f"unknown mesh '{mname}'")
            dataid = m.mesh_names.index(mname)
        e = self.geom_mass[body]
        if gt == GEOM_MESH:
            vol, com, icom = mesh_mass_properties(m.hull_vert[dataid], m.hull_tri[dataid])
            mv = ctx.floats(node, cls, "mass")
            mass = mv[0] if mv is not None else ctx.float(node, cls, "density", 1000.0) * vol
            if mass > 0.0 and vol > 0.0:
                r = q_to_mat(quat)
                c = vadd(pos, m_vec(r, com))
                ig = m_rotate(m_scale(icom, mass / vol), r)
                cc = m_skew(c)
                shifted = m_add(ig, m_scale(m_mul(cc, m_t(cc)), mass))
                e[0] += mass
                e[1] = vadd(e[1], vscale(c, mass))
                e[2] = m_add(e[2], shifted)
        elif gt != GEOM_PLANE:
            vol, unit = _geom_volume_inertia(gt, size)
            mv = ctx.floats(node, cls, "mass")
            mass = mv[0] if mv is not None else ctx.float(node, cls, "density", 1000.0) * vol
            if mass > 0.0 and vol > 0.0:
                ig = m_rotate(m_diag(vscale(unit, mass / vol)), q_to_mat(quat))
                pp = m_skew(pos)
                shifted = m_add(ig, m_scale(m_mul(pp, m_t(pp)), mass))
                e[0] += mass
                e[1] = vadd(e[1], vscale(pos, mass))
                e[2] = m_add(e[2], shifted)
        gid = len(m.geom_type)
        m.geom_names.append(node.get("name", f"geom{gid}"))
        m.geom_type.append(gt)
        m.geom_body.append(body)
        m.geom_pos.append(pos)
        m.geom_quat.append(quat)
        m.geom_size.append(size)
        m.geom_friction.append(friction)
        m.geom_contype.append(contype)
        m.geom_conaffinity.append(conaffinity)
        m.geom_rgba.append(rgba if rgba is not None else (0.5, 0.5, 0.5, 1.0))
        m.geom_dataid.append(dataid)
        m.geom_group.append(group)

    # mjcf.rs:810-827
    def inertial(self, node, body, cls):
        ctx, m = self.ctx, self.m
        pos = ctx.vec3(node, cls, "pos", (0.0, 0.0, 0.0))
        quat = ctx.orientation(node, cls)
        mass = ctx.float(node, cls, "mass", 0.0)
        d = ctx.floats(node, cls, "diaginertia")
        f = ctx.floats(node, cls, "fullinertia")
        if d is not None:
            inertia = m_rotate(m_diag((d[0], d[1], d[2])), q_to_mat(quat))
        elif f is not None:
            inertia = m_rotate((f[0], f[3], f[4], f[3], f[1], f[5], f[4], f[5], f[2]), q_to_mat(quat))
        else:
            raise MjcfError("<inertial> requires diaginertia or fullinertia")
        m.body_mass[body] = mass
        m.body_ipos[body] = pos
        m.body_inertia[body] = inertia
        self.explicit_inertial[body] = True

    # mjcf.rs:829-850
    def finalize_inertia(self):
        m = self.m
        for b in range(1, m.nbody):
            if self.explicit_inertial[b]:
                continue
            mass, mc, second = self.geom_mass[b]
            if mass <= 0.0:
                if m.body_jntnum[b] > 0:
                    raise MjcfError(f"moving body '{m.body_names[b]}' has no mass")
                continue
            com = vscale(mc, 1.0 / mass)
            cx = m_skew(com)
            icom = m_add(second, m_scale(m_mul(cx, m_t(cx)), -mass))
            m.body_mass[b] = mass
            m.body_ipos[b] = com
            m.body_inertia[b] = icom


def _as_u32(x: float) -> int:
    """Rust `f64 as u32`: truncate toward zero, saturate, NaN -> 0."""
    if x != x or x <= 0:
        return 0
    return min(int(x), 0xFFFFFFFF)


def _f32(x: float) -> float:
    return struct.unpack("<f", struct.pack("<f", x))[0]


def _parse_mesh(ctx: _Ctx, m: Model, node, meshdir: str):
    """mjcf.rs:740-772 (point-cloud `vertex` meshes and OBJ files)."""
    f = node.get("file")
    name = node.get("name")
    if name is None and f is not None:
        import os
        name = os.path.splitext(os.path.basename(f))[0]
    if name is None:
        raise MjcfError("mesh needs a name or file")
    if f is not None:
        import os
        verts, tris = _load_obj(os.path.join(meshdir, f))
    else:
        v = ctx.floats(node, "main", "vertex")
        if v is None:
            raise MjcfError(f"mesh '{name}' needs 'file' or 'vertex'")
        verts = [(v[i], v[i + 1], v[i + 2]) for i in range(0, len(v) - 2, 3)]
        tris = []
    scale = ctx.vec3(node, "main", "scale", (1.0, 1.0, 1.0))
    verts = [(p[0] * scale[0], p[1] * scale[1], p[2] * scale[2]) for p in verts]
    hv, ht = convex_hull(verts)
    if not tris:
        verts, tris = hv, ht
    m.mesh_names.append(name)
    m.mesh_vert.append(verts)
    m.mesh_tri.append(tris)
    m.hull_vert.append(hv)
    m.hull_tri.append(ht)


def _load_obj(path):
    verts, tris = [], []
    with open(path) as fh:
        for line in fh:
            p = line.split()
            if not p:
                continue
            if p[0] == "v":
                verts.append((float(p[1]), float(p[2]), float(p[3])))
            elif p[0] == "f":
                idx = [int(t.split("/")[0]) - 1 for t in p[1:]]
                for k in range(1, len(idx) - 1):
                    tris.append((idx[0], idx[k], idx[k + 1]))
    return verts, tris


def _parse_actuator(ctx: _Ctx, m: Model, node):
    """mjcf.rs:852-921 (joint and fixed-tendon transmissions)."""
    tag = node.tag
    if tag not in ("motor", "position", "velocity", "general"):
        raise MjcfError(f"actuator <{tag}> not supported")
    cls = "main"
    if node.get("joint") is not None:
        jn = node.get("joint")
        if jn not in m.jnt_names:
            raise MjcfError(f"actuator references unknown joint '{jn}'")
        j = m.jnt_names.index(jn)
        if m.jnt_type[j] not in (JNT_HINGE, JNT_SLIDE):
            raise MjcfError("actuators on free/ball joints are not supported")
        moment = [(j, 1.0)]
    elif node.get("tendon") is not None:
        tn = node.get("tendon")
        if tn not in m.tendon_names:
            raise MjcfError(f"actuator references unknown tendon '{tn}'")
        moment = list(m.tendon_joints[m.tendon_names.index(tn)])
    else:
        raise MjcfError("only joint and fixed-tendon transmissions are supported")
    gear = ctx.float(node, cls, "gear", 1.0)
    if tag == "motor":
        gain, bias = 1.0, (0.0, 0.0, 0.0)
    elif tag == "position":
        kp = ctx.float(node, cls, "kp", 1.0)
        kv = ctx.float(node, cls, "kv", 0.0)
        gain, bias = kp, (0.0, -kp, -kv)
    elif tag == "velocity":
        kv = ctx.float(node, cls, "kv", 1.0)
        gain, bias = kv, (0.0, 0.0, -kv)
    else:
        gp = ctx.floats(node, cls, "gainprm")
        gain = gp[0] if gp else 1.0
        bp = ctx.floats(node, cls, "biasprm") or []
        if ctx.get(node, cls, "biastype") == "affine":
            bias = tuple(bp[i] if i < len(bp) else 0.0 for i in range(3))
        else:
            bias = (0.0, 0.0, 0.0)

    def limited(flag, rname):
        r = ctx.floats(node, cls, rname)
        f = ctx.get(node, cls, flag)
        lim = True if f == "true" else False if f == "false" else (ctx.autolimits and r is not None)
        return (1 if lim else 0), ((r[0], r[1]) if r is not None else (0.0, 0.0))

    cl, cr = limited("ctrllimited", "ctrlrange")
    fl, fr = limited("forcelimited", "forcerange")
    idx = len(m.actuator_joint)
    m.actuator_names.append(node.get("name", f"actuator{idx}"))
    m.actuator_joint.append(moment[0][0])
    m.actuator_gear.append(gear)
    m.actuator_gain.append(gain)
    m.actuator_bias.append(bias)
    m.actuator_ctrllimited.append(cl)
    m.actuator_ctrlrange.append(cr)
    m.actuator_forcelimited.append(fl)
    m.actuator_forcerange.append(fr)
    m.actuator_moment.append(moment)


def _parse_tendon(ctx: _Ctx, m: Model, node):
    """mjcf.rs:923-947 (fixed tendons only)."""
    if node.tag != "fixed":
        ctx.warnings.append(f"<tendon><{node.tag}> is not supported yet and was ignored")
        return
    joints = []
    for jn in node.findall("joint"):
        name = jn.get("joint", "")
        if name not in m.jnt_names:
            raise MjcfError(f"tendon references unknown joint '{name}'")
        j = m.jnt_names.index(name)
        if m.jnt_type[j] not in (JNT_HINGE, JNT_SLIDE):
            raise MjcfError("fixed tendons need hinge or slide joints")
        coef = _floats(jn.get("coef"))[0] if jn.get("coef") is not None else 1.0
        joints.append((j, coef))
    if not joints:
        raise MjcfError("fixed tendon needs at least one joint")
    tid = len(m.tendon_names)
    m.tendon_names.append(node.get("name", f"tendon{tid}"))
    m.tendon_joints.append(joints)


def _parse_equality(ctx: _Ctx, m: Model, node):
    """mjcf.rs:949-998 (joint equality)."""
    if node.tag != "joint":
        ctx.warnings.append(f"<equality><{node.tag}> is not supported yet and was ignored")
        return
    if node.get("active") == "false":
        return

    def get(name):
        v = node.get(name)
        if v is not None:
            return v
        cls = node.get("class", "main")
        return ctx.defaults.get(cls, {}).get("equality", {}).get(name)

    def joint(a):
        name = node.get(a, "")
        if name not in m.jnt_names:
            raise MjcfError(f"equality references unknown joint '{name}'")
        j = m.jnt_names.index(name)
        if m.jnt_type[j] not in (JNT_HINGE, JNT_SLIDE):
            raise MjcfError("joint equality needs hinge or slide joints")
        return j

    j1 = joint("joint1")
    j2 = joint("joint2") if node.get("joint2") is not None else -1
    poly = [0.0, 1.0, 0.0, 0.0, 0.0]
    if get("polycoef") is not None:
        for k, x in enumerate(_floats(get("polycoef"))[:5]):
            poly[k] = x
    solref = m.solref
    if get("solref") is not None:
        r = _floats(get("solref"))
        solref = (r[0], r[1] if len(r) > 1 else 1.0)
    solimp = list(m.solimp)
    if get("solimp") is not None:
        for k, x in enumerate(_floats(get("solimp"))[:5]):
            solimp[k] = x
    eid = len(m.eq_names)
    m.eq_names.append(node.get("name", f"equality{eid}"))
    m.eq_joint1.append(j1)
    m.eq_joint2.append(j2)
    m.eq_polycoef.append(tuple(poly))
    m.eq_solref.append(tuple(solref))
    m.eq_solimp.append(tuple(solimp))


def load_string(xml: str, asset_dir: str = ".") -> Model:
    """Parse and compile an MJCF string (mjcf.rs:211-395 + model.rs:279-316)."""
    try:
        root = ET.fromstring(xml)
    except ET.ParseError as e:
        raise MjcfError(f"xml parse error: {e}") from e
    if root.tag != "mujoco":
        raise MjcfError("root element must be <mujoco>")
    ctx = _Ctx()
    meshdir = asset_dir
    for c in root.findall("compiler"):
        if c.get("angle") is not None:
            ctx.degrees = c.get("angle") == "degree"
        if c.get("eulerseq") is not None:
            if len(c.get("eulerseq")) != 3:
                raise MjcfError("eulerseq must have 3 characters")
            ctx.eulerseq = c.get("eulerseq")
        if c.get("autolimits") is not None:
            ctx.autolimits = c.get("autolimits") == "true"
        d = c.get("meshdir") or c.get("assetdir")
        if d is not None:
            import os
            meshdir = os.path.join(asset_dir, d)
    for d in root.findall("default"):
        _parse_default(ctx, d, "main", True)

    b = _Builder(ctx)
    m = b.m
    for o in root.findall("option"):
        if o.get("timestep") is not None:
            m.timestep = _floats(o.get("timestep"))[0]
        if o.get("gravity") is not None:
            g = _floats(o.get("gravity"))
            m.gravity = (g[0], g[1], g[2])
        if o.get("solver") is not None:
            s = o.get("solver")
            if s == "Newton":
                m.solver = 0
            elif s == "PGS":
                m.solver = 1
            else:
                ctx.warnings.append(f"solver '{s}' not supported, using Newton")
                m.solver = 0
        if o.get("impratio") is not None:
            m.impratio = _floats(o.get("impratio"))[0]
        if o.get("cone") is not None and o.get("cone") != "pyramidal":
            ctx.warnings.append(f"cone '{o.get('cone')}' not supported, using pyramidal")
        if o.get("tolerance") is not None:
            m.tolerance = _floats(o.get("tolerance"))[0]
        if o.get("o_solref") is not None:
            r = _floats(o.get("o_solref"))
            m.solref = (r[0], r[1])
        if o.get("iterations") is not None:
            m.iterations = int(_floats(o.get("iterations"))[0])
        if o.get("integrator") is not None:
            it = o.get("integrator")
            if it == "Euler":
                m.integrator = 0
            elif it in ("implicitfast", "implicit"):
                m.integrator = 1
            else:
                ctx.warnings.append(f"integrator '{it}' not supported, using Euler")
                m.integrator = 0
    for a in root.findall("asset"):
        for mesh in a.findall("mesh"):
            _parse_mesh(ctx, m, mesh, meshdir)
        for mat in a.findall("material"):
            rgba = ctx.floats(mat, mat.get("class", "main"), "rgba")
            if mat.get("name") is not None and rgba is not None and len(rgba) == 4:
                ctx.materials[mat.get("name")] = tuple(_f32(x) for x in rgba)
    b.add_body("world", 0, (0.0, 0.0, 0.0), Q_ID)
    worlds = root.findall("worldbody")
    if not worlds:
        raise MjcfError("missing <worldbody>")
    for w in worlds:
        b.body_contents(w, 0, "main")
    b.finalize_inertia()
    for t in root.findall("tendon"):
        for c in t:
            _parse_tendon(ctx, m, c)
    for act in root.findall("actuator"):
        for a in act:
            _parse_actuator(ctx, m, a)
    m.nu = len(m.actuator_joint)
    for e in root.findall("equality"):
        for c in e:
            _parse_equality(ctx, m, c)
    for c in root.findall("contact"):
        for x in c:
            if x.tag == "exclude":
                def bid(attr):
                    name = x.get(attr)
                    if name is None:
                        raise MjcfError(f"<exclude> needs {attr}")
                    if name not in m.body_names:
                        raise MjcfError(f"<exclude> references unknown body '{name}'")
                    return m.body_names.index(name)
                m.exclude_pairs.append((bid("body1"), bid("body2")))
            else:
                ctx.warnings.append(f"<contact><{x.tag}> is not supported yet and was ignored")
    for k in root.findall("keyframe"):
        for key in k.findall("key"):
            qpos = _floats(key.get("qpos")) if key.get("qpos") is not None else list(m.qpos0)
            ctrl = _floats(key.get("ctrl")) if key.get("ctrl") is not None else [0.0] * m.nu
            if len(qpos) != m.nq or len(ctrl) != m.nu:
                raise MjcfError(f"keyframe needs {m.nq} qpos and {m.nu} ctrl values")
            m.key_names.append(key.get("name", ""))
            m.key_qpos.append(qpos)
            m.key_ctrl.append(ctrl)
    m.warnings = ctx.warnings
    _compile(m)
    return m


def load_file(path: str) -> Model:
    import os
    with open(path) as fh:
        return load_string(fh.read(), os.path.dirname(os.path.abspath(path)))


# ----------------------------------------------------------------- compile (model.rs:279-451)
def _compile(m: Model):
    if len(m.qpos_reset) != len(m.qpos0):
        m.qpos_reset = list(m.qpos0)
    nb = m.nbody
    m.body_lastdof = [-1] * nb
    m.dof_parent = [-1] * m.nv
    for b in range(1, nb):
        last = m.body_lastdof[m.body_parent[b]]
        for k in range(m.body_dofnum[b]):
            d = m.body_dofadr[b] + k
            m.dof_parent[d] = last
            last = d
        m.body_lastdof[b] = last
    m.dof_blocks = _dof_blocks(m)
    m.body_weldid = list(range(nb))
    for b in range(1, nb):
        if m.body_jntnum[b] == 0:
            m.body_weldid[b] = m.body_weldid[m.body_parent[b]]
    m.pair_candidates = []
    for g1 in range(m.ngeom):
        for g2 in range(g1 + 1, m.ngeom):
            if _static_pair(m, g1, g2):
                m.pair_candidates.append((g1, g2))
    if m.hertz <= 0.0:
        m.hertz = 0.25 / m.timestep


def _dof_blocks(m: Model):
    """model.rs:318-363: one block per tree, merged across tendon actuators."""
    nv = m.nv
    root = list(range(nv))
    for k in range(nv):
        r = k
        while m.dof_parent[r] != -1:
            r = m.dof_parent[r]
        root[k] = r
    group = list(root)

    def find(x):
        while group[x] != x:
            x = group[x]
        return x

    for moment in m.actuator_moment:
        dofs = [m.jnt_dofadr[j] for j, _ in moment]
        for a, b in zip(dofs, dofs[1:]):
            ra, rb = find(root[a]), find(root[b])
            if ra != rb:
                group[max(ra, rb)] = min(ra, rb)
    gid = [find(root[k]) for k in range(nv)]
    blocks, seen, k = [], set(), 0
    while k < nv:
        e = k + 1
        while e < nv and gid[e] == gid[k]:
            e += 1
        if gid[k] in seen:
            return [(0, nv)] if nv > 0 else []
        seen.add(gid[k])
        blocks.append((k, e))
        k = e
    return blocks


def _static_pair(m: Model, g1: int, g2: int) -> bool:
    """model.rs:430-451 without the contype/conaffinity test (applied per env)."""
    b1, b2 = m.geom_body[g1], m.geom_body[g2]
    for a, b in m.exclude_pairs:
        if (a, b) == (b1, b2) or (a, b) == (b2, b1):
            return False
    w1, w2 = m.body_weldid[b1], m.body_weldid[b2]
    if w1 == w2:
        return False
    p1 = m.body_weldid[m.body_parent[w1]]
    p2 = m.body_weldid[m.body_parent[w2]]
    if (p1 == w2 and w2 != 0) or (p2 == w1 and w1 != 0):
        return False
    return not (m.geom_type[g1] == GEOM_PLANE and m.geom_type[g2] == GEOM_PLANE)


def collision_pairs(m: Model) -> List[Tuple[int, int]]:
    """Candidates filtered by the base contype/conaffinity masks."""
    return [(a, b) for a, b in m.pair_candidates
            if (m.geom_contype[a] & m.geom_conaffinity[b]) or (m.geom_contype[b] & m.geom_conaffinity[a])]


# ----------------------------------------------------------------- blob writer
F64, I64, U8 = 1, 2, 3


def _flat(rows):
    out = []
    for r in rows:
        if isinstance(r, (tuple, list)):
            out.extend(r)
        else:
            out.append(r)
    return out


def to_blob(m: Model) -> bytes:
    """Serialise to the model blob of include/pippin_b200.h."""
    import numpy as np

    arrays = []

    def f(name, vals):
        arrays.append((name, F64, np.asarray(_flat(vals), dtype="<f8").tobytes(), len(_flat(vals))))

    def i(name, vals):
        arrays.append((name, I64, np.asarray(_flat(vals), dtype="<i8").tobytes(), len(_flat(vals))))

    def names(name, vals):
        raw = b"\0".join(v.encode() for v in vals) + (b"\0" if vals else b"")
        arrays.append((name, U8, raw, len(raw)))

    f("timestep", [m.timestep])
    f("gravity", m.gravity)
    i("integrator", [m.integrator])
    i("opt_solver", [m.solver])
    i("opt_iterations", [m.iterations])
    f("opt_tolerance", [m.tolerance])
    f("opt_margin", [m.margin])
    f("opt_solref", m.solref)
    f("opt_solimp", m.solimp)
    f("opt_impratio", [m.impratio])
    f("opt_hertz", [m.hertz])
    f("opt_dampratio", [m.dampratio])
    f("opt_slop", [m.slop])
    i("dims", [m.nq, m.nv, m.nu, m.nbody, m.njnt, m.ngeom, len(m.cam_body), len(m.eq_joint1), len(m.mesh_names)])
    for nm in ("body_parent", "body_jntadr", "body_jntnum", "body_dofadr", "body_dofnum", "body_lastdof",
               "body_weldid"):
        i(nm, getattr(m, nm))
    for nm in ("body_pos", "body_quat", "body_mass", "body_ipos", "body_inertia"):
        f(nm, getattr(m, nm))
    for nm in ("jnt_type", "jnt_body", "jnt_qposadr", "jnt_dofadr", "jnt_limited"):
        i(nm, getattr(m, nm))
    for nm in ("jnt_pos", "jnt_axis", "jnt_range", "jnt_stiffness", "jnt_springref"):
        f(nm, getattr(m, nm))
    for nm in ("dof_body", "dof_jnt", "dof_parent"):
        i(nm, getattr(m, nm))
    for nm in ("dof_damping", "dof_armature"):
        f(nm, getattr(m, nm))
    for nm in ("geom_type", "geom_body", "geom_dataid", "geom_group", "geom_contype", "geom_conaffinity"):
        i(nm, getattr(m, nm))
    for nm in ("geom_pos", "geom_quat", "geom_size", "geom_friction", "geom_rgba"):
        f(nm, getattr(m, nm))
    i("cam_body", m.cam_body)
    f("cam_pos", m.cam_pos)
    f("cam_quat", m.cam_quat)
    f("cam_fovy", m.cam_fovy)
    i("actuator_joint", m.actuator_joint)
    i("actuator_ctrllimited", m.actuator_ctrllimited)
    i("actuator_forcelimited", m.actuator_forcelimited)
    f("actuator_gear", m.actuator_gear)
    f("actuator_gain", m.actuator_gain)
    f("actuator_bias", m.actuator_bias)
    f("actuator_ctrlrange", m.actuator_ctrlrange)
    f("actuator_forcerange", m.actuator_forcerange)
    adr, num, mj, mc = [], [], [], []
    for mom in m.actuator_moment:
        adr.append(len(mj))
        num.append(len(mom))
        for j, c in mom:
            mj.append(j)
            mc.append(c)
    i("actuator_moment_adr", adr)
    i("actuator_moment_num", num)
    i("moment_jnt", mj)
    f("moment_coef", mc)
    i("eq_joint1", m.eq_joint1)
    i("eq_joint2", m.eq_joint2)
    f("eq_polycoef", m.eq_polycoef)
    f("eq_solref", m.eq_solref)
    f("eq_solimp", m.eq_solimp)
    i("dof_blocks", m.dof_blocks)
    i("pair_candidates", m.pair_candidates)
    f("qpos0", m.qpos0)
    f("qpos_reset", m.qpos_reset)
    for pre, vs, ts in (("hull", m.hull_vert, m.hull_tri), ("mesh", m.mesh_vert, m.mesh_tri)):
        va, vn, flat_v, ta, tn, flat_t = [], [], [], [], [], []
        for v, t in zip(vs, ts):
            va.append(len(flat_v) // 3)
            vn.append(len(v))
            flat_v.extend(_flat(v))
            ta.append(len(flat_t) // 3)
            tn.append(len(t))
            flat_t.extend(_flat(t))
        i(f"{pre}_vert_adr", va)
        i(f"{pre}_vert_num", vn)
        f(f"{pre}_vert", flat_v)
        i(f"{pre}_tri_adr", ta)
        i(f"{pre}_tri_num", tn)
        i(f"{pre}_tri", flat_t)
    # polygon faces and edges of each hull (general convex narrow phase)
    fa, fn, fplane, fva, fvn, fverts, ea, en, flat_e = [], [], [], [], [], [], [], [], []
    for v, t in zip(m.hull_vert, m.hull_tri):
        faces, edges = hull_features(v, t)
        fa.append(len(fplane) // 4)
        fn.append(len(faces))
        for nrm, d, loop in faces:
            fplane.extend([nrm[0], nrm[1], nrm[2], d])
            fva.append(len(fverts))
            fvn.append(len(loop))
            fverts.extend(loop)
        ea.append(len(flat_e) // 2)
        en.append(len(edges))
        flat_e.extend(_flat(edges))
    i("hull_face_adr", fa)
    i("hull_face_num", fn)
    f("hull_face_plane", fplane)
    i("hull_face_vert_adr", fva)
    i("hull_face_vert_num", fvn)
    i("hull_face_vert", fverts)
    i("hull_edge_adr", ea)
    i("hull_edge_num", en)
    i("hull_edge", flat_e)
    names("names_body", m.body_names)
    names("names_jnt", m.jnt_names)
    names("names_geom", m.geom_names)
    names("names_cam", m.cam_names)
    names("names_actuator", m.actuator_names)
    names("names_mesh", m.mesh_names)

    n = len(arrays)
    header = bytearray(b"PGBLOB01" + struct.pack("<II", 1, n))
    offset = 16 + 64 * n
    body = bytearray()
    entries = bytearray()
    for name, dt, raw, count in arrays:
        enc = name.encode()
        assert len(enc) < 40
        pad = (-(offset + len(body))) % 8
        body.extend(b"\0" * pad)
        entries.extend(enc + b"\0" * (40 - len(enc)))
        entries.extend(struct.pack("<IIQQ", dt, 0, count, offset + len(body)))
        body.extend(raw)
    return bytes(header + entries + body)


def compile_string(xml: str, asset_dir: str = ".") -> bytes:
    return to_blob(load_string(xml, asset_dir))


def compile_file(path: str) -> bytes:
    return to_blob(load_file(path))
