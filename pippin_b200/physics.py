"""The CUDA backend behind the reference's `Physics` trait, for Python.

`CudaPhysics` mirrors `trait Physics` (crates/pippin-env/src/lib.rs:109-155)
method for method, with the semantics of the CPU backend it replaces
(crates/pippin-env/src/pippin_cpu.rs:14-206): env ranges are Python
`range`s (or (start, end) pairs), state is row-major (envs, width) float64,
poses are (envs, ngeom, 12) float32 (`pos[3]` then row-major `mat[9]`),
buffer-size mismatches raise (where the reference's check_len panics) and
`set_param` errors raise `PhysicsError` carrying the backend's message.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _native
from ._native import PgGeomVisual, PgModelDims


class PhysicsError(ValueError):
    """A call the backend rejected (bad range, id, width or value)."""


class Field(enum.IntEnum):
    """crates/pippin-env/src/lib.rs:20-26 (+ the Newton warm start and
    applied forces, crates/pippin/src/batch.rs:98-104)."""
    QPOS = 0
    QVEL = 1
    CTRL = 2
    QACC = 3
    QFRC_APPLIED = 4


class Param(enum.IntEnum):
    """crates/pippin/src/params.rs:10-39."""
    GEOM_FRICTION = 0
    GEOM_SIZE = 1
    GEOM_RGBA = 2
    GEOM_CONTYPE = 3
    GEOM_CONAFFINITY = 4
    BODY_MASS = 5
    DOF_DAMPING = 6
    ACTUATOR_GAIN = 7
    ACTUATOR_BIAS = 8
    BODY_INERTIA = 9
    BODY_IPOS = 10
    QPOS0 = 11

    @staticmethod
    def from_name(name: str) -> Optional["Param"]:
        """params.rs:42-58."""
        try:
            return Param[name.upper()]
        except KeyError:
            return None


class Solver(enum.IntEnum):
    NEWTON = 0
    PGS = 1


class WarmStart(enum.IntEnum):
    REF_PREV_QACC = 0
    COLD = 1
    LEARNED = 2


class Shape(enum.IntEnum):
    PLANE = 0
    SPHERE = 1
    CAPSULE = 2
    BOX = 3
    CYLINDER = 4
    MESH = 5


@dataclass
class Dims:
    """crates/pippin-env/src/lib.rs:28-36."""
    nq: int
    nv: int
    nu: int
    ngeom: int
    ncam: int

    def width(self, f: Field) -> int:
        return {Field.QPOS: self.nq, Field.QVEL: self.nv, Field.CTRL: self.nu, Field.QACC: self.nv,
                Field.QFRC_APPLIED: self.nv}[Field(f)]


@dataclass
class GeomVisual:
    name: str
    shape: Shape
    mesh: Optional[int]
    size: Tuple[float, float, float]
    rgba: Tuple[float, float, float, float]
    body: int
    group: int


@dataclass
class Mesh:
    name: str
    vertices: np.ndarray   # (n, 3) float32
    triangles: np.ndarray  # (m, 3) uint32


@dataclass
class CameraDesc:
    name: str
    fovy: float


@dataclass
class Scene:
    """crates/pippin-env/src/lib.rs:80-86."""
    bodies: List[str] = field(default_factory=list)
    geoms: List[GeomVisual] = field(default_factory=list)
    meshes: List[Mesh] = field(default_factory=list)
    cameras: List[CameraDesc] = field(default_factory=list)


EnvRange = Union[range, Tuple[int, int]]


def fp64_peak(device: int = 0, iters: int = 4000) -> float:
    """Measured FP64 FMA throughput of `device` in TFLOP/s (pg_fp64_peak)."""
    L = _native.load()
    t, ms = C.c_double(), C.c_double()
    if L.pg_fp64_peak(int(device), int(iters), C.byref(t), C.byref(ms)) != 0:
        raise PhysicsError("FP64 peak measurement failed")
    return t.value


def _span(envs: EnvRange) -> Tuple[int, int]:
    if isinstance(envs, range):
        if envs.step != 1:
            raise PhysicsError("env ranges must be contiguous")
        return envs.start, envs.stop
    s, e = envs
    return int(s), int(e)


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class _DeviceArray:
    """__cuda_array_interface__ over FP64 device memory a CudaPhysics owns
    (it holds the owner, so torch's reference to it keeps the handle alive)."""

    def __init__(self, ptr: int, shape, owner):
        self.owner = owner
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (int(ptr), False),
                                         "strides": None, "version": 2}


class CudaPhysics:
    """A batch of environments stepped on one GPU by the sm_100a kernels."""

    def __init__(self, model: Union[bytes, str], num_envs: int, device: int = 0):
        if isinstance(model, str):
            from . import mjcf
            blob = mjcf.compile_string(model) if model.lstrip().startswith("<") else mjcf.compile_file(model)
        else:
            blob = bytes(model)
        self._L = _native.load()
        self._blob = blob
        h = C.c_void_p()
        self._check(self._L.pg_create(blob, len(blob), int(num_envs), int(device), C.byref(h)))
        self._h = h
        d = PgModelDims()
        self._check(self._L.pg_dims(self._h, C.byref(d)))
        self._dims = Dims(d.nq, d.nv, d.nu, d.ngeom, d.ncam)
        self.nbody, self.njnt = d.nbody, d.njnt
        self._n = int(num_envs)
        self._device = int(device)

    # ---- plumbing
    def _check(self, rc: int):
        if rc != 0:
            raise PhysicsError(_native.last_error() or f"pippin_b200 error {rc}")

    def close(self):
        if getattr(self, "_h", None):
            self._L.pg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- Physics trait (lib.rs:109-155)
    def name(self) -> str:
        return self._L.pg_name(self._h).decode()

    def num_envs(self) -> int:
        return self._n

    def dims(self) -> Dims:
        return self._dims

    def scene(self) -> Scene:
        nb, ng, nm, nc = (C.c_int64() for _ in range(4))
        self._check(self._L.pg_scene_counts(self._h, C.byref(nb), C.byref(ng), C.byref(nm), C.byref(nc)))
        gv = (PgGeomVisual * max(ng.value, 1))()
        self._check(self._L.pg_scene_geoms(self._h, gv, ng.value))
        geoms = []
        for g in range(ng.value):
            v = gv[g]
            geoms.append(GeomVisual(self._name(1, g), Shape(v.shape), v.mesh if v.mesh >= 0 else None,
                                    tuple(v.size), tuple(v.rgba), v.body, v.group))
        meshes = []
        for k in range(nm.value):
            nvx, ntr = C.c_int64(), C.c_int64()
            self._check(self._L.pg_scene_mesh(self._h, k, None, 0, None, 0, C.byref(nvx), C.byref(ntr)))
            verts = np.zeros((nvx.value, 3), np.float32)
            tris = np.zeros((ntr.value, 3), np.uint32)
            self._check(self._L.pg_scene_mesh(self._h, k, verts.ctypes.data_as(C.POINTER(C.c_float)), verts.size,
                                              tris.ctypes.data_as(C.POINTER(C.c_uint32)), tris.size, None, None))
            meshes.append(Mesh(self._name(3, k), verts, tris))
        cams = []
        for c in range(nc.value):
            f = C.c_float()
            self._check(self._L.pg_camera_fovy(self._h, c, C.byref(f)))
            cams.append(CameraDesc(self._name(2, c), f.value))
        return Scene([self._name(0, b) for b in range(nb.value)], geoms, meshes, cams)

    def _name(self, table: int, i: int) -> str:
        buf = C.create_string_buffer(256)
        self._check(self._L.pg_name_of(self._h, table, i, buf, 256))
        return buf.value.decode()

    def step(self, envs: EnvRange, nstep: int = 1):
        s, e = _span(envs)
        self._check(self._L.pg_step(self._h, s, e, int(nstep)))

    def step_device(self, envs: EnvRange, nstep: int, ctrl_dev_ptr: int):
        """Set controls from device memory ((envs, nu) FP64 at ctrl_dev_ptr on
        this handle's GPU) and step, in stream order."""
        s, e = _span(envs)
        self._check(self._L.pg_step_device(self._h, s, e, int(nstep), C.c_void_p(ctrl_dev_ptr)))

    def set_warm_mlp(self, weights):
        """Load a learned warm-start network (36662 floats, pippin_b200.warm)."""
        w = np.ascontiguousarray(weights, dtype=np.float32)
        self._check(self._L.pg_set_warm_mlp(self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size))

    def warm_samples(self, envs: EnvRange):
        """One substep of `envs`; returns the touching contacts' features
        (n, 24) and converged frame forces (n, 3) (f_n, f_t1, f_t2) as float32."""
        s, e = _span(envs)
        cap = int(self._L.pg_warm_capacity(self._h))
        X = np.empty((cap, 24), np.float32)
        R = np.empty((cap, 4), np.float32)
        n = C.c_int64()
        self._check(self._L.pg_warm_samples(self._h, s, e, X.ctypes.data_as(C.POINTER(C.c_float)), X.size,
                                            R.ctypes.data_as(C.POINTER(C.c_float)), R.size, C.byref(n)))
        X, R = X[:n.value], R[:n.value]
        mu = X[:, 1]
        F = np.stack([R.sum(axis=1), mu * (R[:, 0] - R[:, 1]), mu * (R[:, 2] - R[:, 3])], axis=1)
        return X, F.astype(np.float32)

    def time_phases(self, envs: EnvRange, nstep: int, ctrl_dev_ptr: int = 0) -> dict:
        """Step like step_device, timing each phase kernel with CUDA events;
        returns the summed device milliseconds per phase."""
        s, e = _span(envs)
        ms = (C.c_float * 4)()
        self._check(self._L.pg_time_phases(self._h, s, e, int(nstep), C.c_void_p(ctrl_dev_ptr or None), ms))
        out = {"smooth": ms[0], "collide": ms[1], "newton": ms[2]}
        if ms[3] > 0.0:
            out["inference"] = ms[3]
        return out

    def reset(self, envs: Sequence[int]):
        ids = np.ascontiguousarray(np.asarray(list(envs), dtype=np.int64))
        self._check(self._L.pg_reset(self._h, ids.ctypes.data_as(C.POINTER(C.c_int64)), len(ids)))

    def get(self, f: Field, envs: EnvRange, out: Optional[np.ndarray] = None) -> np.ndarray:
        s, e = _span(envs)
        w = self._dims.width(f)
        if out is None:
            out = np.empty((e - s, w), np.float64)
        if out.dtype != np.float64 or not out.flags.c_contiguous:
            raise PhysicsError("get: out must be a C-contiguous float64 array")
        self._check(self._L.pg_get(self._h, int(f), s, e, _pd(out), out.size))
        return out

    def set(self, f: Field, envs: EnvRange, src):
        s, e = _span(envs)
        a = np.ascontiguousarray(src, dtype=np.float64)
        self._check(self._L.pg_set(self._h, int(f), s, e, _pd(a), a.size))

    def poses(self, envs: EnvRange, geoms: Optional[np.ndarray] = None, cams: Optional[np.ndarray] = None):
        s, e = _span(envs)
        n = e - s
        d = self._dims
        if geoms is None:
            geoms = np.empty((n, d.ngeom, 12), np.float32)
        if cams is None:
            cams = np.empty((n, d.ncam, 12), np.float32)
        pf = C.POINTER(C.c_float)
        self._check(self._L.pg_poses(self._h, s, e, geoms.ctypes.data_as(pf), geoms.size // 12,
                                     cams.ctypes.data_as(pf), cams.size // 12))
        return geoms, cams

    def poses_device(self, envs: EnvRange, geoms_ptr: int, cams_ptr: int = 0):
        """Poses of `envs` written into device memory on this handle's GPU:
        geoms_ptr holds (envs, ngeom, 12) float32, cams_ptr (envs, ncam, 12)
        (0 when the model has no cameras). Enqueued on stream(); no wait."""
        s, e = _span(envs)
        self._check(self._L.pg_poses_device(self._h, s, e, C.c_void_p(geoms_ptr or None),
                                            C.c_void_p(cams_ptr or None)))

    def param_width(self, p: Param) -> int:
        return self._L.pg_param_width(self._h, int(p))

    def set_param(self, p: Param, elem: int, envs: EnvRange, values):
        s, e = _span(envs)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        self._check(self._L.pg_set_param(self._h, int(p), int(elem), s, e, _pd(v), v.size))

    def get_param(self, p: Param, elem: int, envs: EnvRange) -> np.ndarray:
        s, e = _span(envs)
        out = np.empty((e - s, self.param_width(p)), np.float64)
        self._check(self._L.pg_get_param(self._h, int(p), int(elem), s, e, _pd(out), out.size))
        return out

    def appearance(self, envs: EnvRange) -> np.ndarray:
        """(envs, ngeom, 8) float32: rgba[4], scale[3], pad."""
        s, e = _span(envs)
        out = np.empty((e - s, self._dims.ngeom, 8), np.float32)
        self._check(self._L.pg_appearance(self._h, s, e, out.ctypes.data_as(C.POINTER(C.c_float)),
                                          (e - s) * self._dims.ngeom))
        return out

    # ---- beyond the trait
    def rollout(self, ctrl: np.ndarray, envs: Optional[EnvRange] = None, record: bool = True):
        """Batch::rollout (crates/pippin/src/batch.rs:46-59): ctrl (envs, T, nu)."""
        s, e = _span(envs) if envs is not None else (0, self._n)
        c = np.ascontiguousarray(ctrl, dtype=np.float64)
        if c.ndim != 3 or c.shape[0] != e - s or c.shape[2] != self._dims.nu:
            raise PhysicsError(f"expected ctrl shape ({e - s}, T, {self._dims.nu}), got {c.shape}")
        out = np.empty((e - s, c.shape[1], self._dims.nq), np.float64) if record else None
        self._check(self._L.pg_rollout(self._h, s, e, c.shape[1], _pd(c), _pd(out) if record else None))
        return out

    def set_solver(self, kind: int = -1, iterations: int = -1, tolerance: float = -1.0, warm: int = -1):
        self._check(self._L.pg_set_solver(self._h, int(kind), int(iterations), float(tolerance), int(warm)))

    def stats(self, envs: Optional[EnvRange] = None) -> dict:
        s, e = _span(envs) if envs is not None else (0, self._n)
        arrs = [np.zeros(e - s, np.int32) for _ in range(4)]
        p32 = C.POINTER(C.c_int32)
        self._check(self._L.pg_stats(self._h, s, e, *(a.ctypes.data_as(p32) for a in arrs)))
        return dict(zip(["iters", "ncon", "nrows", "status"], arrs))

    def debug_forward(self, env: int, maxcon: int = 256) -> dict:
        nv = self._dims.nv
        qm = np.zeros((nv, nv))
        bias = np.zeros(nv)
        con = np.zeros((maxcon, 13))
        n = C.c_int64()
        self._check(self._L.pg_debug_forward(self._h, env, _pd(qm), _pd(bias), _pd(con), maxcon, C.byref(n)))
        return {"qm": qm, "qfrc_bias": bias, "contacts": con[:min(n.value, maxcon)], "ncon": n.value}

    def invweight(self, env: int):
        b = np.zeros((self.nbody, 2))
        d = np.zeros(self._dims.nv)
        self._check(self._L.pg_invweight(self._h, env, _pd(b), _pd(d)))
        return b, d

    def set_launch(self, lanes_per_env: int = 0, envs_per_block: int = 0):
        self._check(self._L.pg_set_launch(self._h, lanes_per_env, envs_per_block))

    def launch(self) -> Tuple[int, int, int]:
        g, t, b = C.c_int(), C.c_int(), C.c_int()
        self._check(self._L.pg_get_launch(self._h, C.byref(g), C.byref(t), C.byref(b)))
        return g.value, t.value, b.value

    def phase_launch(self) -> dict:
        """Launch shape (lanes per env, envs per block, blocks) of each phase kernel."""
        out = {}
        for k, name in enumerate(("smooth", "collide", "newton")):
            g, t, b = C.c_int32(), C.c_int32(), C.c_int32()
            self._check(self._L.pg_phase_launch(self._h, k, C.byref(g), C.byref(t), C.byref(b)))
            out[name] = (g.value, t.value, b.value)
        return out

    def autotune(self, nstep: int = 1):
        self._check(self._L.pg_autotune(self._h, int(nstep)))
        return self.launch()

    def synchronize(self):
        self._check(self._L.pg_synchronize(self._h))

    def device_ptr(self, f: Field) -> int:
        p = C.POINTER(C.c_double)()
        self._check(self._L.pg_field_device_ptr(self._h, int(f), C.byref(p)))
        return C.cast(p, C.c_void_p).value

    def device_view(self, f: Field):
        """A zero-copy torch tensor (num_envs, width) float64 over this
        handle's device state for field f: the observation and action buffers
        an on-GPU policy works on, in place of the host copies of
        crates/pippin-env/src/pipeline.rs:65-72. The memory stays the handle's:
        the view keeps this object alive, but close() frees it all the same.
        The physics writes it on stream(): wait for that stream (or call
        synchronize()) before reading, and finish writes before the next step.
        A write through the view is a plain store: set(QPOS) also refreshes the
        kinematics that poses() reports, a write to the QPOS view does not
        until the next step. CTRL and QFRC_APPLIED are plain inputs."""
        import torch

        shape = (self._n, self._dims.width(f))
        return torch.as_tensor(_DeviceArray(self.device_ptr(f), shape, self),
                               device=torch.device("cuda", self._device))

    def stream(self) -> int:
        return self._L.pg_stream(self._h) or 0
