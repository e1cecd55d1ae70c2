"""Oracle (test infrastructure only): ctypes wrapper over the C++ restatement
of the reference CPU engine (liboracle.so, built by oracle/Makefile).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, always as the checker or the timed CPU baseline; the product
package never imports it. The class mirrors the reference's CPU backend
behind the Physics trait (crates/pippin-env/src/pippin_cpu.rs:14-206).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

QPOS, QVEL, CTRL, QACC, QFRC_APPLIED = 0, 1, 2, 3, 4
STAGES = ["kinematics", "crba", "vel_rne", "passive_act", "collide", "factor_solve", "rows", "newton", "pgs",
          "integrate"]


def build(force: bool = False) -> None:
    """Compile liboracle.so / liboracle_fast.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []), check=True)


def _lib(fast: bool = False):
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
    pd, pf, pi64, pi32 = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int64), C.POINTER(C.c_int32)
    L.om_create.restype = vp
    L.om_create.argtypes = [C.c_char_p, C.c_size_t, i32, i32, C.c_char_p, C.c_size_t]
    L.om_destroy.argtypes = [vp]
    L.om_num_threads.argtypes = [vp]
    L.om_dims.argtypes = [vp, pi64]
    L.om_set_solver.argtypes = [vp, i32, i32, dbl]
    L.om_step.argtypes = [vp, i64, i64, i32]
    L.om_rollout.argtypes = [vp, i64, i64, i32, pd, pd]
    L.om_forward.argtypes = [vp, i64, i64]
    L.om_kinematics.argtypes = [vp, i64, i64]
    L.om_reset.argtypes = [vp, pi64, i64]
    L.om_get.argtypes = [vp, i32, i64, i64, pd]
    L.om_set.argtypes = [vp, i32, i64, i64, pd]
    L.om_set_param.argtypes = [vp, i32, i32, i64, i64, pd, C.c_char_p, C.c_size_t]
    L.om_get_param.argtypes = [vp, i32, i32, i64, i64, pd, C.c_char_p, C.c_size_t]
    L.om_param_width.argtypes = [vp, i32]
    L.om_poses.argtypes = [vp, i64, i64, pf, pf]
    L.om_appearance.argtypes = [vp, i64, i64, pf]
    L.om_stats.argtypes = [vp, i64, i64, pi32, pi32, pi32, pi32]
    L.om_debug.argtypes = [vp, i64, pd, pd, pd, pd, i32]
    L.om_body_poses.argtypes = [vp, i64, pd]
    L.om_invweight.argtypes = [vp, i64, pd, pd]
    L.om_flops.argtypes = [vp, pd, i32]
    L.om_impedance.restype = dbl
    L.om_impedance.argtypes = [pd, dbl]
    L.om_vdot.restype = dbl
    L.om_vdot.argtypes = [pd, pd, i64]
    L.om_cholesky_block.argtypes = [pd, i64, i64, i64]
    L.om_cholesky_solve_block.argtypes = [pd, i64, i64, i64, pd]
    L.om_quat_from_axis_angle.argtypes = [pd, dbl, pd]
    L.om_quat_to_mat.argtypes = [pd, pd]
    L.om_hull_support.argtypes = [pd, i64, pi32, i64, pd, i64, pi32]
    _LIBS[name] = L
    return L


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def lib():
    return _lib(False)


class OracleError(RuntimeError):
    pass


class Oracle:
    """Batch of environments on the CPU restatement (one Model copy per env,
    copy on write, as pippin_cpu.rs:14-31)."""

    def __init__(self, blob: bytes, n_envs: int, threads: int = 0, fast: bool = False):
        self.L = _lib(fast)
        err = C.create_string_buffer(512)
        self._blob = blob
        self.h = self.L.om_create(blob, len(blob), n_envs, threads, err, 512)
        if not self.h:
            raise OracleError(err.value.decode())
        d = np.zeros(8, np.int64)
        self.L.om_dims(self.h, _p(d, C.c_int64))
        self.nq, self.nv, self.nu, self.nbody, self.njnt, self.ngeom, self.ncam, self.nmesh = (int(x) for x in d)
        self.n = n_envs
        self.threads = self.L.om_num_threads(self.h)

    def close(self):
        if self.h:
            self.L.om_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def width(self, field):
        return {QPOS: self.nq, QVEL: self.nv, CTRL: self.nu, QACC: self.nv, QFRC_APPLIED: self.nv}[field]

    def set_solver(self, kind=-1, iterations=-1, tolerance=-1.0):
        self.L.om_set_solver(self.h, kind, iterations, tolerance)

    def step(self, start=0, end=None, nstep=1):
        end = self.n if end is None else end
        self.L.om_step(self.h, start, end, nstep)

    def rollout(self, ctrl, start=0, end=None, record=True):
        end = self.n if end is None else end
        ctrl = np.ascontiguousarray(ctrl, dtype=np.float64)
        nstep = ctrl.shape[1]
        out = np.zeros((end - start, nstep, self.nq)) if record else None
        self.L.om_rollout(self.h, start, end, nstep, _p(ctrl), _p(out) if record else None)
        return out

    def forward(self, start=0, end=None):
        self.L.om_forward(self.h, start, self.n if end is None else end)

    def reset(self, ids):
        ids = np.ascontiguousarray(ids, dtype=np.int64)
        self.L.om_reset(self.h, _p(ids, C.c_int64), len(ids))

    def get(self, field, start=0, end=None):
        end = self.n if end is None else end
        out = np.zeros((end - start, self.width(field)))
        self.L.om_get(self.h, field, start, end, _p(out))
        return out

    def set(self, field, values, start=0, end=None):
        end = self.n if end is None else end
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(end - start, self.width(field))
        self.L.om_set(self.h, field, start, end, _p(v))

    def set_param(self, p, elem, values, start=0, end=None):
        end = self.n if end is None else end
        w = self.L.om_param_width(self.h, p)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if v.size != (end - start) * w:
            raise OracleError(f"set_param: buffer has {v.size} elements, expected {end - start} x {w}")
        err = C.create_string_buffer(512)
        if self.L.om_set_param(self.h, p, elem, start, end, _p(v), err, 512):
            raise OracleError(err.value.decode())

    def get_param(self, p, elem, start=0, end=None):
        end = self.n if end is None else end
        w = self.L.om_param_width(self.h, p)
        out = np.zeros((end - start, w))
        err = C.create_string_buffer(512)
        if self.L.om_get_param(self.h, p, elem, start, end, _p(out), err, 512):
            raise OracleError(err.value.decode())
        return out

    def poses(self, start=0, end=None):
        end = self.n if end is None else end
        g = np.zeros((end - start, self.ngeom, 12), np.float32)
        c = np.zeros((end - start, max(self.ncam, 0), 12), np.float32)
        self.L.om_poses(self.h, start, end, _p(g, C.c_float), _p(c, C.c_float))
        return g, c

    def appearance(self, start=0, end=None):
        end = self.n if end is None else end
        a = np.zeros((end - start, self.ngeom, 8), np.float32)
        self.L.om_appearance(self.h, start, end, _p(a, C.c_float))
        return a

    def stats(self, start=0, end=None):
        end = self.n if end is None else end
        k = end - start
        it, nc, nr, st = (np.zeros(k, np.int32) for _ in range(4))
        self.L.om_stats(self.h, start, end, _p(it, C.c_int32), _p(nc, C.c_int32), _p(nr, C.c_int32),
                        _p(st, C.c_int32))
        return {"iters": it, "ncon": nc, "nrows": nr, "status": st}

    def debug(self, env, maxcon=256):
        nv = self.nv
        qm = np.zeros((nv, nv))
        bias = np.zeros(nv)
        qc = np.zeros(nv)
        con = np.zeros((maxcon, 13))
        n = self.L.om_debug(self.h, env, _p(qm), _p(bias), _p(qc), _p(con), maxcon)
        return {"qm": qm, "qfrc_bias": bias, "qfrc_constraint": qc, "contacts": con[:min(n, maxcon)], "ncon": n}

    def body_poses(self, env):
        out = np.zeros((self.nbody, 12))
        self.L.om_body_poses(self.h, env, _p(out))
        return out

    def invweight(self, env):
        b = np.zeros((self.nbody, 2))
        d = np.zeros(self.nv)
        self.L.om_invweight(self.h, env, _p(b), _p(d))
        return b, d

    def flops(self, reset=False):
        out = np.zeros(len(STAGES))
        self.L.om_flops(self.h, _p(out), 1 if reset else 0)
        return dict(zip(STAGES, out))


# ---- known-answer hooks (reference unit tests) ----
def impedance(solimp, pos):
    s = np.ascontiguousarray(solimp, dtype=np.float64)
    return lib().om_impedance(_p(s), float(pos))


def hull_support(verts, edges, dirs):
    """The reference's hull support walk (fasthull.rs:76-120): for each
    direction, the index of the vertex it ends at."""
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
    e = np.ascontiguousarray(edges, dtype=np.int32).reshape(-1, 2)
    d = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(len(d), dtype=np.int32)
    if lib().om_hull_support(_p(v), len(v), _p(e, C.c_int32), len(e), _p(d), len(d), _p(out, C.c_int32)) != 0:
        raise OracleError("hull_support: edge vertex out of range")
    return out


def vdot(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return lib().om_vdot(_p(a), _p(b), min(len(a), len(b)))


def cholesky_block(a, stride, s0, s1):
    return bool(lib().om_cholesky_block(_p(a), stride, s0, s1))


def cholesky_solve_block(l, stride, s0, s1, x):
    lib().om_cholesky_solve_block(_p(l), stride, s0, s1, _p(x))


def quat_from_axis_angle(axis, angle):
    ax = np.ascontiguousarray(axis, dtype=np.float64)
    q = np.zeros(4)
    lib().om_quat_from_axis_angle(_p(ax), float(angle), _p(q))
    return q


def quat_to_mat(q):
    q = np.ascontiguousarray(q, dtype=np.float64)
    m = np.zeros(9)
    lib().om_quat_to_mat(_p(q), _p(m))
    return m
