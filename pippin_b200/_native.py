"""ctypes bindings of the C-ABI in include/pippin_b200.h.

Loads lib/libpippin_b200.so from this package (built by pippin_b200.build).
There is no CPU fallback: a missing library or a missing CUDA device is an
error.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libpippin_b200.so")

PG_OK, PG_ERR_INVALID, PG_ERR_LENGTH, PG_ERR_CUDA, PG_ERR_UNSUPPORTED, PG_ERR_NOMEM = range(6)


class PgModelDims(C.Structure):
    _fields_ = [("nq", C.c_int64), ("nv", C.c_int64), ("nu", C.c_int64), ("ngeom", C.c_int64), ("ncam", C.c_int64),
                ("nbody", C.c_int64), ("njnt", C.c_int64)]


class PgGeomVisual(C.Structure):
    _fields_ = [("shape", C.c_int32), ("mesh", C.c_int32), ("size", C.c_float * 3), ("rgba", C.c_float * 4),
                ("body", C.c_int32), ("group", C.c_int32)]


# (symbol, restype, argtypes) for every function the header declares
_vp, _i64, _i32, _dbl, _sz = C.c_void_p, C.c_int64, C.c_int, C.c_double, C.c_size_t
_pd, _pf, _pi64, _pi32 = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int64), C.POINTER(C.c_int32)
SIGNATURES = [
    ("pg_create", _i32, [C.c_char_p, _sz, _i64, _i32, C.POINTER(_vp)]),
    ("pg_destroy", _i32, [_vp]),
    ("pg_name", C.c_char_p, [_vp]),
    ("pg_num_envs", _i64, [_vp]),
    ("pg_dims", _i32, [_vp, C.POINTER(PgModelDims)]),
    ("pg_step", _i32, [_vp, _i64, _i64, _i64]),
    ("pg_step_device", _i32, [_vp, _i64, _i64, _i64, _vp]),
    ("pg_step_static", _i32, [_vp, _i64, _i64, _i64]),
    ("pg_rollout", _i32, [_vp, _i64, _i64, _i64, _pd, _pd]),
    ("pg_reset", _i32, [_vp, _pi64, _i64]),
    ("pg_get", _i32, [_vp, _i32, _i64, _i64, _pd, _sz]),
    ("pg_set", _i32, [_vp, _i32, _i64, _i64, _pd, _sz]),
    ("pg_poses", _i32, [_vp, _i64, _i64, _pf, _sz, _pf, _sz]),
    ("pg_poses_device", _i32, [_vp, _i64, _i64, _vp, _vp]),
    ("pg_param_width", _i32, [_vp, _i32]),
    ("pg_set_param", _i32, [_vp, _i32, _i64, _i64, _i64, _pd, _sz]),
    ("pg_get_param", _i32, [_vp, _i32, _i64, _i64, _i64, _pd, _sz]),
    ("pg_appearance", _i32, [_vp, _i64, _i64, _pf, _sz]),
    ("pg_scene_counts", _i32, [_vp, _pi64, _pi64, _pi64, _pi64]),
    ("pg_scene_geoms", _i32, [_vp, C.POINTER(PgGeomVisual), _sz]),
    ("pg_scene_mesh", _i32, [_vp, _i64, _pf, _sz, C.POINTER(C.c_uint32), _sz, _pi64, _pi64]),
    ("pg_camera_fovy", _i32, [_vp, _i64, _pf]),
    ("pg_name_of", _i32, [_vp, _i32, _i64, C.c_char_p, _sz]),
    ("pg_set_solver", _i32, [_vp, _i32, _i32, _dbl, _i32]),
    ("pg_stats", _i32, [_vp, _i64, _i64, _pi32, _pi32, _pi32, _pi32]),
    ("pg_debug_forward", _i32, [_vp, _i64, _pd, _pd, _pd, _i64, _pi64]),
    ("pg_invweight", _i32, [_vp, _i64, _pd, _pd]),
    ("pg_set_launch", _i32, [_vp, _i32, _i32]),
    ("pg_get_launch", _i32, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("pg_autotune", _i32, [_vp, _i64]),
    ("pg_synchronize", _i32, [_vp]),
    ("pg_field_device_ptr", _i32, [_vp, _i32, C.POINTER(_pd)]),
    ("pg_stream", _vp, [_vp]),
    ("pg_last_error", C.c_char_p, []),
    ("pg_fp64_peak", _i32, [_i32, _i32, _pd, _pd]),
    ("pg_time_phases", _i32, [_vp, _i64, _i64, _i64, _vp, _pf]),
    ("pg_phase_launch", _i32, [_vp, _i32, _pi32, _pi32, _pi32]),
    ("pg_static_tiles", _i32, [_sz, _i32, _pi64]),
    ("pg_hull_support", _i32, [_vp, _i32, _pd, _i64, _pi32]),
    ("pg_set_warm_mlp", _i32, [_vp, _pf, _sz]),
    ("pg_warm_samples", _i32, [_vp, _i64, _i64, _pf, _sz, _pf, _sz, _pi64]),
    ("pg_warm_capacity", _i64, [_vp]),
    ("pg_mlp_forward", _i32, [_pf, _sz, _pf, _i64, _pf]),
    ("pg_mlp_loss_grad", _i32, [_pf, _sz, _pf, _pf, _i64, _pf, _sz, _pd]),
    ("pg_mlp_train", _i32, [_pf, _pf, _i64, _i32, _i32, C.c_float, C.c_uint64, _pf, _sz, _pd]),
    ("pg_render_create", _i32, [_pf, _i64, C.POINTER(C.c_uint32), _i64, _i64, _i64, _pf, _i64, _pf, _i64, _i64, _pf,
                                _i32, C.POINTER(_vp)]),
    ("pg_render_destroy", _i32, [_vp]),
    ("pg_render_frames", _i32, [_vp, _i64, _pf, _sz, _pf, _sz, _pf, _sz, C.POINTER(C.c_uint8), _pf, _pi32]),
    ("pg_render_frames_device", _i32, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("pg_render_stream", _vp, [_vp]),
    ("pg_render_synchronize", _i32, [_vp]),
]

_lib = None


class NativeLibraryError(RuntimeError):
    """The CUDA backend library is missing or cannot be loaded."""


def load(path: str = LIB_PATH):
    """Load (once) and return the library with typed signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise NativeLibraryError(
            f"{path} not found: build it with `python -m pippin_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return (load().pg_last_error() or b"").decode()
