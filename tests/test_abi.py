"""The C-ABI library loads and exports every function include/pippin_b200.h
declares; the Python bindings cover the same set. No GPU needed (nothing
here calls into CUDA)."""
import ctypes
import os
import re

import pytest

from pippin_b200 import _native

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_functions():
    names = set()
    for h in sorted(os.listdir(INCLUDE)):
        if h.endswith(".h"):
            text = re.sub(r"/\*.*?\*/", "", open(os.path.join(INCLUDE, h)).read(), flags=re.S)
            names |= set(re.findall(r"^[a-z_][\w\s\*]*?\b(pg_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_header_declares_the_api():
    names = declared_functions()
    for must in ["pg_create", "pg_destroy", "pg_step", "pg_reset", "pg_get", "pg_set", "pg_poses", "pg_set_param",
                 "pg_get_param", "pg_appearance", "pg_scene_geoms", "pg_last_error", "pg_stats"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from pippin_b200 import build
    build.build()
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_match_header():
    bound = {name for name, _, _ in _native.SIGNATURES}
    assert bound == set(declared_functions())


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(_native.NativeLibraryError):
        _native._lib = None
        try:
            _native.load(str(tmp_path / "nope.so"))
        finally:
            _native._lib = None


def test_static_scratch_capacity_and_rejection():
    """pg_step_static's capacity check is pure arithmetic (no GPU): whole
    blocks of tiles out of the fixed array, and a clear rejection when one
    block does not fit."""
    from pippin_b200 import build
    build.build()
    L = _native.load()
    tiles = ctypes.c_int64(-1)
    usable = (16 << 20) - 256 - 64
    assert L.pg_static_tiles(1 << 17, 16, ctypes.byref(tiles)) == _native.PG_OK
    assert tiles.value == usable // (1 << 17) // 16 * 16
    # an exact fit leaves the 64-byte tail free
    assert L.pg_static_tiles(usable // 8, 8, ctypes.byref(tiles)) == _native.PG_OK and tiles.value == 8
    assert L.pg_static_tiles(usable // 8 + 1, 8, ctypes.byref(tiles)) == _native.PG_ERR_UNSUPPORTED
    assert tiles.value == 0
    msg = _native.last_error()
    assert "bytes of scratch per block" in msg and "use pg_step" in msg
    assert L.pg_static_tiles(0, 8, ctypes.byref(tiles)) == _native.PG_ERR_INVALID


def test_device_view_describes_the_state_buffer():
    """The array interface behind CudaPhysics.device_view: the field's device
    address, (num_envs, width) float64, row-major, and a reference to the
    owner that keeps the handle alive while a view exists."""
    from pippin_b200.physics import _DeviceArray
    owner = object()
    a = _DeviceArray(0x7F0000001000, (16384, 15), owner)
    cai = a.__cuda_array_interface__
    assert cai["shape"] == (16384, 15) and cai["typestr"] == "<f8" and cai["strides"] is None
    assert cai["data"] == (0x7F0000001000, False) and cai["version"] == 2
    assert a.owner is owner
