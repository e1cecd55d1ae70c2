"""pg_step_static (stepping without allocating) against pg_step.

pg_step_static is for callers that cannot let a call allocate device memory:
another component owns the GPU's memory, a latency-critical loop must stay out
of the allocator, or memory is already exhausted. It takes its scratch from a
fixed array in the library instead of the handle's buffer. Two handles start
from the same state; one steps with pg_step, the other with pg_step_static
through the C-ABI, twice in a row (the second call finds the array holding the
first call's contents), and the states must agree within the parity
tolerance of the other GPU tests. The batch is larger than the number of envs
the static scratch steps at once, so the work loop runs several rounds.
"""
import ctypes as C

import numpy as np
import pytest

from pippin_b200 import CudaPhysics, Field, Param, _native, mjcf, scenes

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1.0))


def test_static_scratch_step_matches_pg_step():
    L = _native.load()
    n = 1024
    m = mjcf.load_string(scenes.ant_xml(tolerance=1e-10))
    blob = mjcf.to_blob(m)
    ref, stat = CudaPhysics(blob, n), CudaPhysics(blob, n)
    rng = np.random.default_rng(11)
    q = np.tile(np.array(m.qpos0), (n, 1)) + rng.uniform(-0.1, 0.1, (n, m.nq))
    v = rng.normal(0, 0.1, (n, m.nv))
    for p in (ref, stat):
        p.set(Field.QPOS, range(n), q)
        p.set(Field.QVEL, range(n), v)
    for call in range(2):
        ctrl = rng.uniform(-1, 1, (n, m.nu))
        ref.set(Field.CTRL, range(n), ctrl)
        stat.set(Field.CTRL, range(n), ctrl)
        ref.step(range(n), 40)
        rc = L.pg_step_static(stat._h, 0, n, 40)
        assert rc == 0, _native.last_error()
        stat.synchronize()
        for f in (Field.QPOS, Field.QVEL, Field.QACC):
            a, b = stat.get(f, range(n)), ref.get(f, range(n))
            assert np.isfinite(a).all()
            assert rel(a, b) < TOL, (call, f, rel(a, b))
    assert stat.stats()["ncon"].sum() > 0  # the Ant reached the ground: contacts were exercised


def test_static_scratch_rejects_bad_ranges():
    L = _native.load()
    p = CudaPhysics(scenes.ant_xml(), 4)
    assert L.pg_step_static(p._h, 2, 9, 1) != 0
    assert "out of bounds" in _native.last_error()
    assert L.pg_step_static(p._h, 1, 1, 3) == 0  # empty range: nothing to do


def test_static_scratch_island_path_matches_pg_step():
    """The tabletop (36 dofs in six free bodies) takes the tile Newton with
    islands, whose per-tile scratch is far larger than Ant's: fewer tiles fit
    the static array, so 512 envs step in many rounds. Objects fall onto the
    table and each other during the two calls."""
    L = _native.load()
    n = 512
    plan = scenes.tabletop(n, seed=3)
    blob = mjcf.to_blob(mjcf.load_string(plan.xml))
    ref, stat = CudaPhysics(blob, n), CudaPhysics(blob, n)
    for p in (ref, stat):
        p.set_solver(tolerance=TOL, iterations=30)
        plan.apply(lambda pid, elem, vals, p=p: p.set_param(Param(pid), elem, range(n), vals),
                   lambda p=p: p.reset(range(n)))
    for call in range(2):
        ref.step(range(n), 60)
        rc = L.pg_step_static(stat._h, 0, n, 60)
        assert rc == 0, _native.last_error()
        stat.synchronize()
        for f in (Field.QPOS, Field.QVEL, Field.QACC):
            a, b = stat.get(f, range(n)), ref.get(f, range(n))
            assert np.isfinite(a).all()
            assert rel(a, b) < TOL, (call, f, rel(a, b))
    st = stat.stats()
    assert st["nrows"].sum() > 0 and (st["status"] == 0).all()
