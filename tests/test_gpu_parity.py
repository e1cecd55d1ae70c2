"""CUDA backend vs the oracle (C++ restatement of the reference CPU engine).

Tolerances (relative to the quantity's scale, max(|ref|_inf, 1)):
  M(q), c(q, qdot)                 1e-12
  contact pos / normal / depth     1e-12 (same count, pairs and order)
  per-step qacc, qvel, qpos        1e-10 (identical input states each step)
  contact-free 1 s trajectories    1e-8
"""
import ctypes as C

import numpy as np
import pytest

from oracle.oracle import CTRL, QACC, QPOS, QVEL, Oracle
from pippin_b200 import CudaPhysics, Field, Param, PhysicsError, _native, mjcf, scenes
from tests import scenarios as S

pytestmark = pytest.mark.gpu

TOL_MC = 1e-12
TOL_STEP = 1e-10
TOL_TRAJ = 1e-8


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1.0))


def random_state(m, n, rng, qnoise=0.1, vscale=0.1):
    q = np.tile(np.array(m.qpos0), (n, 1)) + rng.uniform(-qnoise, qnoise, (n, m.nq))
    v = rng.normal(0, vscale, (n, m.nv))
    return q, v


def pair(xml, n, tolerance=None):
    m = mjcf.load_string(xml)
    blob = mjcf.to_blob(m)
    g = CudaPhysics(blob, n)
    o = Oracle(blob, n, threads=4)
    if tolerance is not None:
        g.set_solver(tolerance=tolerance)
        o.set_solver(tolerance=tolerance)
    return m, g, o


MODELS = {
    "ant": scenes.ant_xml,
    "cartpole": scenes.cartpole_xml,
    "arm3d": scenes.arm3d_xml,
    "arm3hinge": scenes.arm3hinge_xml,
    "box_drop": scenes.box_drop_xml,
    "shapes_on_box": lambda: S.ON_BOX,
    "box_stack": lambda: S.box_stack_xml(),
    "mesh_and_box": lambda: S.MESH_AND_BOX,
    "mesh_stack": lambda: S.mesh_stack_xml(),
    "cylinders": lambda: S.CYLINDERS,
    "hull_tumble": scenes.hull_tumble_xml,
    "big_hulls": lambda: S.big_hulls_xml(),
    # joint equality rows, fixed tendons, implicitfast actuators
    "equality_chain": lambda: S.EQUALITY_CHAIN,
    "equality_chain_solo": lambda: S.EQUALITY_CHAIN.replace(
        '<body name="ball" pos="0.3 0.02 0.2"><freejoint/><geom type="sphere" size="0.06"/></body>', ""),
    "tendon_arm": lambda: S.TENDON_ARM,
    "implicitfast_arm": lambda: S.IMPLICITFAST_ARM,
}


@pytest.mark.parametrize("name", list(MODELS))
def test_forward_parity(name):
    """M, bias forces and contact sets on random states (forward.rs:263-271)."""
    n = 32
    m, g, o = pair(MODELS[name](), n)
    rng = np.random.default_rng(1)
    q, v = random_state(m, n, rng, qnoise=0.3, vscale=1.0)
    for sim in (g, o):
        sim.set(QPOS if sim is o else Field.QPOS, q) if sim is o else sim.set(Field.QPOS, range(n), q)
    o.set(QVEL, v)
    g.set(Field.QVEL, range(n), v)
    o.forward()
    for e in range(n):
        dg = g.debug_forward(e)
        do = o.debug(e)
        assert rel(dg["qm"], do["qm"]) < TOL_MC, (e, rel(dg["qm"], do["qm"]))
        assert rel(dg["qfrc_bias"], do["qfrc_bias"]) < TOL_MC, e
        assert dg["ncon"] == do["ncon"], (e, dg["ncon"], do["ncon"])
        if do["ncon"]:
            cg, co = dg["contacts"], do["contacts"]
            np.testing.assert_array_equal(cg[:, 10:13], co[:, 10:13])
            assert rel(cg[:, :10], co[:, :10]) < TOL_MC, e


def _copy_state(src_g, dst_o, n):
    for fg, fo in ((Field.QPOS, QPOS), (Field.QVEL, QVEL), (Field.QACC, QACC), (Field.CTRL, CTRL)):
        dst_o.set(fo, src_g.get(fg, range(n)))


def test_ant_step_parity_on_identical_states():
    """Per-step Newton output on identical input states (config 1 setup,
    tolerance 1e-10), through falls, ground contact and joint limits."""
    n, T = 64, 120
    m, g, o = pair(scenes.ant_xml(), n, tolerance=1e-10)
    rng = np.random.default_rng(0)
    q, v = random_state(m, n, rng)
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    worst = {"qacc": 0.0, "qvel": 0.0, "qpos": 0.0}
    contacts_seen = 0
    for t in range(T):
        g.set(Field.CTRL, range(n), rng.uniform(-1, 1, (n, m.nu)))
        _copy_state(g, o, n)
        g.step(range(n), 1)
        o.step(0, n, 1)
        sg, so = g.stats(), o.stats()
        np.testing.assert_array_equal(sg["ncon"], so["ncon"])
        np.testing.assert_array_equal(sg["nrows"], so["nrows"])
        assert not sg["status"].any()
        contacts_seen += int(so["ncon"].sum())
        for fg, fo, key in ((Field.QACC, QACC, "qacc"), (Field.QVEL, QVEL, "qvel"), (Field.QPOS, QPOS, "qpos")):
            a, b = g.get(fg, range(n)), o.get(fo)
            for e in range(n):
                worst[key] = max(worst[key], rel(a[e], b[e]))
    assert contacts_seen > 0
    assert worst["qacc"] < TOL_STEP, worst
    assert worst["qvel"] < TOL_STEP, worst
    assert worst["qpos"] < TOL_STEP, worst


@pytest.mark.parametrize("name", ["cartpole", "arm3d", "arm3hinge"])
def test_contact_free_trajectories(name):
    """Config 2: random states, per-env masses x U[0.5, 2], 1 s of motion."""
    n = 64
    m, g, o = pair(MODELS[name](), n)
    rng = np.random.default_rng(2)
    q = np.tile(np.array(m.qpos0), (n, 1))
    for j in range(m.njnt):
        qa = m.jnt_qposadr[j]
        if m.jnt_type[j] == mjcf.JNT_HINGE:
            q[:, qa] = rng.uniform(-np.pi, np.pi, n)
        elif m.jnt_type[j] == mjcf.JNT_SLIDE:
            q[:, qa] = rng.uniform(-0.5, 0.5, n)
        elif m.jnt_type[j] == mjcf.JNT_BALL:
            w = rng.normal(size=(n, 4))
            q[:, qa:qa + 4] = w / np.linalg.norm(w, axis=1, keepdims=True)
    v = rng.normal(0, 1, (n, m.nv))
    for b in range(1, m.nbody):
        scale = rng.uniform(0.5, 2.0, n)
        vals = (np.array(m.body_mass[b]) * scale).reshape(n, 1)
        g.set_param(Param.BODY_MASS, b, range(n), vals)
        o.set_param(5, b, vals)
    for e in range(0, n, 7):
        bg, dg = g.invweight(e)
        bo, do = o.invweight(e)
        assert rel(bg, bo) < TOL_MC and rel(dg, do) < TOL_MC
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    o.set(QPOS, q)
    o.set(QVEL, v)
    steps = int(round(1.0 / m.timestep))
    ctrl = rng.uniform(-1, 1, (n, steps, max(m.nu, 0)))
    og = g.rollout(ctrl)
    oo = o.rollout(ctrl)
    assert rel(og[:, -1], oo[:, -1]) < TOL_TRAJ, rel(og[:, -1], oo[:, -1])


def test_set_const_matches_oracle():
    n = 8
    m, g, o = pair(scenes.ant_xml(), n)
    for e in range(n):
        bg, dg = g.invweight(e)
        bo, do = o.invweight(e)
        assert rel(bg, bo) < TOL_MC and rel(dg, do) < TOL_MC
    g.set_param(Param.BODY_IPOS, 2, range(2, 5), np.full((3, 3), 0.01))
    o.set_param(10, 2, np.full((3, 3), 0.01), 2, 5)
    g.set_param(Param.BODY_INERTIA, 3, range(1, 3), [[0.1, 0.2, 0.3], [0.2, 0.2, 0.2]])
    o.set_param(9, 3, [[0.1, 0.2, 0.3], [0.2, 0.2, 0.2]], 1, 3)
    for e in range(n):
        bg, dg = g.invweight(e)
        bo, do = o.invweight(e)
        assert rel(bg, bo) < TOL_MC and rel(dg, do) < TOL_MC, e


@pytest.mark.parametrize("check", S.CONTACT_CHECKS, ids=lambda f: f.__name__)
def test_contact_behaviour_newton(check):
    check(S.CudaSim, S.NEWTON)


@pytest.mark.parametrize("check", S.CONTACT_CHECKS, ids=lambda f: f.__name__)
def test_contact_behaviour_pgs(check):
    check(S.CudaSim, S.PGS)


@pytest.mark.parametrize("solver", [S.NEWTON, S.PGS], ids=["newton", "pgs"])
@pytest.mark.parametrize("check", S.GENERAL_CHECKS, ids=lambda f: f.__name__)
def test_general_convex_behaviour(check, solver):
    """The reference's mesh.rs scenes through the general convex path."""
    check(S.CudaSim, solver)


@pytest.mark.parametrize("name", ["hull_tumble", "cylinders", "mesh_stack", "big_hulls"])
def test_general_convex_step_parity(name):
    """Per-step Newton output on identical input states while hulls and
    cylinders fall, collide and settle (tolerance 1e-10). The oracle scans
    every vertex and tests every edge pair; the device walks large hulls'
    vertex graphs and prunes edges (big_hulls: hulls of 276 and 96 vertices,
    48-gon faces clipped in shared memory)."""
    n = 16
    m, g, o = pair(MODELS[name](), n, tolerance=1e-10)
    T = int(round(0.6 / m.timestep))
    rng = np.random.default_rng(4)
    q, v = random_state(m, n, rng, qnoise=0.02, vscale=0.5)
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    contacts_seen = 0
    for t in range(T):
        _copy_state(g, o, n)
        g.step(range(n), 1)
        o.step(0, n, 1)
        sg, so = g.stats(), o.stats()
        assert not sg["status"].any(), (t, sg["status"])
        np.testing.assert_array_equal(sg["ncon"], so["ncon"])
        contacts_seen += int(so["ncon"].sum())
        for fg, fo in ((Field.QACC, QACC), (Field.QVEL, QVEL), (Field.QPOS, QPOS)):
            a, b = g.get(fg, range(n)), o.get(fo)
            for e in range(n):
                assert rel(a[e], b[e]) < TOL_STEP, (t, e, fg, rel(a[e], b[e]))
    assert contacts_seen > 0


def test_hull_support_walk_on_device_matches_brute_force():
    """fasthull.rs:217-240 on the device: the collision kernel's support walk
    over the hull of the 600-point lumpy sphere (276 vertices) projects as far
    as a scan of every hull vertex along each of 2000 directions (1e-12)."""
    L = _native.load()
    m = mjcf.load_string(S.big_hulls_xml())
    g = CudaPhysics(mjcf.to_blob(m), 1)
    v = np.asarray(m.hull_vert[0], dtype=np.float64)
    assert len(v) >= 64
    d = np.ascontiguousarray(S.support_directions())
    out = np.zeros(len(d), dtype=np.int32)
    rc = L.pg_hull_support(g._h, 0, d.ctypes.data_as(C.POINTER(C.c_double)), len(d),
                           out.ctypes.data_as(C.POINTER(C.c_int32)))
    assert rc == 0, _native.last_error()
    assert ((out >= 0) & (out < len(v))).all()
    exact = (v @ d.T).max(axis=0)
    got = np.einsum("ij,ij->i", v[out], d)
    assert np.abs(exact - got).max() < 1e-12
    assert L.pg_hull_support(g._h, 2, d.ctypes.data_as(C.POINTER(C.c_double)), 1,
                             out.ctypes.data_as(C.POINTER(C.c_int32))) != 0  # no mesh 2


@pytest.mark.parametrize("solver", ["newton", "pgs"])
@pytest.mark.parametrize("name", ["equality_chain", "equality_chain_solo", "tendon_arm", "implicitfast_arm"])
def test_branch_step_parity(name, solver):
    """Per-step output on identical input states for the branches the
    workload models do not reach: joint equality rows with a polynomial
    coupling, a fixed joint and a per-equality solref (newton.rs:171-195;
    the solo chain takes the register Newton, the chain with a free ball the
    island path), fixed-tendon actuators (mjcf.rs:852-947) and implicitfast
    position/velocity actuators with joint damping (forward.rs:407-431),
    each with floor contacts and joint limits. PGS runs with its warm start
    cleared each step, as in test_pgs_step_parity. PGS stops sweeping once a
    sweep changes no velocity by more than 1e-5 (solver.rs:36): where a
    rounding difference moves that decision by one sweep (the sweep counts
    differ, in at most 1% of the env-steps) the two runs agree to that
    stopping tolerance (1e-4 on qvel) rather than to 1e-10."""
    n = 32
    m, g, o = pair(MODELS[name](), n, tolerance=1e-10)
    if solver == "pgs":
        g.set_solver(kind=1)
        o.set_solver(kind=1)
    rng = np.random.default_rng(7)
    q, v = random_state(m, n, rng)
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    rows_seen = contacts_seen = flips = 0
    for t in range(150):
        g.set(Field.CTRL, range(n), rng.uniform(-1, 1, (n, m.nu)))
        if solver == "pgs":
            st = {f: g.get(f, range(n)) for f in (Field.QPOS, Field.QVEL, Field.QACC, Field.CTRL)}
            g.reset(range(n))
            o.reset(list(range(n)))
            for f, fo in ((Field.QPOS, QPOS), (Field.QVEL, QVEL), (Field.QACC, QACC), (Field.CTRL, CTRL)):
                g.set(f, range(n), st[f])
                o.set(fo, st[f])
        else:
            _copy_state(g, o, n)
        g.step(range(n), 1)
        o.step(0, n, 1)
        sg, so = g.stats(), o.stats()
        assert not sg["status"].any(), (t, sg["status"])
        np.testing.assert_array_equal(sg["ncon"], so["ncon"])
        np.testing.assert_array_equal(sg["nrows"], so["nrows"])
        rows_seen += int(so["nrows"].sum())
        contacts_seen += int(so["ncon"].sum())
        same = sg["iters"] == so["iters"] if solver == "pgs" else np.ones(n, bool)
        flips += int((~same).sum())
        for fg, fo in ((Field.QACC, QACC), (Field.QVEL, QVEL), (Field.QPOS, QPOS)):
            a, b = g.get(fg, range(n)), o.get(fo)
            for e in range(n):
                if same[e]:
                    assert rel(a[e], b[e]) < TOL_STEP, (t, e, fg, rel(a[e], b[e]))
                elif fg != Field.QACC:
                    assert np.max(np.abs(a[e] - b[e])) < 1e-4, (t, e, fg)
    assert rows_seen > 0 and contacts_seen > 0
    assert flips <= 0.01 * n * 150, flips


def _pgs_pair(name, n):
    m, g, o = pair(MODELS[name](), n)
    g.set_solver(kind=1)
    o.set_solver(kind=1)
    return m, g, o


@pytest.mark.parametrize("name,tol,resting", [("ant", TOL_STEP, False), ("box_drop", TOL_STEP, False),
                                              ("box_stack", 1e-4, True), ("shapes_on_box", 1e-4, True)])
def test_pgs_step_parity(name, tol, resting):
    """PGS (solver.rs:63-251) per step on identical input states, with the
    warm start cleared on both backends (reset, then the state set again),
    through falls, contacts and joint limits. A normal row's bias changes
    branch discontinuously where sep + slop crosses zero (solver.rs:176-181),
    which is where resting contacts sit: in the resting stacks a rounding
    difference in the depth can pick the other branch, after which the two
    runs agree only to the sweeps' own stopping tolerance, a 1e-5 velocity
    change (solver.rs:36). Those scenes are held to 1e-4 on qpos and qvel
    instead of 1e-10 on qpos, qvel and qacc."""
    n = 32
    m, g, o = _pgs_pair(name, n)
    T = min(int(round(0.6 / m.timestep)), 300)
    rng = np.random.default_rng(3)
    q, v = random_state(m, n, rng)
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    rows_seen = 0
    for t in range(T):
        if m.nu:
            g.set(Field.CTRL, range(n), rng.uniform(-1, 1, (n, m.nu)))
        st = {f: g.get(f, range(n)) for f in (Field.QPOS, Field.QVEL, Field.QACC, Field.CTRL)}
        g.reset(range(n))
        o.reset(list(range(n)))
        for f, fo in ((Field.QPOS, QPOS), (Field.QVEL, QVEL), (Field.QACC, QACC), (Field.CTRL, CTRL)):
            g.set(f, range(n), st[f])
            o.set(fo, st[f])
        g.step(range(n), 1)
        o.step(0, n, 1)
        sg, so = g.stats(), o.stats()
        assert not sg["status"].any()
        np.testing.assert_array_equal(sg["ncon"], so["ncon"])
        np.testing.assert_array_equal(sg["nrows"], so["nrows"])
        rows_seen += int(so["nrows"].sum())
        fields = ((Field.QPOS, QPOS), (Field.QVEL, QVEL)) + (() if resting else ((Field.QACC, QACC),))
        for fg, fo in fields:
            a, b = g.get(fg, range(n)), o.get(fo)
            for e in range(n):
                assert rel(a[e], b[e]) < tol, (t, e, fg, rel(a[e], b[e]))
    assert rows_seen > 0


def test_pgs_warm_start_trajectory():
    """PGS with its warm start (solver.rs:254-289) carried by each backend
    from step to step: boxes fall, land and settle; 0.8 s of trajectory."""
    n = 32
    m, g, o = _pgs_pair("box_drop", n)
    T = int(round(0.8 / m.timestep))
    rng = np.random.default_rng(3)
    q, v = random_state(m, n, rng)
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    o.set(QPOS, q)
    o.set(QVEL, v)
    contact_steps = 0
    for t in range(T):
        g.step(range(n), 1)
        o.step(0, n, 1)
        sg, so = g.stats(), o.stats()
        np.testing.assert_array_equal(sg["ncon"], so["ncon"])
        np.testing.assert_array_equal(sg["iters"], so["iters"])
        contact_steps += int((so["ncon"] > 0).sum())
    assert contact_steps > n * T // 4
    for fg, fo in ((Field.QPOS, QPOS), (Field.QVEL, QVEL)):
        assert rel(g.get(fg, range(n)), o.get(fo)) < TOL_TRAJ


@pytest.mark.parametrize("check", S.PARAM_CHECKS, ids=lambda f: f.__name__)
def test_param_behaviour(check):
    check(S.CudaSim)


def test_invalid_params_rejected():
    S.check_invalid_params_rejected(S.CudaSim, PhysicsError)


def test_poses_and_appearance_match_oracle():
    n = 16
    m, g, o = pair(scenes.ant_xml(), n)
    rng = np.random.default_rng(3)
    q, v = random_state(m, n, rng)
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    o.set(QPOS, q)
    o.set(QVEL, v)
    g.step(range(n), 5)
    o.step(0, n, 5)
    gg, gc = g.poses(range(n))
    og, oc = o.poses()
    np.testing.assert_allclose(gg, og, rtol=0, atol=1e-6)
    g.set_param(Param.GEOM_SIZE, 1, range(0, 2), [[0.3, 0, 0], [0.2, 0, 0]])
    o.set_param(1, 1, [[0.3, 0, 0], [0.2, 0, 0]], 0, 2)
    np.testing.assert_array_equal(g.appearance(range(n)), o.appearance())


def test_device_poses_equal_host_poses():
    """pg_poses_device writes the poses pg_poses returns, bit for bit, into
    device buffers, for a sub-range and in stream order after a step."""
    import torch
    n = 40
    xml = scenes.ant_xml().replace("</worldbody>", '<camera name="side" pos="0 -3 1" euler="70 0 0"/></worldbody>')
    m = mjcf.load_string(xml)
    ncam = len(m.cam_body)
    assert ncam >= 1
    g = CudaPhysics(mjcf.to_blob(m), n)
    rng = np.random.default_rng(4)
    q, v = random_state(m, n, rng)
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    dev = torch.device("cuda", 0)
    for s, e in ((0, n), (7, 31)):
        g.step(range(n), 3)
        hg, hc = g.poses(range(s, e))
        dg = torch.full(((e - s) * m.ngeom * 12,), float("nan"), dtype=torch.float32, device=dev)
        dc = torch.full(((e - s) * ncam * 12,), float("nan"), dtype=torch.float32, device=dev)
        torch.cuda.synchronize()
        g.poses_device(range(s, e), dg.data_ptr(), dc.data_ptr())
        g.synchronize()
        np.testing.assert_array_equal(dg.cpu().numpy().view(np.uint32), hg.reshape(-1).view(np.uint32))
        np.testing.assert_array_equal(dc.cpu().numpy().view(np.uint32), hc.reshape(-1).view(np.uint32))
    with pytest.raises(PhysicsError):
        g.poses_device(range(0, 2), 0, 0)
    g.close()


def test_device_views_are_the_state_in_place():
    """device_view gives zero-copy torch tensors over the handle's device
    state: they read what get() returns after each step, and controls written
    through the CTRL view drive the next steps exactly as set() does."""
    import torch
    n = 48
    m = mjcf.load_string(scenes.ant_xml())
    rng = np.random.default_rng(6)
    q, v = random_state(m, n, rng)
    ctrl = rng.uniform(-1, 1, (n, m.nu))
    a, b = CudaPhysics(mjcf.to_blob(m), n), CudaPhysics(mjcf.to_blob(m), n)
    for g in (a, b):
        g.set(Field.QPOS, range(n), q)
        g.set(Field.QVEL, range(n), v)
    qv, cv = b.device_view(Field.QPOS), b.device_view(Field.CTRL)
    assert qv.shape == (n, m.nq) and cv.shape == (n, m.nu) and qv.dtype == torch.float64 and qv.is_cuda
    assert qv.data_ptr() == b.device_ptr(Field.QPOS) and cv.data_ptr() == b.device_ptr(Field.CTRL)
    for k in range(3):
        a.set(Field.CTRL, range(n), ctrl * (k + 1) / 3)
        b.synchronize()
        cv.copy_(torch.from_numpy(ctrl * (k + 1) / 3).to(cv.device))
        torch.cuda.synchronize()
        a.step(range(n), 4)
        b.step(range(n), 4)
        b.synchronize()
        np.testing.assert_array_equal(qv.cpu().numpy(), b.get(Field.QPOS, range(n)))
        np.testing.assert_array_equal(b.get(Field.QPOS, range(n)), a.get(Field.QPOS, range(n)))
        np.testing.assert_array_equal(b.device_view(Field.QVEL).cpu().numpy(), a.get(Field.QVEL, range(n)))
    # a policy on the physics stream: the controls are computed from the
    # viewed qpos and stored in place, in stream order, with no host sync
    stream = torch.cuda.ExternalStream(b.stream(), device=qv.device)
    for _ in range(3):
        # (a halving and a clamp: exact on both sides, so both handles see the same controls)
        a.set(Field.CTRL, range(n), np.clip(0.5 * a.get(Field.QPOS, range(n))[:, 7:7 + m.nu], -1.0, 1.0))
        a.step(range(n), 2)
        with torch.cuda.stream(stream):
            cv.copy_(torch.clamp(0.5 * qv[:, 7:7 + m.nu], -1.0, 1.0))
            b.step(range(n), 2)
    b.synchronize()
    np.testing.assert_array_equal(qv.cpu().numpy(), a.get(Field.QPOS, range(n)))
    a.close()
    b.close()


def test_reset_keeps_qacc_and_restores_state():
    n = 4
    m, g, o = pair(scenes.ant_xml(), n)
    g.set(Field.CTRL, range(n), np.ones((n, m.nu)))
    g.step(range(n), 30)
    qacc = g.get(Field.QACC, range(n))
    g.set_param(Param.QPOS0, 0, range(1, 2), [np.array(m.qpos0) + 0.01])
    g.reset([1, 3])
    q = g.get(Field.QPOS, range(n))
    np.testing.assert_array_equal(q[1], np.array(m.qpos0) + 0.01)
    np.testing.assert_array_equal(q[3], np.array(m.qpos0))
    assert not g.get(Field.QVEL, range(n))[[1, 3]].any()
    assert not g.get(Field.CTRL, range(n))[[1, 3]].any()
    np.testing.assert_array_equal(g.get(Field.QACC, range(n)), qacc)


def test_subranges_step_like_the_whole():
    """Stepping halves separately equals stepping all envs (the async
    pipeline steps groups, backends_agree.rs:12-14)."""
    n = 32
    m = mjcf.load_string(scenes.ant_xml())
    blob = mjcf.to_blob(m)
    a, b = CudaPhysics(blob, n), CudaPhysics(blob, n)
    rng = np.random.default_rng(4)
    q, v = random_state(m, n, rng)
    for p in (a, b):
        p.set(Field.QPOS, range(n), q)
        p.set(Field.QVEL, range(n), v)
    a.step(range(n), 40)
    b.step(range(0, 13), 40)
    b.step(range(13, n), 40)
    np.testing.assert_array_equal(a.get(Field.QPOS, range(n)), b.get(Field.QPOS, range(n)))


def test_queued_newton_order_steps_like_one_wave():
    """With more envs than the Newton grid has tiles, the Newton phase takes
    envs in the order the collision phase wrote (envs with contacts first);
    with a tile per env it takes them in index order. Both must give every
    env the same bits: all 12000 envs at once against ranges of 2000 (one
    wave each), for pg_step and for pg_rollout (whose per-substep qpos goes
    to the env's own row of the output)."""
    n, t = 12000, 6
    m = mjcf.load_string(scenes.ant_xml(tolerance=1e-10))
    blob = mjcf.to_blob(m)
    a, b = CudaPhysics(blob, n), CudaPhysics(blob, n)
    lanes, per_block, blocks = a.phase_launch()["newton"]
    assert per_block * blocks < n  # the queued, ordered path
    rng = np.random.default_rng(12)
    q, v = random_state(m, n, rng, qnoise=0.3, vscale=0.5)
    q[:, 2] = rng.uniform(0.2, 0.9, n)  # torso heights: some envs touch the floor, others fly
    for p in (a, b):
        p.set(Field.QPOS, range(n), q)
        p.set(Field.QVEL, range(n), v)
    a.step(range(n), 30)
    for s0 in range(0, n, 2000):
        b.step(range(s0, min(n, s0 + 2000)), 30)
    assert a.stats()["ncon"].any() and not a.stats()["ncon"].all()
    for f in (Field.QPOS, Field.QVEL, Field.QACC):
        np.testing.assert_array_equal(a.get(f, range(n)), b.get(f, range(n)))
    np.testing.assert_array_equal(a.stats()["iters"], b.stats()["iters"])
    ctrl = rng.uniform(-1, 1, (n, t, m.nu))
    out_a = a.rollout(ctrl)
    out_b = np.concatenate([b.rollout(ctrl[s0:s0 + 2000], range(s0, min(n, s0 + 2000)))
                            for s0 in range(0, n, 2000)])
    np.testing.assert_array_equal(out_a, out_b)


def test_rollout_matches_step_loop():
    n, t = 8, 30
    m = mjcf.load_string(scenes.ant_xml())
    blob = mjcf.to_blob(m)
    a, b = CudaPhysics(blob, n), CudaPhysics(blob, n)
    ctrl = np.sin(np.arange(n * t * m.nu) * 0.37).reshape(n, t, m.nu)
    out = a.rollout(ctrl)
    for k in range(t):
        b.set(Field.CTRL, range(n), ctrl[:, k])
        b.step(range(n), 1)
    np.testing.assert_array_equal(out[:, -1], b.get(Field.QPOS, range(n)))


def test_errors_are_reported():
    g = CudaPhysics(scenes.ant_xml(), 4)
    with pytest.raises(PhysicsError):
        g.step(range(2, 9), 1)
    with pytest.raises(PhysicsError):
        g.get(Field.QPOS, range(4), out=np.zeros((4, 3)))
    with pytest.raises(PhysicsError):
        g.set(Field.CTRL, range(4), np.zeros(5))
    with pytest.raises(PhysicsError):
        g.reset([7])
    with pytest.raises(PhysicsError):
        CudaPhysics(b"not a model blob", 1)
    g.step(range(2, 2), 5)  # empty range is a no-op
    assert g.name() == "pippin-cuda"
    sc = g.scene()
    assert len(sc.geoms) == 14 and sc.geoms[0].name == "floor"


def test_zero_envs():
    g = CudaPhysics(scenes.ant_xml(), 0)
    g.step(range(0, 0), 3)
    assert g.get(Field.QPOS, range(0, 0)).shape == (0, 15)


def test_full_size_ant_properties():
    """Config 1 at full size (4096 envs x 200 steps, tol 1e-10): finite
    state, no status flags, unit free-joint quaternions, contacts present,
    and per-step parity on a sample of envs at the last step."""
    n, T = 4096, 200
    m, g, o = pair(scenes.ant_xml(), n, tolerance=1e-10)
    rng = np.random.default_rng(5)
    q, v = random_state(m, n, rng)
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    ctrl = rng.uniform(-1, 1, (n, T, m.nu))
    traj = g.rollout(ctrl)
    assert np.isfinite(traj).all()
    st = g.stats()
    assert not st["status"].any()
    quat = traj[:, -1, 3:7]
    np.testing.assert_allclose(np.linalg.norm(quat, axis=1), 1.0, atol=1e-12)
    sample = rng.choice(n, 64, replace=False)
    og = Oracle(mjcf.compile_string(scenes.ant_xml()), 64, threads=4)
    og.set_solver(tolerance=1e-10)
    for fg, fo in ((Field.QPOS, QPOS), (Field.QVEL, QVEL), (Field.QACC, QACC), (Field.CTRL, CTRL)):
        og.set(fo, g.get(fg, range(n))[sample])
    g.step(range(n), 1)
    og.step(0, 64, 1)
    assert rel(g.get(Field.QACC, range(n))[sample], og.get(QACC)) < TOL_STEP


def _tabletop_pair(n, seed=0):
    plan = scenes.tabletop(n, seed=seed)
    m = mjcf.load_string(plan.xml)
    blob = mjcf.to_blob(m)
    g = CudaPhysics(blob, n)
    o = Oracle(blob, n, threads=4)
    plan.apply(lambda p, elem, vals: g.set_param(Param(p), elem, range(n), vals), lambda: g.reset(range(n)))
    plan.apply(lambda p, elem, vals: o.set_param(p, elem, np.asarray(vals), 0, n), lambda: o.reset(list(range(n))))
    return m, g, o


def test_tabletop_step_parity():
    """Config 3 (tabletop, per-env objects by slot masks, sizes, masses and
    inertias): per-step Newton output on identical input states while the
    objects drop onto the table and land (tolerance 1e-10)."""
    n = 16
    m, g, o = _tabletop_pair(n)
    contacts_seen = 0
    for t in range(160):
        _copy_state(g, o, n)
        g.step(range(n), 1)
        o.step(0, n, 1)
        sg, so = g.stats(), o.stats()
        assert not sg["status"].any(), (t, sg["status"])
        np.testing.assert_array_equal(sg["ncon"], so["ncon"])
        contacts_seen += int(so["ncon"].sum())
        for fg, fo in ((Field.QACC, QACC), (Field.QVEL, QVEL), (Field.QPOS, QPOS)):
            a, b = g.get(fg, range(n)), o.get(fo)
            for e in range(n):
                assert rel(a[e], b[e]) < TOL_STEP, (t, e, fg, rel(a[e], b[e]))
    assert contacts_seen > n * 20


@pytest.mark.parametrize("solver,vmax", [(0, 1e-3), (1, 0.2)], ids=["newton", "pgs"])
def test_tabletop_objects_come_to_rest(solver, vmax):
    """Every active object of every env lands on the table and stops sliding
    within 2 s. Angular velocity is not checked: without torsional friction
    (the reference's contact model has none) an object set spinning about the
    vertical by an impact keeps spinning. PGS leaves slow rolling (the oracle
    shows up to 0.065 m/s after 2 s on these envs), Newton stops everything."""
    n = 64
    plan = scenes.tabletop(n, seed=1)
    m = mjcf.load_string(plan.xml)
    g = CudaPhysics(mjcf.to_blob(m), n)
    g.set_solver(kind=solver)
    plan.apply(lambda p, elem, vals: g.set_param(Param(p), elem, range(n), vals), lambda: g.reset(range(n)))
    g.step(range(n), int(round(2.0 / m.timestep)))
    q, v = g.get(Field.QPOS, range(n)), g.get(Field.QVEL, range(n))
    assert not g.stats()["status"].any()
    for e in range(n):
        for s in range(6):
            x, z = q[e, 7 * s], q[e, 7 * s + 2]
            if x < 50:  # active slot: on the table top (0.4 m) within its size, not sliding
                assert 0.4 < z < 0.5, (e, s, z)
                assert np.linalg.norm(v[e, 6 * s:6 * s + 3]) < vmax, (e, s, v[e, 6 * s:6 * s + 3])


def test_handles_with_different_launch_shapes():
    """A handle created after another with a larger launch shape must not
    shrink the kernels' shared-memory limit under it."""
    blob = mjcf.compile_string(scenes.ant_xml())
    big = CudaPhysics(blob, 512)
    big.set_launch(16, 16)
    small = CudaPhysics(blob, 64)
    small.set_launch(16, 2)
    big.step(range(512), 3)
    small.step(range(64), 3)
    assert not big.stats()["status"].any() and not small.stats()["status"].any()


def _sample_step_parity(g, blob, n, sample, params=(), tol=TOL_STEP):
    """One step of `sample` envs on the oracle from the GPU's current state
    (and the given per-env parameters) against the GPU's own step."""
    k = len(sample)
    og = Oracle(blob, k, threads=4)
    og.set_solver(tolerance=1e-10)
    for pid, elem, vals in params:
        og.set_param(pid, elem, np.asarray(vals)[sample], 0, k)
    for fg, fo in ((Field.QPOS, QPOS), (Field.QVEL, QVEL), (Field.QACC, QACC), (Field.CTRL, CTRL)):
        og.set(fo, g.get(fg, range(n))[sample])
    g.step(range(n), 1)
    og.step(0, k, 1)
    assert rel(g.get(Field.QACC, range(n))[sample], og.get(QACC)) < tol


@pytest.mark.parametrize("name", ["cartpole", "arm3hinge"])
def test_full_size_contact_free_properties(name):
    """Config 2 at full size (16384 envs, random states over the joint
    ranges, qvel N(0, 1), per-env masses x U[0.5, 2], 1 s): finite state, no
    status flags, invweight0 of sampled envs as the oracle's, and per-step
    parity on a sample of envs at the end."""
    n = 16384
    m = mjcf.load_string(MODELS[name]())
    blob = mjcf.to_blob(m)
    g = CudaPhysics(blob, n)
    g.set_solver(tolerance=1e-10)
    rng = np.random.default_rng(8)
    q = np.tile(np.array(m.qpos0), (n, 1))
    for j in range(m.njnt):
        qa = m.jnt_qposadr[j]
        if m.jnt_type[j] == mjcf.JNT_HINGE:
            q[:, qa] = rng.uniform(-np.pi, np.pi, n)
        elif m.jnt_type[j] == mjcf.JNT_SLIDE:
            q[:, qa] = rng.uniform(-0.5, 0.5, n)
    params = []
    for b in range(1, m.nbody):
        vals = (np.array(m.body_mass[b]) * rng.uniform(0.5, 2.0, n)).reshape(n, 1)
        g.set_param(Param.BODY_MASS, b, range(n), vals)
        params.append((5, b, vals))
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), rng.normal(0, 1, (n, m.nv)))
    steps = int(round(1.0 / m.timestep))
    traj = g.rollout(rng.uniform(-1, 1, (n, steps, max(m.nu, 0))))
    assert np.isfinite(traj).all()
    assert not g.stats()["status"].any()
    sample = rng.choice(n, 64, replace=False)
    _sample_step_parity(g, blob, n, sample, params)


def test_full_size_tabletop_properties():
    """Config 3 at full size (8192 envs, 2-6 objects each, 2 s at dt 0.002):
    finite state, no status flags, unit quaternions, no object through the
    floor, nearly every active object at rest on the table or on another
    object (a sphere set rolling keeps rolling: the contact model has no
    rolling friction), and per-step parity on a sample of envs."""
    n = 8192
    plan = scenes.tabletop(n, seed=9)
    m = mjcf.load_string(plan.xml)
    blob = mjcf.to_blob(m)
    g = CudaPhysics(blob, n)
    g.set_solver(tolerance=1e-10)
    params = []

    def setp(pid, elem, vals):
        g.set_param(Param(pid), elem, range(n), vals)
        params.append((pid, elem, np.asarray(vals).reshape(n, -1)))

    plan.apply(setp, lambda: g.reset(range(n)))
    g.step(range(n), int(round(2.0 / m.timestep)))
    q, v = g.get(Field.QPOS, range(n)), g.get(Field.QVEL, range(n))
    assert np.isfinite(q).all() and np.isfinite(v).all()
    assert not g.stats()["status"].any()
    resting, total = 0, 0
    for s in range(6):
        np.testing.assert_allclose(np.linalg.norm(q[:, 7 * s + 3:7 * s + 7], axis=1), 1.0, atol=1e-10)
        assert (q[:, 7 * s + 2] > 0.0).all()
        active = q[:, 7 * s] < 50
        z = q[active, 7 * s + 2]
        still = np.linalg.norm(v[active, 6 * s:6 * s + 3], axis=1) < 1e-3
        resting += int(((z > 0.4) & (z < 0.6) & still).sum())
        total += int(active.sum())
    assert resting >= 0.98 * total, (resting, total)
    sample = np.random.default_rng(9).choice(n, 32, replace=False)
    _sample_step_parity(g, blob, n, sample, [p for p in params if p[0] != 11])


def test_full_size_hull_tumble_properties():
    """Config 4 at full size (4096 envs of 8 hulls with 8-32 vertices, linear
    N(0, 0.5^2) and angular N(0, 3^2) velocities, 1 s, Newton): finite state,
    no status flags, unit quaternions, contacts, and per-step parity on a
    sample of envs."""
    n = 4096
    xml = scenes.hull_tumble_xml()
    m = mjcf.load_string(xml)
    blob = mjcf.to_blob(m)
    g = CudaPhysics(blob, n)
    g.set_solver(tolerance=1e-10)
    rng = np.random.default_rng(10)
    q = np.tile(np.array(m.qpos0), (n, 1))
    v = np.zeros((n, m.nv))
    for b in range(m.nv // 6):
        v[:, 6 * b:6 * b + 3] = rng.normal(0, 0.5, (n, 3))
        v[:, 6 * b + 3:6 * b + 6] = rng.normal(0, 3.0, (n, 3))
    g.set(Field.QPOS, range(n), q)
    g.set(Field.QVEL, range(n), v)
    g.step(range(n), int(round(1.0 / m.timestep)))
    q = g.get(Field.QPOS, range(n))
    st = g.stats()
    assert np.isfinite(q).all() and np.isfinite(g.get(Field.QVEL, range(n))).all()
    assert not st["status"].any()
    assert st["ncon"].mean() > 1
    for b in range(m.nq // 7):
        np.testing.assert_allclose(np.linalg.norm(q[:, 7 * b + 3:7 * b + 7], axis=1), 1.0, atol=1e-10)
    _sample_step_parity(g, blob, n, rng.choice(n, 32, replace=False))
