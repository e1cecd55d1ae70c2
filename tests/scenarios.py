"""Behavioural scenarios of the reference's integration tests, runnable on
either backend (the oracle on the CPU, the CUDA backend on a GPU).

Each check mirrors one test of crates/pippin/tests/contact.rs or
crates/pippin-env/tests/params.rs (cited per function) with the same
scene, duration and tolerance; the scenes are written here as MJCF.
"""
import math

import numpy as np

from pippin_b200 import mjcf, scenes

NEWTON, PGS = 0, 1


class OracleSim:
    """Adapter over oracle.Oracle with the calls the scenarios use."""

    def __init__(self, xml, n=1, solver=NEWTON):
        from oracle.oracle import Oracle
        self.m = mjcf.load_string(xml)
        self.o = Oracle(mjcf.to_blob(self.m), n, threads=1)
        self.o.set_solver(kind=solver)

    def step(self, nstep, start=0, end=None):
        self.o.step(start, end, nstep)

    def qpos(self):
        from oracle.oracle import QPOS
        return self.o.get(QPOS)

    def qvel(self):
        from oracle.oracle import QVEL
        return self.o.get(QVEL)

    def set_ctrl(self, c):
        from oracle.oracle import CTRL
        self.o.set(CTRL, c)

    def set_param(self, p, elem, values, start, end):
        self.o.set_param(p, elem, values, start, end)

    def get_param(self, p, elem, start, end):
        return self.o.get_param(p, elem, start, end)

    def appearance(self):
        return self.o.appearance()

    def body_pos(self, name, env=0):
        b = self.m.body_id(name)
        return self.o.body_poses(env)[b, :3]


class CudaSim:
    """Adapter over pippin_b200.CudaPhysics with the same calls."""

    def __init__(self, xml, n=1, solver=NEWTON):
        from pippin_b200 import CudaPhysics
        self.m = mjcf.load_string(xml)
        self.p = CudaPhysics(mjcf.to_blob(self.m), n)
        self.n = n
        if solver != NEWTON:
            self.p.set_solver(kind=solver)

    def step(self, nstep, start=0, end=None):
        self.p.step(range(start, self.n if end is None else end), nstep)

    def qpos(self):
        from pippin_b200 import Field
        return self.p.get(Field.QPOS, range(self.n))

    def qvel(self):
        from pippin_b200 import Field
        return self.p.get(Field.QVEL, range(self.n))

    def set_ctrl(self, c):
        from pippin_b200 import Field
        self.p.set(Field.CTRL, range(self.n), c)

    def set_param(self, p, elem, values, start, end):
        self.p.set_param(p, elem, range(start, end), values)

    def get_param(self, p, elem, start, end):
        return self.p.get_param(p, elem, range(start, end))

    def appearance(self):
        return self.p.appearance(range(self.n))

    def body_pos(self, name, env=0):
        # free-joint bodies: world position is the joint's qpos
        b = self.m.body_id(name)
        j = self.m.body_jntadr[b]
        qa = self.m.jnt_qposadr[j]
        return self.qpos()[env, qa:qa + 3]


def free_body_pos(sim, name, env=0):
    m = sim.m
    b = m.body_id(name)
    qa = m.jnt_qposadr[m.body_jntadr[b]]
    return sim.qpos()[env, qa:qa + 3]


def steps(sim, seconds):
    return int(round(seconds / sim.m.timestep))


# ---- crates/pippin/tests/contact.rs
BOX_ON_PLANE = ('<mujoco><worldbody><geom type="plane" size="5 5 .1"/>'
                '<body name="b" pos="0 0 0.3" euler="3 5 0"><freejoint/><geom type="box" size=".1 .1 .1"/></body>'
                '</worldbody></mujoco>')


def check_box_rests_on_plane(make, solver):
    """contact.rs:30-47"""
    s = make(BOX_ON_PLANE, 1, solver)
    s.step(steps(s, 3.0))
    p = free_body_pos(s, "b")
    assert abs(p[2] - 0.1) < 2e-3, p
    assert abs(p[0]) < 1e-2 and abs(p[1]) < 1e-2, p
    assert np.linalg.norm(s.qvel()[0]) < 1e-3


SPHERE_CAPSULE = ('<mujoco><worldbody><geom type="plane" size="5 5 .1"/>'
                  '<body name="s" pos="0 0 0.5"><freejoint/><geom type="sphere" size=".05"/></body>'
                  '<body name="c" pos="1 0 0.5" euler="90 0 0"><freejoint/><geom type="capsule" size=".04 .2"/></body>'
                  '</worldbody></mujoco>')


def check_sphere_and_capsule_rest(make, solver):
    """contact.rs:49-63"""
    s = make(SPHERE_CAPSULE, 1, solver)
    s.step(steps(s, 3.0))
    assert abs(free_body_pos(s, "s")[2] - 0.05) < 2e-3
    assert abs(free_body_pos(s, "c")[2] - 0.04) < 2e-3


def box_stack_xml(n=5):
    body = "".join(f'<body name="b{i}" pos="0 0 {0.05 + 0.1 * i + 0.001 * i!r}"><freejoint/>'
                   f'<geom type="box" size=".05 .05 .05"/></body>' for i in range(n))
    return f'<mujoco><option timestep="0.002"/><worldbody><geom type="plane" size="5 5 .1"/>{body}</worldbody></mujoco>'


def check_box_stack_is_stable(make, solver):
    """contact.rs:65-81"""
    s = make(box_stack_xml(), 1, solver)
    s.step(steps(s, 5.0))
    top = free_body_pos(s, "b4")
    assert abs(top[0]) < 5e-3 and abs(top[1]) < 5e-3, top
    assert abs(top[2] - 0.45) < 1e-2, top


def incline_xml(deg, mu):
    return ('<mujoco><option timestep="0.002"/><worldbody>'
            f'<geom type="plane" size="5 5 .1" euler="0 {deg!r} 0" friction="{mu!r}"/>'
            f'<body name="b" pos="0 0 0.1" euler="0 {deg!r} 0"><freejoint/>'
            f'<geom type="box" size=".05 .05 .05" friction="{mu!r}"/></body></worldbody></mujoco>')


def check_friction_holds(make, solver):
    """contact.rs:92-102: tan(20 deg) < mu = 0.5 sticks"""
    s = make(incline_xml(20.0, 0.5), 1, solver)
    s.step(steps(s, 0.5))
    p0 = free_body_pos(s, "b").copy()
    s.step(steps(s, 1.0))
    p1 = free_body_pos(s, "b")
    assert np.linalg.norm(p1 - p0) < 2e-3


def check_friction_slides(make, solver):
    """contact.rs:104-121: a = g (sin t - mu cos t) within 3%"""
    deg, mu = 35.0, 0.3
    s = make(incline_xml(deg, mu), 1, solver)
    s.step(steps(s, 0.3))
    v0 = np.linalg.norm(s.qvel()[0, :3])
    s.step(steps(s, 0.5))
    v1 = np.linalg.norm(s.qvel()[0, :3])
    t = math.radians(deg)
    expected = 9.81 * (math.sin(t) - mu * math.cos(t))
    measured = (v1 - v0) / 0.5
    assert abs(measured - expected) / expected < 0.03, (measured, expected)


HINGE_LIMIT = ('<mujoco><option timestep="0.002"/><worldbody>'
               '<body pos="0 0 1"><joint name="h" axis="0 1 0" range="-30 30"/>'
               '<geom type="capsule" fromto="0 0 0 0.5 0 0" size="0.03" contype="0" conaffinity="0"/></body>'
               '</worldbody></mujoco>')


def check_joint_limit(make, solver):
    """contact.rs:123-142"""
    s = make(HINGE_LIMIT, 1, solver)
    qmax = 0.0
    for _ in range(20):
        s.step(100)
        qmax = max(qmax, s.qpos()[0, 0])
    lim = math.radians(30)
    assert qmax < lim + 0.05
    assert abs(s.qpos()[0, 0] - lim) < 0.01


ON_BOX = ('<mujoco><worldbody><geom type="box" size="1 1 .1" pos="0 0 -.1"/>'
          '<body name="s" pos="0 0 0.3"><freejoint/><geom type="sphere" size=".05"/></body>'
          '<body name="c" pos="0.5 0 0.3" euler="0 90 0"><freejoint/><geom type="capsule" size=".03 .1"/></body>'
          '<body name="bx" pos="-0.5 0 0.3" euler="0 0 30"><freejoint/><geom type="box" size=".05 .05 .05"/></body>'
          '</worldbody></mujoco>')


def check_shapes_on_box(make, solver):
    """contact.rs:144-160"""
    s = make(ON_BOX, 1, solver)
    s.step(steps(s, 3.0))
    assert abs(free_body_pos(s, "s")[2] - 0.05) < 2e-3
    assert abs(free_body_pos(s, "c")[2] - 0.03) < 2e-3
    assert abs(free_body_pos(s, "bx")[2] - 0.05) < 2e-3


# ---- crates/pippin-env/tests/params.rs
INCLINE_PARAMS = ('<mujoco><option timestep="0.002"/><worldbody>'
                  '<geom name="floor" type="plane" size="5 5 .1" euler="0 25 0" friction="0.1"/>'
                  '<body name="b" pos="0 0 0.1" euler="0 25 0"><freejoint/>'
                  '<geom name="box" type="box" size=".05 .05 .05" friction="0.1"/></body></worldbody></mujoco>')
GEOM_FRICTION, GEOM_SIZE, GEOM_CONTYPE, GEOM_CONAFFINITY, BODY_MASS = 0, 1, 3, 4, 5


def check_friction_per_env(make):
    """params.rs:21-37"""
    s = make(INCLINE_PARAMS, 2, NEWTON)
    floor, boxg = 0, 1
    s.set_param(GEOM_FRICTION, boxg, [0.9], 1, 2)
    s.set_param(GEOM_FRICTION, floor, [0.9], 1, 2)
    s.step(500)
    q = s.qpos()
    slid = lambda r: math.hypot(r[0], r[1])
    assert slid(q[0]) > 0.1
    assert slid(q[1]) < 0.01
    out = s.get_param(GEOM_FRICTION, boxg, 0, 2)
    assert list(out[:, 0]) == [0.1, 0.9]


BALL = ('<mujoco><worldbody><geom type="plane" size="5 5 .1"/>'
        '<body pos="0 0 0.3"><freejoint/><geom name="ball" type="sphere" size=".05"/></body></worldbody></mujoco>')


def check_size_and_parking(make):
    """params.rs:39-59"""
    s = make(BALL, 3, NEWTON)
    s.set_param(GEOM_SIZE, 1, [0.1, 0.0, 0.0], 1, 2)
    s.set_param(GEOM_CONTYPE, 1, [0.0], 2, 3)
    s.set_param(GEOM_CONAFFINITY, 1, [0.0], 2, 3)
    s.step(1000)
    q = s.qpos()
    assert abs(q[0, 2] - 0.05) < 2e-3
    assert abs(q[1, 2] - 0.10) < 2e-3
    assert q[2, 2] < -1.0
    ap = s.appearance()  # (envs, ngeom, 8): rgba[4], scale[3], pad
    assert ap[2, 1, 4] == 1.0 and ap[1, 1, 4] == 2.0
    assert ap[0, 1, 4] == 1.0


MASS_LINK = ('<mujoco><option gravity="0 0 0"/><worldbody>'
             '<body name="link"><joint name="j" axis="0 0 1"/>'
             '<geom type="capsule" fromto="0 0 0 0.3 0 0" size="0.02" mass="1"/></body></worldbody>'
             '<actuator><motor joint="j"/></actuator></mujoco>')


def check_mass_per_env(make):
    """params.rs:61-74: 4x mass -> 1/4 the angle"""
    s = make(MASS_LINK, 2, NEWTON)
    s.set_param(BODY_MASS, 1, [4.0], 1, 2)
    s.set_ctrl(np.array([[1.0], [1.0]]))
    s.step(200)
    q = s.qpos()
    assert abs(q[0, 0] / q[1, 0] - 4.0) < 1e-6


def check_invalid_params_rejected(make, error):
    """params.rs:76-85"""
    import pytest
    s = make(INCLINE_PARAMS, 2, NEWTON)
    with pytest.raises(error):
        s.set_param(GEOM_SIZE, 0, [1.0] * 6, 0, 2)
    with pytest.raises(error):
        s.set_param(GEOM_FRICTION, 99, [1.0], 0, 1)
    with pytest.raises(error):
        s.set_param(BODY_MASS, 1, [-1.0], 0, 1)
    out = s.get_param(GEOM_FRICTION, 1, 0, 2)
    assert list(out[:, 0]) == [0.1, 0.1]


# ---- crates/pippin/tests/mesh.rs (the general convex narrow phase)
CUBE = ("-0.05 -0.05 -0.05  0.05 -0.05 -0.05  -0.05 0.05 -0.05  0.05 0.05 -0.05 "
        "-0.05 -0.05 0.05  0.05 -0.05 0.05  -0.05 0.05 0.05  0.05 0.05 0.05")
MESH_AND_BOX = ('<mujoco><asset><mesh name="cube" vertex="' + CUBE + '"/></asset><worldbody>'
                '<geom type="plane" size="5 5 .1"/>'
                '<body name="m" pos="0 0 0.3" euler="4 7 0"><freejoint/><geom type="mesh" mesh="cube"/></body>'
                '<body name="b" pos="1 0 0.3" euler="4 7 0"><freejoint/><geom type="box" size=".05 .05 .05"/></body>'
                '</worldbody></mujoco>')


def mesh_stack_xml(n=4):
    xml = ('<mujoco><asset><mesh name="cube" vertex="' + CUBE + '"/></asset><worldbody>'
           '<geom type="plane" size="5 5 .1"/>')
    for i in range(n):
        xml += (f'<body name="c{i}" pos="0 0 {0.05 + 0.101 * i}" euler="0 0 {9 * i}"><freejoint/>'
                '<geom type="mesh" mesh="cube"/></body>')
    return xml + '</worldbody></mujoco>'


CYLINDERS = ('<mujoco><worldbody><geom type="box" size="1 1 .1" pos="0 0 -.1"/>'
             '<body name="up" pos="0 0 0.3"><freejoint/><geom type="cylinder" size=".04 .06"/></body>'
             '<body name="side" pos="0.5 0 0.3" euler="90 0 0"><freejoint/><geom type="cylinder" size=".04 .06"/></body>'
             '<body name="onup" pos="0 0 0.5"><freejoint/><geom type="cylinder" size=".03 .03"/></body>'
             '</worldbody></mujoco>')


def check_mesh_cube_rests_like_box(make, solver):
    """mesh.rs:24-45"""
    s = make(MESH_AND_BOX, 1, solver)
    s.step(steps(s, 3.0))
    zm, zb = free_body_pos(s, "m")[2], free_body_pos(s, "b")[2]
    assert abs(zm - zb) < 1e-3, (zm, zb)
    assert abs(zm - 0.05) < 2e-3, zm
    assert np.linalg.norm(s.qvel()[0]) < 1e-3, np.linalg.norm(s.qvel()[0])


def check_mesh_cubes_stack(make, solver):
    """mesh.rs:47-64"""
    s = make(mesh_stack_xml(), 1, solver)
    s.step(steps(s, 5.0))
    top = free_body_pos(s, "c3")
    assert abs(top[0]) < 5e-3 and abs(top[1]) < 5e-3, top
    assert abs(top[2] - 0.35) < 1e-2, top


def check_cylinders_rest(make, solver):
    """mesh.rs:66-82"""
    s = make(CYLINDERS, 1, solver)
    s.step(steps(s, 3.0))
    assert abs(free_body_pos(s, "up")[2] - 0.06) < 2e-3, free_body_pos(s, "up")
    assert abs(free_body_pos(s, "side")[2] - 0.04) < 2e-3, free_body_pos(s, "side")
    assert abs(free_body_pos(s, "onup")[2] - 0.15) < 3e-3, free_body_pos(s, "onup")


GENERAL_CHECKS = [check_mesh_cube_rests_like_box, check_mesh_cubes_stack, check_cylinders_rest]
CONTACT_CHECKS = [check_box_rests_on_plane, check_sphere_and_capsule_rest, check_box_stack_is_stable,
                  check_friction_holds, check_friction_slides, check_joint_limit, check_shapes_on_box]
PARAM_CHECKS = [check_friction_per_env, check_size_and_parking, check_mass_per_env]


# ---- hot-path branches the workload models do not reach: joint equality rows
# (newton.rs:171-195), fixed-tendon transmissions (mjcf.rs:852-947) and the
# implicitfast actuator terms (forward.rs:407-431). Each scene also touches
# the floor, so that equality / limit rows meet contact rows in one solve.
EQUALITY_CHAIN = (
    '<mujoco><option timestep="0.005"/><worldbody><geom type="plane" size="5 5 .1"/>'
    '<body name="l1" pos="0 0 0.55"><joint name="j1" axis="0 1 0" range="-100 100"/>'
    '<geom type="capsule" fromto="0 0 0 0.22 0 0" size="0.03"/>'
    '<body name="l2" pos="0.22 0 0"><joint name="j2" axis="0 1 0"/>'
    '<geom type="capsule" fromto="0 0 0 0.22 0 0" size="0.03"/>'
    '<body name="l3" pos="0.22 0 0"><joint name="j3" axis="0 1 0"/><joint name="j3b" axis="1 0 0"/>'
    '<geom type="capsule" fromto="0 0 0 0.2 0 0" size="0.03"/>'
    '<body name="tip" pos="0.2 0 0"><joint name="j4" type="slide" axis="1 0 0" range="-0.05 0.05"/>'
    '<geom type="sphere" size="0.05"/></body></body></body></body>'
    '<body name="ball" pos="0.3 0.02 0.2"><freejoint/><geom type="sphere" size="0.06"/></body>'
    '</worldbody>'
    '<equality><joint joint1="j2" joint2="j1" polycoef="0.1 0.5 0.3 -0.05 0.01"/>'
    '<joint joint1="j3b"/><joint joint1="j4" joint2="j3" polycoef="0 0.02 0 0 0" solref="0.05 1"/></equality>'
    '<actuator><motor joint="j1" gear="8"/><motor joint="j3" gear="3"/></actuator></mujoco>')

TENDON_ARM = (
    '<mujoco><option timestep="0.004"/><worldbody><geom type="plane" size="5 5 .1"/>'
    '<body name="base" pos="0 0 0.45"><joint name="yaw" axis="0 0 1" damping="0.2"/>'
    '<geom type="cylinder" size="0.05 0.04"/>'
    '<body name="up" pos="0 0 0.05"><joint name="sh" axis="0 1 0" range="-120 120"/>'
    '<geom type="capsule" fromto="0 0 0 0.25 0 0" size="0.035"/>'
    '<body name="fore" pos="0.25 0 0"><joint name="el" axis="0 1 0" range="-150 150"/>'
    '<geom type="capsule" fromto="0 0 0 0.22 0 0" size="0.03"/>'
    '<body name="hand" pos="0.22 0 0"><joint name="wr" axis="1 0 0"/>'
    '<geom type="box" size="0.06 0.05 0.04"/></body></body></body></body></worldbody>'
    '<tendon><fixed name="flex"><joint joint="sh" coef="1"/><joint joint="el" coef="-0.5"/></fixed>'
    '<fixed name="twist"><joint joint="yaw" coef="0.3"/><joint joint="wr" coef="1"/></fixed></tendon>'
    '<actuator><motor tendon="flex" gear="12" ctrlrange="-1 1"/><motor tendon="twist" gear="0.3"/>'
    '<motor joint="el" gear="4"/></actuator></mujoco>')

IMPLICITFAST_ARM = (
    '<mujoco><option timestep="0.005" integrator="implicitfast"/>'
    '<default><joint damping="0.05" armature="0.01"/></default>'
    '<worldbody><geom type="plane" size="5 5 .1"/>'
    '<body name="base" pos="0 0 0.4"><joint name="a0" axis="0 0 1"/>'
    '<geom type="cylinder" size="0.05 0.04"/>'
    '<body name="l1" pos="0 0 0.05"><joint name="a1" axis="0 1 0" range="-110 110"/>'
    '<geom type="capsule" fromto="0 0 0 0.24 0 0" size="0.035"/>'
    '<body name="l2" pos="0.24 0 0"><joint name="a2" axis="0 1 0"/>'
    '<geom type="capsule" fromto="0 0 0 0.22 0 0" size="0.03"/>'
    '<body name="l3" pos="0.22 0 0"><joint name="a3" type="slide" axis="1 0 0" range="-0.04 0.04"/>'
    '<geom type="box" size="0.035 0.035 0.035"/></body></body></body></body>'
    '<body name="block" pos="0.35 0 0.05"><freejoint/><geom type="box" size="0.05 0.05 0.05"/></body>'
    '</worldbody>'
    '<actuator><position joint="a1" kp="40" kv="4"/><velocity joint="a2" kv="3"/>'
    '<position joint="a0" kp="10" kv="1" ctrlrange="-1 1"/><velocity joint="a3" kv="5" forcerange="-2 2"/>'
    '<motor joint="a2" gear="2"/></actuator></mujoco>')


# ----------------------------------------------------------------- large hulls
# the reference's support-walk test inputs and the large-hull scene, kept in
# the package for the bench
lumpy_sphere_points = scenes.lumpy_sphere_points
support_directions = scenes.support_directions
big_hulls_xml = scenes.big_hulls_xml
