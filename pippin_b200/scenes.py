"""Model builders for the workloads: MJCF strings generated in code.

The Ant, cartpole, 3-D arm, pendulum, box-drop and tumble models compile to
the same model blob as the reference repository's `assets/*.xml` (checked by
tests/test_scenes.py where that repository is available), so parity and
benchmark runs do not depend on files outside this package.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

# (leg body, hip joint, ankle joint, outward direction in xy, ankle axis, ankle range in degrees)
_ANT_LEGS = [
    ("front_left_leg", "aux_1", 1, (1, 1), "-1 1 0", "30 70"),
    ("front_right_leg", "aux_2", 2, (-1, 1), "1 1 0", "-70 -30"),
    ("back_leg", "aux_3", 3, (-1, -1), "-1 1 0", "-70 -30"),
    ("right_back_leg", "aux_4", 4, (1, -1), "1 1 0", "30 70"),
]
_ANT_ACTUATED = [4, 1, 2, 3]  # actuator order: legs 4, 1, 2, 3 (hip then ankle)


def _fmt(x: float) -> str:
    return repr(float(x)) if not float(x).is_integer() else str(int(x))


def ant_xml(timestep: float = 0.01, solver: Optional[str] = None, iterations: Optional[int] = None,
            tolerance: Optional[float] = None) -> str:
    """Four-legged Ant: free-joint sphere torso, 4 legs of 2 hinges with capsule
    geoms, 8 motors (gear 150, ctrl in [-1, 1]), plane floor; nq=15, nv=14."""
    opts = [f'timestep="{_fmt(timestep)}"']
    if solver:
        opts.append(f'solver="{solver}"')
    if iterations is not None:
        opts.append(f'iterations="{iterations}"')
    if tolerance is not None:
        opts.append(f'tolerance="{tolerance!r}"')
    legs = []
    for leg, aux, k, (sx, sy), axis, rng in _ANT_LEGS:
        a = f"{_fmt(0.2 * sx)} {_fmt(0.2 * sy)} 0"
        f = f"{_fmt(0.4 * sx)} {_fmt(0.4 * sy)} 0"
        legs.append(
            f'<body name="{leg}"><geom type="capsule" fromto="0 0 0 {a}" size="0.08"/>'
            f'<body name="{aux}" pos="{a}"><joint name="hip_{k}" axis="0 0 1" range="-30 30"/>'
            f'<geom type="capsule" fromto="0 0 0 {a}" size="0.08"/>'
            f'<body pos="{a}"><joint name="ankle_{k}" axis="{axis}" range="{rng}"/>'
            f'<geom type="capsule" fromto="0 0 0 {f}" size="0.08"/></body></body></body>')
    motors = "".join(f'<motor joint="hip_{k}"/><motor joint="ankle_{k}"/>' for k in _ANT_ACTUATED)
    return (
        '<mujoco model="ant"><compiler angle="degree"/>'
        f'<option {" ".join(opts)}/>'
        '<default><joint armature="1" damping="1"/>'
        '<geom density="5.0" friction="1 0.5 0.5" rgba="0.8 0.6 0.4 1"/>'
        '<motor ctrlrange="-1 1" gear="150"/></default>'
        '<worldbody><geom name="floor" type="plane" size="40 40 40" rgba="0.8 0.9 0.8 1"/>'
        '<body name="torso" pos="0 0 0.75"><freejoint name="root"/>'
        '<geom name="torso_geom" type="sphere" size="0.25"/>'
        + "".join(legs) +
        f'</body></worldbody><actuator>{motors}</actuator></mujoco>')


def cartpole_xml() -> str:
    """Cart on a slider with a two-link pole (no contacts); nq=nv=3, nu=2."""
    return (
        '<mujoco model="cartpole"><option timestep="0.005"/>'
        '<default><geom contype="0" conaffinity="0"/><joint damping="0.02"/></default>'
        '<worldbody><body name="cart" pos="0 0 0.5">'
        '<joint name="slider" type="slide" axis="1 0 0"/>'
        '<geom type="box" size="0.2 0.1 0.05" density="500"/>'
        '<body name="pole" pos="0 0 0"><joint name="hinge" type="hinge" axis="0 1 0" armature="0.01"/>'
        '<geom type="capsule" fromto="0 0 0 0.02 0 0.6" size="0.03"/>'
        '<body name="pole2" pos="0.02 0 0.6"><joint name="hinge2" type="hinge" axis="0 1 0" ref="10"/>'
        '<geom type="capsule" fromto="0 0 0 0 0 0.5" size="0.025"/></body></body></body></worldbody>'
        '<actuator><motor joint="slider" gear="10" ctrlrange="-1 1"/>'
        '<position joint="hinge2" kp="5" kv="0.2"/></actuator></mujoco>')


def arm3d_xml() -> str:
    """3-D arm with hinge, two-hinge, ball and slide joints, position and
    velocity actuators (no contacts); nq=9, nv=8, nu=4."""
    return (
        '<mujoco model="arm3d"><compiler angle="radian"/>'
        '<option timestep="0.002" gravity="0 0 -9.81"/>'
        '<default><geom contype="0" conaffinity="0" density="800"/>'
        '<default class="link"><joint damping="0.1" armature="0.02"/></default></default>'
        '<worldbody><body name="base" pos="0 0 0.3" euler="0 0 0.3" childclass="link">'
        '<joint name="j0" axis="0 0 1"/><geom type="cylinder" size="0.06 0.05"/>'
        '<body name="l1" pos="0 0 0.08" quat="0.9 0.1 0.2 0.1">'
        '<joint name="j1" axis="0 1 0" pos="0 0 -0.02"/>'
        '<geom type="capsule" fromto="0 0 0 0.3 0 0.1" size="0.04"/>'
        '<body name="l2" pos="0.3 0 0.1" xyaxes="0 1 0 -1 0 0">'
        '<joint name="j2" axis="1 0 0"/><joint name="j2b" axis="0 0 1"/>'
        '<geom type="box" size="0.12 0.03 0.02" pos="0.1 0 0" euler="0.2 0.1 0"/>'
        '<body name="l3" pos="0.22 0 0"><joint name="j3" type="ball" pos="0.01 0.02 0"/>'
        '<geom type="sphere" size="0.05" pos="0.05 0.01 0"/>'
        '<geom type="capsule" size="0.02 0.05" pos="0.1 0 0" zaxis="1 0 0"/>'
        '<body name="finger" pos="0.15 0 0"><joint name="j4" type="slide" axis="0 1 1"/>'
        '<inertial pos="0.01 0 0" mass="0.1" diaginertia="0.001 0.002 0.0015" quat="0.8 0.6 0 0"/>'
        '<geom type="box" size="0.02 0.02 0.02"/></body></body></body></body></body></worldbody>'
        '<actuator><motor joint="j0" gear="5"/><position joint="j1" kp="20" kv="1"/>'
        '<velocity joint="j2" kv="2"/><motor joint="j4"/></actuator></mujoco>')


def arm3hinge_xml() -> str:
    """Three-link 3-D hinge arm (yaw, pitch, pitch), no contacts; nq=nv=nu=3."""
    return (
        '<mujoco model="arm3hinge"><option timestep="0.002"/>'
        '<default><geom contype="0" conaffinity="0" density="1000"/>'
        '<joint damping="0.05" armature="0.01"/></default>'
        '<worldbody><body name="l0" pos="0 0 0.5"><joint name="yaw" axis="0 0 1"/>'
        '<geom type="capsule" fromto="0 0 0 0 0 0.2" size="0.04"/>'
        '<body name="l1" pos="0 0 0.2"><joint name="shoulder" axis="0 1 0"/>'
        '<geom type="capsule" fromto="0 0 0 0.3 0 0" size="0.035"/>'
        '<body name="l2" pos="0.3 0 0"><joint name="elbow" axis="0 1 0"/>'
        '<geom type="capsule" fromto="0 0 0 0.25 0 0.05" size="0.03"/>'
        '</body></body></body></worldbody>'
        '<actuator><motor joint="yaw" gear="2"/><motor joint="shoulder" gear="4"/>'
        '<motor joint="elbow" gear="2"/></actuator></mujoco>')


def pendulum_xml() -> str:
    return (
        '<mujoco model="pendulum"><option timestep="0.002"/><worldbody>'
        '<body name="pole" pos="0 0 1"><joint name="hinge" type="hinge" axis="0 1 0" damping="0.05"/>'
        '<geom type="capsule" fromto="0 0 0 0 0 -0.5" size="0.04" contype="0" conaffinity="0"/>'
        '</body></worldbody><actuator><motor joint="hinge" gear="2" ctrlrange="-1 1"/></actuator></mujoco>')


def box_drop_xml() -> str:
    """Box, sphere and capsule dropped on a plane (free joints)."""
    return (
        '<mujoco model="box_drop"><option timestep="0.002"/><worldbody>'
        '<geom type="plane" size="5 5 .1"/>'
        '<body pos="0 0 0.3" euler="10 20 5"><freejoint/><geom type="box" size=".05 .05 .05"/></body>'
        '<body pos="0.3 0 0.2"><freejoint/><geom type="sphere" size=".04"/></body>'
        '<body pos="-0.3 0 0.2" euler="0 80 30"><freejoint/><geom type="capsule" size=".03 .08"/></body>'
        '</worldbody></mujoco>')


def tumble_xml() -> str:
    return (
        '<mujoco model="tumble"><option timestep="0.001" gravity="0 0 -9.81"/><worldbody>'
        '<body name="brick" pos="0.1 -0.2 1" euler="20 30 40"><freejoint/>'
        '<geom type="box" size="0.3 0.1 0.05" contype="0" conaffinity="0"/>'
        '<body name="appendage" pos="0.3 0 0"><joint type="hinge" axis="0 0 1" damping="0.01"/>'
        '<geom type="capsule" fromto="0 0 0 0.2 0.1 0" size="0.02" contype="0" conaffinity="0"/>'
        '</body></body></worldbody></mujoco>')


REFERENCE_ASSETS = {
    "ant.xml": ant_xml,
    "cartpole.xml": cartpole_xml,
    "arm3d.xml": arm3d_xml,
    "pendulum.xml": pendulum_xml,
    "box_drop.xml": box_drop_xml,
    "tumble.xml": tumble_xml,
}


def hull_tumble_xml(n_hulls: int = 8, seed: int = 0, timestep: float = 0.002) -> str:
    """Convex hulls tumbling onto a plane (the general convex narrow phase):
    `n_hulls` free bodies, each a mesh of 8 to 32 points drawn uniformly on
    an ellipsoid with semi-axes U[0.02, 0.06] (hulled by the model compiler),
    placed on a grid 0.25 m above the floor with a random orientation."""
    import numpy as np

    rng = np.random.default_rng(seed)
    assets, bodies = [], []
    for i in range(n_hulls):
        npt = int(rng.integers(8, 33))
        axes = rng.uniform(0.02, 0.06, 3)
        d = rng.normal(size=(npt, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        pts = d * axes
        assets.append(f'<mesh name="h{i}" vertex="{" ".join(_fmt(round(x, 6)) for x in pts.ravel())}"/>')
        x, y = 0.15 * (i % 4) - 0.225, 0.15 * (i // 4) - 0.075
        e = rng.uniform(-180, 180, 3)
        bodies.append(f'<body name="b{i}" pos="{_fmt(round(x, 4))} {_fmt(round(y, 4))} 0.25" '
                      f'euler="{_fmt(round(e[0], 3))} {_fmt(round(e[1], 3))} {_fmt(round(e[2], 3))}">'
                      f'<freejoint/><geom type="mesh" mesh="h{i}"/></body>')
    return (f'<mujoco model="hull_tumble"><option timestep="{_fmt(timestep)}"/><asset>{"".join(assets)}</asset>'
            f'<worldbody><geom name="floor" type="plane" size="5 5 .1"/>{"".join(bodies)}</worldbody></mujoco>')


class TabletopPlan:
    """A tabletop model shared by every env plus the per-env parameters that
    make each env different (the slot scheme of python/pippin/scene.py:21-25,
    325-346): each object slot is a free body holding one geom per candidate
    shape (box, cylinder, sphere); per env the chosen candidate is enabled
    (contype/conaffinity 1) and sized, the others are removed from collision,
    and the body takes the chosen shape's mass and inertia. Unused slots are
    parked on the floor far from the table with their box enabled."""

    def __init__(self, xml, nq, params, qpos0):
        self.xml = xml
        self.nq = nq
        self.params = params  # [(param id, element, (envs, width) values)], applied in order
        self.qpos0 = qpos0    # (envs, nq) reset pose

    def apply(self, set_param, reset):
        """set_param(param_id, element, values) for all envs; then the reset
        pose (param 11) and reset(), so that qpos starts at it."""
        for p, elem, vals in self.params:
            set_param(p, elem, vals)
        set_param(11, 0, self.qpos0)
        reset()


def tabletop(num_envs: int, seed: int = 0, slots: int = 6, count=(2, 6), timestep: float = 0.002,
             table=(0.5, 0.4), height: float = 0.4, thickness: float = 0.02) -> TabletopPlan:
    """Config-3 tabletop: a plane, a table (top and four legs) and `slots`
    object slots; per env `count` objects (uniform integer range) drawn from
    {box with half-extents U[0.015, 0.035]^3, cylinder with radius
    U[0.015, 0.03] and half-height U[0.02, 0.05], sphere with radius
    U[0.015, 0.035]}, friction U[0.3, 1.0], density U[500, 1500], dropped
    5-15 cm above the table top at a uniform random orientation."""
    import numpy as np

    rng = np.random.default_rng(seed)
    tx, ty = table
    z_top = height
    legs = (height - 2 * thickness) / 2
    body = [f'<body name="table" pos="0 0 0"><geom name="table_top" type="box" pos="0 0 {_fmt(height - thickness)}" '
            f'size="{_fmt(tx)} {_fmt(ty)} {_fmt(thickness)}"/>']
    for i, (sx, sy) in enumerate([(1, 1), (1, -1), (-1, 1), (-1, -1)]):
        body.append(f'<geom name="table_leg{i}" type="box" pos="{_fmt(sx * (tx - 0.03))} {_fmt(sy * (ty - 0.03))} '
                    f'{_fmt(legs)}" size="0.02 0.02 {_fmt(legs)}"/>')
    body.append('</body>')
    for s in range(slots):
        body.append(f'<body name="slot{s}" pos="{_fmt(100 + 2 * s)} 0 0.05"><freejoint name="slot{s}_joint"/>'
                    f'<geom name="slot{s}_c0" type="box" size="0.035 0.035 0.035"/>'
                    f'<geom name="slot{s}_c1" type="cylinder" size="0.03 0.05"/>'
                    f'<geom name="slot{s}_c2" type="sphere" size="0.035"/></body>')
    xml = (f'<mujoco model="tabletop"><option timestep="{_fmt(timestep)}"/><worldbody>'
           f'<geom name="floor" type="plane" size="5 5 .1"/>{"".join(body)}</worldbody></mujoco>')
    # ids follow the compiler's order: world 0, table 1, slots 2..; geoms floor 0,
    # table 1..5, then 3 per slot; each slot's free joint takes 7 qpos
    ngeom_static = 6
    nq = 7 * slots
    n = num_envs
    shape = lambda k: (n, k)
    contype = np.zeros((slots, 3, n, 1))
    size = np.zeros((slots, 3, n, 3))
    fric = np.zeros((slots, 3, n, 1))
    rgba = np.zeros((slots, 3, n, 4))
    mass = np.zeros((slots, n, 1))
    inertia = np.zeros((slots, n, 3))
    qpos0 = np.zeros((n, nq))
    nominal = [(0.035, 0.035, 0.035), (0.03, 0.05, 0.0), (0.035, 0.0, 0.0)]
    for e in range(n):
        k = int(rng.integers(count[0], count[1] + 1))
        placed = []
        for s in range(slots):
            active = s < k
            c = int(rng.integers(3)) if active else 0
            dens = rng.uniform(500, 1500)
            mu = rng.uniform(0.3, 1.0)
            col = (*rng.uniform(0.2, 0.9, 3), 1.0)
            if c == 0:
                a, b, cc = rng.uniform(0.015, 0.035, 3)
                m = dens * 8 * a * b * cc
                sz, I = (a, b, cc), (m * (b * b + cc * cc) / 3, m * (a * a + cc * cc) / 3, m * (a * a + b * b) / 3)
                rad, rest = math.sqrt(a * a + b * b + cc * cc), cc
            elif c == 1:
                r, h = rng.uniform(0.015, 0.03), rng.uniform(0.02, 0.05)
                m = dens * math.pi * r * r * 2 * h
                ix = m * (3 * r * r + 4 * h * h) / 12
                sz, I = (r, h, 0.0), (ix, ix, m * r * r / 2)
                rad, rest = math.sqrt(r * r + h * h), h
            else:
                r = rng.uniform(0.015, 0.035)
                m = dens * 4 / 3 * math.pi * r ** 3
                sz, I = (r, 0.0, 0.0), (0.4 * m * r * r,) * 3
                rad, rest = r, r
            for ci in range(3):
                on = (ci == c) and active or (not active and ci == 0)
                contype[s, ci, e, 0] = 1.0 if on else 0.0
                size[s, ci, e] = sz if ci == c else nominal[ci]
                fric[s, ci, e, 0] = mu
                rgba[s, ci, e] = col if (ci == c and active) else (0, 0, 0, 0)
            mass[s, e, 0] = m
            inertia[s, e] = I
            q = qpos0[e, 7 * s:7 * s + 7]
            if active:
                for _ in range(100):
                    x, y = rng.uniform(-tx + 0.1, tx - 0.1), rng.uniform(-ty + 0.1, ty - 0.1)
                    if all((x - px) ** 2 + (y - py) ** 2 > (rad + pr) ** 2 for px, py, pr in placed):
                        break
                placed.append((x, y, rad))
                w = rng.normal(size=4)
                w /= np.linalg.norm(w)
                q[:] = (x, y, z_top + rad + rng.uniform(0.05, 0.15), *w)
            else:
                q[:] = (100 + 2 * s + 0.01 * e, 0.0, rest + 1e-3, 1.0, 0.0, 0.0, 0.0)
    params = []
    for s in range(slots):
        for ci in range(3):
            g = ngeom_static + 3 * s + ci
            params += [(3, g, contype[s, ci]), (4, g, contype[s, ci]), (1, g, size[s, ci]), (0, g, fric[s, ci]),
                       (2, g, rgba[s, ci])]
        b = 2 + s
        params += [(5, b, mass[s]), (9, b, inertia[s])]  # mass first: it rescales inertia (params.rs:145-156)
    return TabletopPlan(xml, nq, params, qpos0)


def lumpy_sphere_points(n: int = 600, scale: float = 1.0):
    """The point set of the reference's support-walk test
    (crates/pippin/src/fasthull.rs:221-229): n points on a golden-angle
    spiral over a sphere whose radius has a lump pattern, squashed to 0.7 in
    z. Its hull keeps the points outside the dips: 276 of the 600."""
    import numpy as np

    i = np.arange(n, dtype=np.float64)
    t = i * 2.399963
    p = np.arccos(1.0 - 2.0 * (i + 0.5) / n)
    r = 1.0 + 0.2 * np.sin(3.0 * t) * np.cos(2.0 * p)
    pts = np.stack([r * np.sin(p) * np.cos(t), r * np.sin(p) * np.sin(t), 0.7 * r * np.cos(p)], axis=1)
    return pts * scale


def support_directions(n: int = 2000):
    """The query directions of fasthull.rs:231-233 (unit vectors)."""
    import numpy as np

    a = np.arange(n, dtype=np.float64) * 0.731
    d = np.stack([np.sin(a) * np.cos(1.3 * a), np.cos(0.7 * a), np.sin(2.1 * a)], axis=1)
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def lumpy_hull_xml(scale: float = 0.05) -> str:
    """One free body whose geom is the hull of the 600-point lumpy sphere
    (276 vertices: its support points come from the walk)."""
    pts = " ".join(repr(float(x)) for x in lumpy_sphere_points(600, scale).ravel())
    return ('<mujoco><asset><mesh name="lumpy" vertex="' + pts + '"/></asset><worldbody>'
            '<geom type="plane" size="5 5 .1"/><body name="l" pos="0 0 0.1"><freejoint/>'
            '<geom type="mesh" mesh="lumpy"/></body></worldbody></mujoco>')


def _verts(pts):
    import numpy as np

    return " ".join(repr(float(x)) for x in np.asarray(pts).ravel())


def prism_points(sides=48, r=0.05, h=0.03):
    """The vertices of a regular prism (sides-gon of radius r, half-height h)."""
    import numpy as np

    th = 2.0 * np.pi * np.arange(sides) / sides
    ring = np.stack([r * np.cos(th), r * np.sin(th)], axis=1)
    return np.concatenate([np.column_stack([ring, np.full(sides, -h)]), np.column_stack([ring, np.full(sides, h)])])


def big_hulls_xml():
    """Hulls past the scan limit and faces past a lane's clip buffers: two
    lumpy spheres of 276 hull vertices (the support walk on both sides of a
    pair), a 48-sided prism (96 vertices, 48-gon caps: clipped in shared
    memory), a box, a sphere and a capsule, dropped onto a plane and onto
    each other."""
    lumpy = _verts(lumpy_sphere_points(600, 0.05))
    prism = _verts(prism_points())
    return ('<mujoco><option timestep="0.002"/><asset>'
            f'<mesh name="lumpy" vertex="{lumpy}"/><mesh name="prism" vertex="{prism}"/></asset><worldbody>'
            '<geom type="plane" size="5 5 .1"/>'
            '<body name="l1" pos="0 0 0.06" euler="10 20 30"><freejoint/><geom type="mesh" mesh="lumpy"/></body>'
            '<body name="l2" pos="0.02 0.01 0.16" euler="40 5 70"><freejoint/><geom type="mesh" mesh="lumpy"/></body>'
            '<body name="p" pos="0.3 0 0.04"><freejoint/><geom type="mesh" mesh="prism"/></body>'
            '<body name="b" pos="0.31 0.01 0.1" euler="0 0 20"><freejoint/><geom type="box" size=".03 .03 .02"/></body>'
            '<body name="p2" pos="0.6 0 0.1" euler="90 0 0"><freejoint/><geom type="mesh" mesh="prism"/></body>'
            '<body name="s" pos="0.03 0.01 0.25"><freejoint/><geom type="sphere" size=".02"/></body>'
            '<body name="c" pos="0.6 0.01 0.22" euler="0 80 10"><freejoint/><geom type="capsule" size=".015 .04"/></body>'
            '</worldbody></mujoco>')
