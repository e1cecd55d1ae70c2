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
