"""The oracle against the reference's behavioural integration tests
(crates/pippin/tests/contact.rs, crates/pippin/tests/mesh.rs,
crates/pippin-env/tests/params.rs), both constraint solvers, plus the
rollout/step-loop and reset-reference checks."""
import numpy as np
import pytest

from pippin_b200 import mjcf, scenes
from tests import scenarios as S


@pytest.mark.parametrize("solver", [S.NEWTON, S.PGS], ids=["newton", "pgs"])
@pytest.mark.parametrize("check", S.CONTACT_CHECKS, ids=lambda f: f.__name__)
def test_contact_behaviour(oracle_lib, check, solver):
    check(S.OracleSim, solver)


@pytest.mark.parametrize("solver", [S.NEWTON, S.PGS], ids=["newton", "pgs"])
@pytest.mark.parametrize("check", S.GENERAL_CHECKS, ids=lambda f: f.__name__)
def test_general_convex_behaviour(oracle_lib, check, solver):
    check(S.OracleSim, solver)


@pytest.mark.parametrize("check", S.PARAM_CHECKS, ids=lambda f: f.__name__)
def test_param_behaviour(oracle_lib, check):
    check(S.OracleSim)


def test_invalid_params_rejected(oracle_lib):
    from oracle.oracle import OracleError
    S.check_invalid_params_rejected(S.OracleSim, OracleError)


@pytest.mark.parametrize("xml", [scenes.cartpole_xml, scenes.tumble_xml])
def test_rollout_matches_step_loop(oracle_lib, xml):
    """contact.rs:161-184: rollout and a per-step set/step loop agree bitwise."""
    from oracle.oracle import CTRL, QPOS, Oracle
    blob = mjcf.compile_string(xml())
    a = Oracle(blob, 3, threads=2)
    b = Oracle(blob, 3, threads=2)
    nu, nq, n, t = a.nu, a.nq, 3, 50
    ctrl = np.sin(np.arange(n * t * max(nu, 1))[: n * t * nu] * 0.37).reshape(n, t, nu)
    out = a.rollout(ctrl)
    for k in range(t):
        if nu:
            b.set(CTRL, ctrl[:, k])
        b.step(0, n, 1)
    np.testing.assert_array_equal(out[:, -1], b.get(QPOS))


def test_reset_state_param_keeps_kinematic_reference(oracle_lib):
    """contact.rs:186-205: qpos0 changes the reset state, not the reference pose."""
    from oracle.oracle import QPOS, Oracle
    xml = ('<mujoco><worldbody><body name="b"><joint name="h" axis="0 0 1" ref="30"/>'
           '<geom type="box" size=".1 .02 .02" pos=".1 0 0" contype="0" conaffinity="0"/></body></worldbody></mujoco>')
    blob = mjcf.compile_string(xml)
    m = Oracle(blob, 1)
    m.set_param(11, 0, [1.0])
    m.reset([0])
    assert m.get(QPOS)[0, 0] == 1.0
    m0 = Oracle(blob, 1)
    m0.set(QPOS, [[1.0]])
    np.testing.assert_allclose(m.body_poses(0)[1, 3:], m0.body_poses(0)[1, 3:], rtol=0, atol=1e-15)
