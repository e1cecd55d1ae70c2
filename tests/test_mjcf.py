"""Model compiler: the generated workload models equal the reference's
assets, the blob round-trips through the oracle's reader, and the compile
step reproduces the reference's structural facts for Ant."""
import hashlib
import json
import os
from collections import Counter

import pytest

from pippin_b200 import mjcf, scenes
from tests.conftest import REFERENCE, have_reference


@pytest.mark.skipif(not have_reference(), reason="reference repository not present")
@pytest.mark.parametrize("asset", sorted(scenes.REFERENCE_ASSETS))
def test_generated_models_match_reference_assets(asset):
    ref = mjcf.compile_file(os.path.join(REFERENCE, "assets", asset))
    assert mjcf.compile_string(scenes.REFERENCE_ASSETS[asset]()) == ref


@pytest.mark.parametrize("asset", sorted(scenes.REFERENCE_ASSETS))
def test_generated_models_match_recorded_asset_blobs(asset):
    """The same check without a reference checkout: the blob's SHA-256 equals
    the one recorded from the reference's asset (tests/golden/make_blob_hashes.py)."""
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_blobs.json")) as fh:
        want = json.load(fh)[asset]
    blob = mjcf.compile_string(scenes.REFERENCE_ASSETS[asset]())
    assert len(blob) == want["bytes"]
    assert hashlib.sha256(blob).hexdigest() == want["sha256"]


def test_ant_structure():
    m = mjcf.load_string(scenes.ant_xml())
    assert (m.nq, m.nv, m.nu, m.nbody, m.njnt, m.ngeom) == (15, 14, 8, 14, 9, 14)
    pairs = mjcf.collision_pairs(m)
    assert len(pairs) == 57
    kinds = Counter((m.geom_type[a], m.geom_type[b]) for a, b in pairs)
    assert kinds == {(2, 2): 40, (0, 2): 12, (1, 2): 4, (0, 1): 1}
    assert m.dof_blocks == [(0, 14)]
    assert m.dof_damping[:6] == [0.0] * 6 and m.dof_damping[6:] == [1.0] * 8
    assert all(m.jnt_limited[1:]) and not m.jnt_limited[0]


def test_blob_loads_in_oracle(oracle_lib):
    from oracle.oracle import Oracle, OracleError
    for fn in scenes.REFERENCE_ASSETS.values():
        o = Oracle(mjcf.compile_string(fn()), 2)
        assert o.n == 2
    with pytest.raises(OracleError):
        Oracle(b"PGBLOB01" + b"\0" * 8, 1)


def test_free_bodies_get_separate_blocks():
    m = mjcf.load_string(scenes.box_drop_xml())
    assert m.dof_blocks == [(0, 6), (6, 12), (12, 18)]


def test_invalid_models_are_rejected():
    with pytest.raises(mjcf.MjcfError):
        mjcf.load_string("<robot/>")
    with pytest.raises(mjcf.MjcfError):
        mjcf.load_string('<mujoco><worldbody><joint type="hinge"/></worldbody></mujoco>')
    with pytest.raises(mjcf.MjcfError):
        mjcf.load_string('<mujoco><worldbody><body><joint type="hinge"/></body></worldbody></mujoco>')
