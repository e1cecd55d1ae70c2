"""The oracle against the reference's known-answer unit tests.

Values come from tests/golden/reference_kats.json (extracted from the
reference's test sources by tests/golden/make_kats.py; each entry names its
file:line).
"""
import json
import math
import os

import numpy as np
import pytest

from pippin_b200 import mjcf

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


def test_impedance_curve(oracle_lib):
    k = KATS["impedance"]
    for c in k["cases"]:
        assert abs(oracle_lib.impedance(k["solimp"], c["pos"]) - c["expected"]) < c["tol"]


def test_dot_matches_sequential_sum(oracle_lib):
    k = KATS["dot"]
    for n in range(k["n_max"]):
        a = np.array([math.sin(i * k["a_sin_step"]) for i in range(n)])
        b = np.array([math.cos(i * k["b_cos_step"]) for i in range(n)])
        s = 0.0
        for x, y in zip(a, b):
            s += x * y
        assert abs(oracle_lib.vdot(a, b) - s) < k["tol"], n


def test_block_cholesky_matches_dense(oracle_lib):
    k = KATS["block_cholesky"]
    n = k["n"]
    a = np.zeros((n, n))
    for s0, s1 in k["blocks"]:
        for i in range(s0, s1):
            for j in range(s0, s1):
                a[i, j] = k["diag_base"] + i if i == j else k["off_base"] + k["off_step"] * (i + j)
    rhs = np.array([1.0 + i for i in range(n)])
    dense, x1 = a.copy(), rhs.copy()
    assert oracle_lib.cholesky_block(dense, n, 0, n)
    oracle_lib.cholesky_solve_block(dense, n, 0, n, x1)
    blk, x2 = a.copy(), rhs.copy()
    for s0, s1 in k["blocks"]:
        assert oracle_lib.cholesky_block(blk, n, s0, s1)
        oracle_lib.cholesky_solve_block(blk, n, s0, s1, x2)
    assert np.max(np.abs(x1 - x2)) < k["tol"]


def test_cholesky_solves(oracle_lib):
    k = KATS["cholesky_solve"]
    a = np.array(k["a"], dtype=np.float64)
    orig = a.reshape(3, 3).copy()
    assert oracle_lib.cholesky_block(a, 3, 0, 3)
    x = np.array(k["b"], dtype=np.float64)
    oracle_lib.cholesky_solve_block(a, 3, 0, 3, x)
    assert np.max(np.abs(orig @ x - np.array(k["b"]))) < k["tol"]


def test_quat_mat_roundtrip(oracle_lib):
    k = KATS["quat_roundtrip"]
    q = oracle_lib.quat_from_axis_angle(k["axis"], k["angle"])
    q2 = mjcf.q_from_mat(tuple(oracle_lib.quat_to_mat(q)))
    assert np.max(np.abs(np.array(q) - np.array(q2))) < k["tol"]
    # the compiler's restatement agrees with the oracle's
    assert np.allclose(mjcf.q_axis_angle(tuple(k["axis"]), k["angle"]), q, rtol=0, atol=0)


def test_cube_mass_properties_are_exact():
    k = KATS["cube_mass"]
    h = k["half"]
    off = k["offset"]
    pts = [((-h if i & 1 == 0 else h) + off[0], (-h if i & 2 == 0 else h) + off[1], (-h if i & 4 == 0 else h) + off[2])
           for i in range(8)]
    verts, tris = mjcf.convex_hull(pts)
    vol, com, icom = mjcf.mesh_mass_properties(verts, tris)
    side = 2 * h
    assert abs(vol - side ** 3) < k["tol"]
    assert np.linalg.norm(np.array(com) - np.array(off)) < k["tol"]
    expected = vol * side * side / 6.0
    for i in range(3):
        assert abs(icom[4 * i] - expected) < k["tol"]
    assert abs(icom[1]) < k["tol"] and abs(icom[2]) < k["tol"] and abs(icom[5]) < k["tol"]


def test_hull_support_walk_matches_brute_force():
    """fasthull.rs:217-240 restated: on the hull of 600 points of a lumpy
    sphere, the support walk's vertex projects as far as a scan over every
    hull vertex along each of 2000 directions (1e-12)."""
    from oracle.oracle import hull_support

    from . import scenarios as S

    verts, tris = mjcf.convex_hull([tuple(p) for p in S.lumpy_sphere_points()])
    _, edges = mjcf.hull_features(verts, tris)
    v = np.asarray(verts)
    assert len(v) >= 64  # the walk, not the scan
    d = S.support_directions()
    walked = hull_support(v, edges, d)
    exact = (v @ d.T).max(axis=0)
    got = np.einsum("ij,ij->i", v[walked], d)
    assert np.abs(exact - got).max() < 1e-12
