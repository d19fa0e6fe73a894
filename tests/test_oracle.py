"""Pins the CPU oracle (oracle/ndg_oracle.c) before anything is checked against it.

1. Golden vectors of the reference's own tests: Legendre-Gauss N = 16 nodes
   and weights (tests/polynomials_test.cu:187-226) and its derivative and
   boundary-extrapolation checks (:232-277).
2. Bit-for-bit agreement with the reference's own CPU path compiled from its
   sources (oracle/_ref/libndgref.so): all twelve NDG tables, the mesh
   topology, and multi-step solutions on periodic, wall, symmetry and
   outflow meshes.
3. The committed reference fixtures (tests/golden/ref_*.npz).
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from oracle import pyoracle
from oracle.pyoracle import OracleSolver, oracle_table
from tests import meshgen

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_legendre_n16_golden_vectors():
    gold = json.load(open(os.path.join(GOLDEN, "legendre_n16.json")))
    nodes = oracle_table(16, 128, 0, 16)
    weights = oracle_table(16, 128, 1, 16)
    # The reference requires 1e-6; the 22-digit literals allow a 2-ulp check.
    np.testing.assert_allclose(nodes, gold["nodes"], rtol=0, atol=4e-16)
    np.testing.assert_allclose(weights, gold["weights"], rtol=0, atol=4e-16)


def test_derivative_and_extrapolation_known_answers():
    # tests/polynomials_test.cu:232-277: D sin(pi x) ~ pi cos(pi x), and the
    # +-1 interpolants/derivative interpolants on sin(pi x), N = 16.
    N = 16
    x = oracle_table(16, 128, 0, N)
    D = oracle_table(16, 128, 7, N).reshape(N + 1, N + 1)
    phi = np.sin(np.pi * x)
    assert np.max(np.abs(D @ phi - np.pi * np.cos(np.pi * x))) < 1e-4
    lL, lR = oracle_table(16, 128, 3, N), oracle_table(16, 128, 4, N)
    phi_L, phi_R = lL @ phi, lR @ phi
    assert abs(phi_L - np.sin(-np.pi)) < 1e-6 and abs(phi_R - np.sin(np.pi)) < 1e-6
    dL, dR = oracle_table(16, 128, 5, N), oracle_table(16, 128, 6, N)
    assert abs(dL @ (phi_L - phi) - np.pi * np.cos(-np.pi)) < 1e-6
    assert abs(dR @ (phi_R - phi) - np.pi * np.cos(np.pi)) < 1e-6


def test_tables_bitwise_vs_reference(ref_available):
    for N in range(0, 17):
        for t in range(12):
            a = pyoracle.ref_table(16, 9, t, N)
            b = oracle_table(16, 9, t, N)
            assert np.array_equal(a, b), (t, N)


ZONES = [
    ("periodic", dict(x_periodic=True, y_periodic=True)),
    ("wall", dict(boundary=meshgen.WALL)),
    ("symmetry", dict(boundary=meshgen.SYMMETRY)),
    ("outflow", dict(boundary=meshgen.OUTFLOW)),
    ("inflow", dict(boundary=meshgen.INFLOW)),
    ("x_periodic_walls", dict(x_periodic=True, boundary=meshgen.WALL)),
    ("rowmajor_jitter", dict(order="rowmajor", jitter=0.1, x_periodic=True, y_periodic=True)),
]


@pytest.mark.parametrize("name,kw", ZONES, ids=[z[0] for z in ZONES])
def test_topology_bitwise_vs_reference(ref_available, name, kw):
    res = 6 if kw.get("order") == "rowmajor" else 8
    zone = meshgen.uniform_zone(res, **kw)
    r = pyoracle.RefSolver(zone, 3)
    o = OracleSolver(zone, 3)
    assert (r.n_elements, r.n_elements_total, r.n_faces, r.n_nodes) == (o.n_elements, o.n_elements_total, o.n_faces, o.n_nodes)
    fr, fo = r.faces(), o.faces()
    for k in fo:
        assert np.array_equal(fr[k], fo[k]), k
    er, eo = r.elements(), o.elements()
    for k in eo:
        assert np.array_equal(er[k], eo[k]), k
    for kind in range(7):
        assert np.array_equal(r.boundary(kind), o.boundary(kind)), kind


@pytest.mark.parametrize("name,kw", ZONES, ids=[z[0] for z in ZONES])
@pytest.mark.parametrize("N", [1, 4, 7])
def test_steps_bitwise_vs_reference(ref_available, name, kw, N):
    res = 6 if kw.get("order") == "rowmajor" else 4
    zone = meshgen.uniform_zone(res, **kw)
    r = pyoracle.RefSolver(zone, N)
    o = OracleSolver(zone, N)
    r.initial_conditions()
    o.initial_conditions()
    assert r.delta_t() == o.delta_t()
    tr = r.run(7, 0.05)
    to = o.run(7, 0.05)
    assert tr == to
    for f in ("p", "u", "v", "Gp", "Gu", "Gv", "kp", "ku", "kv"):
        assert np.array_equal(r.field(f), o.field(f)), f


def test_error_estimator_bitwise_vs_reference(ref_available):
    zone = meshgen.uniform_zone(8, x_periodic=True, y_periodic=True)
    r = pyoracle.RefSolver(zone, 6, tolerance_min=1e-4, tolerance_max=1e-8)
    o = OracleSolver(zone, 6, tolerance_min=1e-4, tolerance_max=1e-8)
    r.initial_conditions()
    o.initial_conditions()
    r.run(3)
    o.run(3)
    r.estimate_error()
    o.estimate_error()
    er, eo = r.error(), o.error()
    for k in er:
        assert np.array_equal(er[k], eo[k]), k


@pytest.mark.parametrize("name", ["ref_periodic_r16_n4_s200", "ref_periodic_r8_n8_s20", "ref_wall_r8_n6_s30", "ref_outflow_r4_n5_s10"])
def test_oracle_matches_committed_reference_fixtures(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    zone = meshgen.uniform_zone(int(g["res"]), boundary=int(g["boundary"]), x_periodic=bool(g["periodic"]), y_periodic=bool(g["periodic"]))
    o = OracleSolver(zone, int(g["N"]))
    o.initial_conditions()
    assert o.delta_t() == float(g["dt"])
    t = o.run(int(g["steps"]))
    assert t == float(g["time"])
    for f in ("p", "u", "v"):
        assert np.array_equal(o.field(f), g[f]), f
