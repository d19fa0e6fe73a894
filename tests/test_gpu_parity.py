"""GPU parity of the fused FP64 stage kernels against the CPU oracle.

* NDG_FP64_STRICT must reproduce the oracle (and so the reference's CPU
  path) bit for bit, on every order 1..16 and every boundary kind whose
  boundary data does not go through exp().
* NDG_FP64 (FMA contraction, reciprocal multiplies) must stay within
  1e-12 relative L2 of the oracle on p, u, v after every test's steps.
* The committed reference fixtures, batched instances, the shortened last
  step of solve(), single stages, and size-independent properties at the
  full 256 x 256, N = 8 workload (linearity, energy decay) are checked too.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from oracle.pyoracle import OracleSolver
from tests import meshgen

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-12  # relative L2 of the FP64 form against the FP64 oracle


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


def pair(zone: dict, N: int, precision: int, keep_derivative: bool = False):
    m = ndg.Mesh2D_t(zone, N, precision=precision, keep_derivative=keep_derivative)
    o = OracleSolver(zone, N)
    o.initial_conditions()
    for f in ("p", "u", "v"):
        m.set_field(f, o.field(f))
    return m, o


ZONES = {
    "periodic": dict(x_periodic=True, y_periodic=True),
    "wall": dict(boundary=meshgen.WALL),
    "symmetry": dict(boundary=meshgen.SYMMETRY),
    "outflow": dict(boundary=meshgen.OUTFLOW),
    "null": dict(boundary=meshgen.NULL),
    "x_periodic_wall": dict(x_periodic=True, boundary=meshgen.WALL),
    "jitter_rowmajor": dict(order="rowmajor", jitter=0.1, x_periodic=True, y_periodic=True),
}


@pytest.mark.parametrize("kind", list(ZONES))
@pytest.mark.parametrize("N", [2, 4, 8])
def test_strict_bitwise_and_fast_tolerance(kind, N):
    kw = ZONES[kind]
    res = 6 if kw.get("order") == "rowmajor" else 8
    zone = meshgen.uniform_zone(res, **kw)
    steps = 12
    o = OracleSolver(zone, N)
    o.initial_conditions()
    o.run(steps)
    for precision in (ndg.FP64_STRICT, ndg.FP64):
        m, _ = pair(zone, N, precision, keep_derivative=True)
        assert ndg.Solver2D_t.get_delta_t(m) == o.delta_t()
        t = ndg.Solver2D_t.run(m, steps)
        assert abs(t - steps * o.delta_t()) < 1e-14
        for f, g in (("p", "p"), ("u", "u"), ("v", "v"), ("k_p", "kp"), ("k_u", "ku"), ("k_v", "kv"), ("G_p", "Gp"), ("G_v", "Gv")):
            got, want = m.get_field(f), o.field(g)
            if precision == ndg.FP64_STRICT:
                assert np.array_equal(got, want), (f, np.max(np.abs(got - want)))
            else:
                assert rel_l2(got, want) < TOL, (f, rel_l2(got, want))


@pytest.mark.parametrize("N", list(range(1, 17)))
def test_every_order(N):
    zone = meshgen.uniform_zone(4, x_periodic=True, boundary=meshgen.WALL)
    o = OracleSolver(zone, N)
    o.initial_conditions()
    o.run(3)
    for precision in (ndg.FP64_STRICT, ndg.FP64):
        m, _ = pair(zone, N, precision)
        ndg.Solver2D_t.run(m, 3)
        for f in ("p", "u", "v"):
            got, want = m.get_field(f), o.field(f)
            if precision == ndg.FP64_STRICT and N != 15:
                assert np.array_equal(got, want), (N, f)
            else:
                # N = 15: one wall-ghost node misses the reference's 2-ulp node
                # match and is interpolated there (1e-16 level), copied here.
                assert rel_l2(got, want) < TOL, (N, f, rel_l2(got, want))


def test_inflow_boundary_tolerance():
    # Inflow ghosts evaluate exp() on the device; CUDA's exp and glibc's may
    # differ in the last bit, so only the tolerance applies.
    zone = meshgen.uniform_zone(4, boundary=meshgen.INFLOW)
    o = OracleSolver(zone, 5)
    o.initial_conditions()
    o.run(10, 0.25)
    for precision in (ndg.FP64_STRICT, ndg.FP64):
        m, _ = pair(zone, 5, precision)
        ndg.Solver2D_t.run(m, 10, 0.25)
        for f in ("p", "u", "v"):
            assert rel_l2(m.get_field(f), o.field(f)) < TOL


def test_device_initial_condition_matches_reference_plane_wave():
    zone = meshgen.uniform_zone(16, x_periodic=True, y_periodic=True, jitter=0.05, order="rowmajor")
    m = ndg.Mesh2D_t(zone, 6)
    m.initial_conditions()
    o = OracleSolver(zone, 6)
    o.initial_conditions()
    for f in ("p", "u", "v"):
        assert rel_l2(m.get_field(f), o.field(f)) < 1e-15
        np.testing.assert_allclose(m.get_field(f), o.field(f), rtol=0, atol=1e-15)


@pytest.mark.parametrize("name", ["ref_periodic_r16_n4_s200", "ref_periodic_r8_n8_s20", "ref_wall_r8_n6_s30", "ref_outflow_r4_n5_s10"])
def test_committed_reference_fixtures(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    zone = meshgen.uniform_zone(int(g["res"]), boundary=int(g["boundary"]), x_periodic=bool(g["periodic"]), y_periodic=bool(g["periodic"]))
    m = ndg.Mesh2D_t(zone, int(g["N"]))
    m.initial_conditions()
    assert ndg.Solver2D_t.get_delta_t(m) == float(g["dt"])
    t = ndg.Solver2D_t.run(m, int(g["steps"]))
    assert t == float(g["time"])
    for f in ("p", "u", "v"):
        assert rel_l2(m.get_field(f), g[f]) < TOL, (f, rel_l2(m.get_field(f), g[f]))


def test_single_stages_match_oracle():
    zone = meshgen.uniform_zone(8, x_periodic=True, boundary=meshgen.WALL)
    m, o = pair(zone, 6, ndg.FP64_STRICT, keep_derivative=True)
    dt = o.delta_t()
    for m_ in range(3):
        o.stage(m_, 0.1, dt)
        ndg.Solver2D_t.stage(m, m_, 0.1, dt)
        for f, g in (("p", "p"), ("k_u", "ku"), ("G_v", "Gv")):
            assert np.array_equal(m.get_field(f), o.field(g)), (m_, f)


def test_solve_shortens_last_step():
    zone = meshgen.uniform_zone(8, x_periodic=True, y_periodic=True)
    m, o = pair(zone, 4, ndg.FP64_STRICT)
    t_end = 0.1  # dt = 1/128 does not divide 0.1
    t, n = ndg.Solver2D_t(0.5, [t_end]).solve(m)
    dt = o.delta_t()
    time, steps = 0.0, 0
    while time < t_end:
        step = dt if time + dt <= t_end else t_end - time
        for s in range(3):
            o.stage(s, time, step)
        time += step
        steps += 1
    assert (t, n) == (time, steps)
    for f in ("p", "u", "v"):
        assert np.array_equal(m.get_field(f), o.field(f)), f


def test_batched_instances_equal_independent_runs():
    zone = meshgen.uniform_zone(8, x_periodic=True, y_periodic=True)
    N, steps = 5, 15
    o = OracleSolver(zone, N)
    o.initial_conditions()
    base = {f: o.field(f) for f in ("p", "u", "v")}
    rng = np.random.default_rng(0)
    inits = [base, {f: 0.5 * base[f] for f in base}, {f: rng.standard_normal(base[f].size) for f in base}]
    m = ndg.Mesh2D_t(zone, N, n_instances=len(inits), precision=ndg.FP64_STRICT)
    for f in ("p", "u", "v"):
        m.set_field(f, np.concatenate([ini[f] for ini in inits]))
    ndg.Solver2D_t.run(m, steps)
    for i, ini in enumerate(inits):
        oi = OracleSolver(zone, N)
        for f in ("p", "u", "v"):
            oi.set_field(f, ini[f])
        oi.run(steps)
        for f in ("p", "u", "v"):
            assert np.array_equal(m.get_field(f, instance=i), oi.field(f)), (i, f)


def test_full_size_workload_against_oracle_and_properties():
    """256 x 256, N = 8, periodic: a few steps against the oracle, then
    linearity (the scheme is linear: doubling the state doubles the result
    exactly) and the energy decay of the upwind flux, over more steps."""
    zone = meshgen.uniform_zone(256, x_periodic=True, y_periodic=True)
    N = 8
    m = ndg.Mesh2D_t(zone, N)
    m.initial_conditions()
    o = OracleSolver(zone, N)
    o.initial_conditions()
    o.run(2)
    ndg.Solver2D_t.run(m, 2)
    for f in ("p", "u", "v"):
        assert rel_l2(m.get_field(f), o.field(f)) < TOL
    q = {f: m.get_field(f) for f in ("p", "u", "v")}
    # Energy with quadrature weights (uniform affine mesh: constant Jacobian).
    w = ndg.tables_compute(N, 2, "weights", N)
    W = np.outer(w, w).ravel()
    K = m.n_elements_

    def energy(fields):
        return sum(float(np.sum(fields[f].reshape(K, -1) ** 2 * W)) for f in fields)

    e0 = energy(q)
    ndg.Solver2D_t.run(m, 20)
    q1 = {f: m.get_field(f) for f in ("p", "u", "v")}
    assert energy(q1) <= e0 * (1 + 1e-14)
    m2 = ndg.Mesh2D_t(zone, N)
    for f in ("p", "u", "v"):
        m2.set_field(f, 2.0 * q[f])
    ndg.Solver2D_t.run(m2, 20)
    for f in ("p", "u", "v"):
        assert rel_l2(m2.get_field(f), 2.0 * q1[f]) < 1e-15
