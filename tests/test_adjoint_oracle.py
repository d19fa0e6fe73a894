"""The CPU discrete adjoint of the oracle (oracle/ndg_oracle.c), the
reference gradient of the library's adjoint, checked on its own: with c = 1
its variable-speed forward is the reference's stage bit for bit, its
transposed operator passes the dot-product test, its speed derivative
matches finite differences, and the gradient of the misfit matches central
differences in the initial pressure and the wave speed.
"""
from __future__ import annotations

import numpy as np
import pytest

from tests import adjoint_setup as A
from tests import meshgen

MESHES = {
    "periodic": dict(x_periodic=True, y_periodic=True),
    "walls": dict(boundary=meshgen.WALL),
    "jittered_outflow": dict(boundary=meshgen.OUTFLOW, jitter=0.1, seed=3),
    "symmetry_x_periodic": dict(x_periodic=True, boundary=meshgen.SYMMETRY),
}


def _rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("kind", list(MESHES))
def test_unit_speed_is_the_reference_stage(kind):
    from oracle.pyoracle import OracleSolver
    zone = meshgen.uniform_zone(8, **MESHES[kind])
    a, b = OracleSolver(zone, 4), OracleSolver(zone, 4)
    a.set_speed(np.ones(a.n_elements))
    for o in (a, b):
        o.set_field("p", A.gaussian_pulse(zone, 4, sigma=0.3))
    dt = b.delta_t()
    for o in (a, b):
        for m in range(3):
            o.stage(m, 0.0, dt)
    for f in ("p", "u", "v"):
        assert np.array_equal(a.field(f), b.field(f)), f


@pytest.mark.parametrize("kind", list(MESHES))
def test_operator_transpose(kind):
    zone = meshgen.uniform_zone(8, **MESHES[kind])
    o, _, _ = A.oracle_problem(zone, 4, A.speed_field(zone, seed=1), np.zeros((0, 2)))
    rng = np.random.default_rng(7)
    n = 3 * o._field_size()
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    Lx = o.operator(x)
    LTy, _ = o.operator_transpose(x, y)
    lhs, rhs = float(Lx @ y), float(x @ LTy)
    assert _rel(lhs, rhs) < 1e-12 * np.linalg.norm(Lx) * np.linalg.norm(y) / abs(lhs)


@pytest.mark.parametrize("kind", ["periodic", "walls", "jittered_outflow"])
def test_operator_speed_derivative(kind):
    zone = meshgen.uniform_zone(8, **MESHES[kind])
    c = A.speed_field(zone, seed=2)
    o, _, _ = A.oracle_problem(zone, 3, c, np.zeros((0, 2)))
    rng = np.random.default_rng(3)
    n = 3 * o._field_size()
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    _, dc = o.operator_transpose(x, y)
    d = rng.standard_normal(c.size)
    eps = 1e-3  # y . L(c) x is linear in c: the central difference is exact up to rounding
    o.set_speed(c + eps * d)
    fp = float(y @ o.operator(x))
    o.set_speed(c - eps * d)
    fm = float(y @ o.operator(x))
    assert _rel((fp - fm) / (2 * eps), float(dc @ d)) < 1e-9


def _problem(kind="walls", res=8, N=3, n_rec=8):
    zone = meshgen.uniform_zone(res, **MESHES[kind])
    c = A.speed_field(zone, seed=4)
    xy = A.circle_receivers(n_rec, 0.6)
    o, el, w = A.oracle_problem(zone, N, c, xy)
    p0 = A.gaussian_pulse(zone, N, sigma=0.25)
    return zone, c, o, el, w, p0


def test_full_map_dot_product():
    """F: p0 -> receiver samples is linear (u0 = v0 = 0); the adjoint with
    p0 = 0 and targets -r/dt returns F^T r."""
    zone, c, o, el, w, p0 = _problem()
    dt, n = A.cfl_dt(zone, 3, c), 15
    rng = np.random.default_rng(5)
    x = rng.standard_normal(p0.size)
    Fx = o.adjoint_solve(x, dt, n, el, w)["samples"][1:]
    r = rng.standard_normal((n + 1, el.size))
    r[0] = 0.0
    g = o.adjoint_solve(np.zeros_like(x), dt, n, el, w, targets=-r / dt)
    lhs, rhs = float((Fx * r[1:]).sum()), float(x @ g["p0"])
    assert _rel(lhs, rhs) < 1e-12


def test_gradient_matches_central_differences():
    zone, c, o, el, w, p0 = _problem("periodic")
    dt, n = A.cfl_dt(zone, 3, c), 20
    # targets from a run with a perturbed speed
    o.set_speed(c * (1 + 0.05 * np.sin(3 * A.element_centres(zone)[:, 0])))
    target = o.adjoint_solve(p0, dt, n, el, w)["samples"]
    o.set_speed(c)
    g = o.adjoint_solve(p0, dt, n, el, w, targets=target)
    assert g["J"] > 0
    rng = np.random.default_rng(9)
    dp = rng.standard_normal(p0.size)
    eps = 1e-4  # J is quadratic in p0
    Jp = o.adjoint_solve(p0 + eps * dp, dt, n, el, w, targets=target)["J"]
    Jm = o.adjoint_solve(p0 - eps * dp, dt, n, el, w, targets=target)["J"]
    assert _rel((Jp - Jm) / (2 * eps), float(g["p0"] @ dp)) < 1e-8
    dcv = rng.standard_normal(c.size)
    eps = 1e-6
    o.set_speed(c + eps * dcv)
    Jp = o.adjoint_solve(p0, dt, n, el, w, targets=target)["J"]
    o.set_speed(c - eps * dcv)
    Jm = o.adjoint_solve(p0, dt, n, el, w, targets=target)["J"]
    assert _rel((Jp - Jm) / (2 * eps), float(g["c"] @ dcv)) < 1e-6
