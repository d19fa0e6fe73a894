"""p-adaptation and the mixed-order stage path against the reference's CPU
path (Mesh2D_t::adapt, src/meshes/Mesh2D_t.cpp:1644-2268).

After the same steps and error estimate, the reference and the library
adapt the same mesh: element, ghost and face orders must agree exactly, the
interpolated fields bit for bit, and further steps on the mixed-order mesh
bit for bit in FP64_STRICT and within 1e-12 relative L2 in FP64 (the mesh
with an inflow side uses CUDA's exp, so it is held to the tolerance).
"""
from __future__ import annotations

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from tests import meshgen

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _pair(mesh, N, N_max, precision, tol_min=1e-6):
    from oracle.pyoracle import RefSolver
    if isinstance(mesh, str):
        ref = RefSolver(mesh, N, N_max=N_max)
        m = ndg.Mesh2D_t(mesh, N, maximum_N=N_max, tolerance_min=1e-6, tolerance_max=1e-14, precision=precision)
    else:
        ref = RefSolver(mesh, N, N_max=N_max, tolerance_min=tol_min, tolerance_max=1e-14, max_split_level=0)
        m = ndg.Mesh2D_t(mesh, N, maximum_N=N_max, tolerance_min=tol_min, tolerance_max=1e-14, precision=precision)
    # The device initial condition evaluates CUDA's exp (within an ulp of the
    # host's), so both start from the reference's fields.
    ref.initial_conditions()
    for f in ("p", "u", "v"):
        m.set_field(f, ref.field(f))
    return ref, m


def _adapt_both(ref, m, steps):
    ref.run(steps)
    ndg.Solver2D_t.run(m, steps)
    ref.estimate_error()
    m.estimate_error()
    want, got = ref.error(), m.error()
    assert np.array_equal(got["refine"], want["refine"])
    ref.adapt()
    m.adapt()


def _check_topology(ref, m):
    assert (m.n_elements_, m.n_elements_total_, m.n_faces_) == (ref.n_elements, ref.n_elements_total, ref.n_faces)
    em, er = m.elements(), ref.elements()
    assert np.array_equal(em["N"], er["N"])
    assert np.array_equal(m.faces()["N"], ref.faces()["N"])


@pytest.mark.parametrize("precision", [ndg.FP64_STRICT, ndg.FP64])
def test_p_adapt_periodic_walls(precision, ref_available):
    if not ref_available:
        pytest.skip("reference CPU build not present")
    zone = meshgen.uniform_zone(16, x_periodic=True, boundary=meshgen.WALL)
    ref, m = _pair(zone, 4, 8, precision)
    _adapt_both(ref, m, 10)
    _check_topology(ref, m)
    N = m.elements()["N"][:m.n_elements_]
    assert len(set(N.tolist())) == 2  # a mixed-order mesh
    for f in ("p", "u", "v"):
        got, want = m.get_field(f), ref.field(f)
        if precision == ndg.FP64_STRICT:
            assert np.array_equal(got, want), f
        else:
            assert rel_l2(got, want) < TOL, (f, rel_l2(got, want))
    ref.run(6)
    ndg.Solver2D_t.run(m, 6)
    for f in ("p", "u", "v"):
        got, want = m.get_field(f), ref.field(f)
        if precision == ndg.FP64_STRICT:
            assert np.array_equal(got, want), f
        else:
            assert rel_l2(got, want) < TOL, (f, rel_l2(got, want))


def test_p_adapt_twice_and_estimate_on_mixed_orders(ref_available):
    if not ref_available:
        pytest.skip("reference CPU build not present")
    zone = meshgen.uniform_zone(16, y_periodic=True, boundary=meshgen.WALL)
    ref, m = _pair(zone, 4, 10, ndg.FP64_STRICT)
    _adapt_both(ref, m, 8)
    _adapt_both(ref, m, 8)
    _check_topology(ref, m)
    assert len(set(m.elements()["N"][:m.n_elements_].tolist())) >= 2
    ref.estimate_error()
    m.estimate_error()
    want, got = ref.error(), m.error()
    ok = ~np.isnan(want["p_error"])
    np.testing.assert_allclose(got["p_error"][ok], want["p_error"][ok], rtol=1e-13, atol=0)
    ref.run(4)
    ndg.Solver2D_t.run(m, 4)
    for f in ("p", "u", "v"):
        assert np.array_equal(m.get_field(f), ref.field(f)), f


def test_p_adapt_all_boundary_kinds(tmp_path, ref_available):
    """Wall, outflow (farfield), symmetry and inflow sides after p-adaptation:
    re-ordered ghosts project through the mortar path (and carry the zeroed
    scaling factor of Element2D_t::resize_boundary_storage)."""
    if not ref_available:
        pytest.skip("reference CPU build not present")
    zone = meshgen.uniform_zone(16)
    path = str(tmp_path / "mesh.su2")
    meshgen.write_su2(path, zone, meshgen.su2_markers(zone))
    from oracle.pyoracle import RefSolver
    ref = RefSolver(path, 4, N_max=8)
    m = ndg.Mesh2D_t(path, 4, maximum_N=8, precision=ndg.FP64_STRICT)
    ref.initial_conditions()
    for f in ("p", "u", "v"):
        m.set_field(f, ref.field(f))
    _adapt_both(ref, m, 10)
    _check_topology(ref, m)
    assert len(set(m.elements()["N"].tolist())) >= 2
    for f in ("p", "u", "v"):
        assert rel_l2(m.get_field(f), ref.field(f)) < TOL, f
    ref.run(5)
    ndg.Solver2D_t.run(m, 5)
    for f in ("p", "u", "v"):
        assert rel_l2(m.get_field(f), ref.field(f)) < TOL, f


def test_adapt_requires_estimate_then_splits_from_device_estimate():
    zone = meshgen.uniform_zone(16, x_periodic=True, y_periodic=True)
    m = ndg.Mesh2D_t(zone, 4, maximum_N=8, max_split_level=1, tolerance_min=1e-6)
    m.initial_conditions()
    with pytest.raises(ndg.NdgError):
        m.adapt()
    ndg.Solver2D_t.run(m, 10)
    m.estimate_error()
    e = m.error()
    m.adapt()
    splits = int(((e["refine"] == 1) & (e["p_sigma"] < 1)).sum())
    assert m.n_elements_ == 256 + 3 * splits
    assert splits > 0
    ndg.Solver2D_t.run(m, 3)
    assert np.isfinite(m.get_field("p")).all()


@pytest.mark.parametrize("precision", [ndg.FP64_STRICT, ndg.FP64])
@pytest.mark.parametrize("kind", ["x_periodic_walls", "periodic_jittered", "outflow"])
def test_h_adapt_fields_and_steps(kind, precision, ref_available):
    """Element splitting: children interpolated from their parents, then steps
    on the nonconforming mesh (several faces per side, mortar projections),
    against the reference after each of two adaptation rounds. The flags come
    from the reference's estimate so that both adapt the same elements."""
    if not ref_available:
        pytest.skip("reference CPU build not present")
    from oracle.pyoracle import RefSolver
    kw = {"x_periodic_walls": dict(x_periodic=True, boundary=meshgen.WALL),
          "periodic_jittered": dict(x_periodic=True, y_periodic=True, jitter=0.1, seed=2),
          "outflow": dict(boundary=meshgen.OUTFLOW)}[kind]
    zone = meshgen.uniform_zone(8, **kw)
    ref = RefSolver(zone, 4, N_max=8, max_split_level=2, tolerance_min=1e-4, tolerance_max=1e-14)
    m = ndg.Mesh2D_t(zone, 4, maximum_N=8, max_split_level=2, tolerance_min=1e-4, tolerance_max=1e-14, precision=precision)
    ref.initial_conditions()
    for f in ("p", "u", "v"):
        m.set_field(f, ref.field(f))

    def check(stage):
        for f in ("p", "u", "v"):
            got, want = m.get_field(f), ref.field(f)
            if precision == ndg.FP64_STRICT:
                assert np.array_equal(got, want), (stage, f)
            else:
                assert rel_l2(got, want) < TOL, (stage, f, rel_l2(got, want))

    split = False
    for rnd in range(2):
        ref.run(10)
        ndg.Solver2D_t.run(m, 10)
        ref.estimate_error()
        e = ref.error()
        ref.adapt()
        m.adapt(e["refine"], e["p_sigma"])
        _check_topology(ref, m)
        split |= m.n_elements_ > 64
        check(f"after adapt {rnd}")
    assert split
    ref.run(5)
    ndg.Solver2D_t.run(m, 5)
    check("after steps")


def test_solve_with_adaptivity_interval(ref_available):
    """ndg_solve with adaptivity_interval > 0 follows the reference loop
    (include/solvers/Solver2D_t.tcu:35-110): after every interval-th step the
    error is estimated and the mesh adapted, the step size follows the new
    mesh, and the last step is shortened to land on t_end."""
    if not ref_available:
        pytest.skip("reference CPU build not present")
    from oracle.pyoracle import RefSolver
    zone = meshgen.uniform_zone(8, x_periodic=True, boundary=meshgen.WALL)
    kw = dict(tolerance_min=1e-4, tolerance_max=1e-14)
    ref = RefSolver(zone, 4, N_max=8, max_split_level=1, adaptivity_interval=5, **kw)
    m = ndg.Mesh2D_t(zone, 4, maximum_N=8, max_split_level=1, adaptivity_interval=5, precision=ndg.FP64_STRICT, **kw)
    ref.initial_conditions()
    for f in ("p", "u", "v"):
        m.set_field(f, ref.field(f))
    t_end = 12.4 * ref.delta_t()
    t, steps = 0.0, 0
    while t < t_end:
        dt = ref.delta_t()
        if t + dt > t_end:
            dt = t_end - t
            for s in range(3):
                ref.stage(s, t, dt)
            t = t + dt
        else:
            t = ref.run(1, t)
        steps += 1
        if steps % 5 == 0:
            ref.estimate_error()
            ref.adapt()
    t_got, n_got = ndg.Solver2D_t(0.5, [t_end]).solve(m)
    assert n_got == steps and t_got == t
    _check_topology(ref, m)
    assert m.n_elements_ > 64 or len(set(m.elements()["N"].tolist())) > 1
    for f in ("p", "u", "v"):
        assert np.array_equal(m.get_field(f), ref.field(f)), f
