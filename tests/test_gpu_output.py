"""Solution output, output files and pre-conditioning on the GPU against the
reference's own CPU code (oracle/_ref):

* ndg_get_solution against Mesh2D_t::get_complete_solution
  (src/meshes/Mesh2D_t.cpp:4251-4296): coordinates, fields and time
  derivatives bit for bit after the same strict FP64 steps, on uniform and
  on adapted (mixed-order) meshes; the analytic error to 1e-13 of its
  largest value (CUDA's exp against the host's in the plane wave);
* Mesh2D_t.write_complete_data through the writer: the files hold what
  get_solution returns, and the element arrays the mesh state;
* Solver2D_t.solve with a DataWriter_t: outputs at the reference's times;
* Solver2D_t::pre_condition and pre_condition_iterative
  (include/solvers/Solver2D_t.tpp:136-334): the same adapted topology as the
  reference, and its initial conditions on it.
"""
from __future__ import annotations

import json

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from oracle import pyoracle
from tests import meshgen
from tests.vtu import read_grid

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not pyoracle.ref_available(), reason="reference checker not built (oracle/_ref/libndgref.so)")]
EXACT = ("x", "y", "p", "u", "v", "dp_dt", "du_dt", "dv_dt")
ANALYTIC = ("p_analytical_error", "u_analytical_error", "v_analytical_error")


def _pair(zone, N, n_interp, N_max=None, tol_min=1e-6, max_split_level=0):
    from oracle.pyoracle import RefSolver
    ref = RefSolver(zone, N, N_max=N_max, n_interp=n_interp, tolerance_min=tol_min, tolerance_max=1e-14,
                    max_split_level=max_split_level)
    m = ndg.Mesh2D_t(zone, N, maximum_N=N_max, n_interpolation_points=n_interp, tolerance_min=tol_min,
                     tolerance_max=1e-14, max_split_level=max_split_level, precision=ndg.FP64_STRICT, keep_derivative=True)
    ref.initial_conditions()
    for f in ("p", "u", "v"):
        m.set_field(f, ref.field(f))
    return ref, m


def _compare(ref, m, time, copy_state=False):
    if copy_state:
        # the reference's state itself (steps with an inflow side evaluate
        # CUDA's exp at the boundary, so the stepped fields differ in the last
        # bits): the output interpolation alone must then agree bit for bit
        for ours, theirs in (("p", "p"), ("u", "u"), ("v", "v"), ("G_p", "Gp"), ("G_u", "Gu"), ("G_v", "Gv")):
            m.set_field(ours, ref.field(theirs))
    want = ref.complete_solution(time)
    got = m.get_complete_solution(time)
    for k in EXACT:
        assert np.array_equal(got[k], want[k]), k
    for k in ANALYTIC:
        # the interpolation weights have both signs, so a point's sum can
        # cancel: the bound is relative to the array's largest value
        np.testing.assert_allclose(got[k], want[k], rtol=1e-13, atol=1e-13 * np.abs(want[k]).max(), err_msg=k)
    return got


@pytest.mark.parametrize("N", [1, 4, 8, 12])
@pytest.mark.parametrize("kind", ["periodic_jittered", "walls", "all_kinds"])
@pytest.mark.parametrize("n_interp", [2, 6])
def test_output_matches_reference(N, kind, n_interp, tmp_path):
    if kind == "all_kinds":
        zone = str(tmp_path / "mesh.su2")
        z = meshgen.uniform_zone(8)
        meshgen.write_su2(zone, z, meshgen.su2_markers(z))
    else:
        kw = {"periodic_jittered": dict(x_periodic=True, y_periodic=True, jitter=0.1, seed=5),
              "walls": dict(boundary=meshgen.WALL)}[kind]
        zone = meshgen.uniform_zone(8, **kw)
    ref, m = _pair(zone, N, n_interp)
    ref.run(7)
    ndg.Solver2D_t.run(m, 7)
    _compare(ref, m, 0.21, copy_state=(kind == "all_kinds"))
    m.close()


def test_output_on_an_adapted_mesh():
    zone = meshgen.uniform_zone(16, y_periodic=True, boundary=meshgen.WALL)
    ref, m = _pair(zone, 4, 5, N_max=10)
    for _ in range(2):
        ref.run(8)
        ndg.Solver2D_t.run(m, 8)
        ref.estimate_error()
        m.estimate_error()
        ref.adapt()
        m.adapt()
    orders = m.elements()["N"][:m.n_elements_]
    assert len(set(orders.tolist())) > 1, "the test needs a mixed-order mesh"
    ref.run(3)
    ndg.Solver2D_t.run(m, 3)
    _compare(ref, m, 0.5)
    m.close()


def test_writer_end_to_end(tmp_path):
    zone = meshgen.uniform_zone(8, x_periodic=True, boundary=meshgen.WALL)
    m = ndg.Mesh2D_t(zone, 5, maximum_N=7, n_interpolation_points=4, keep_derivative=True, tolerance_min=1e-7)
    m.initial_conditions()
    ndg.Solver2D_t.run(m, 12)
    m.estimate_error()
    w = ndg.DataWriter_t(str(tmp_path / "wave.pvtu"))
    m.write_complete_data(0.125, w)
    sol = m.get_complete_solution(0.125)
    g = read_grid(str(tmp_path / "wave_t0_125000000s.pvtu"))
    assert np.array_equal(g["points"][:, 0], sol["x"]) and np.array_equal(g["points"][:, 1], sol["y"])
    pd = g["point_data"]
    assert np.array_equal(pd["Pressure"], sol["p"])
    assert np.array_equal(pd["Velocity"], np.stack([sol["u"], sol["v"]], axis=1))
    assert np.array_equal(pd["PressureDerivative"], sol["dp_dt"])
    assert np.array_equal(pd["PressureAnalyticalError"], sol["p_analytical_error"])
    eg = read_grid(str(tmp_path / "wave_element_t0_125000000s.pvtu"))
    cd = eg["cell_data"]
    err = m.error()
    assert np.array_equal(cd["N"], m.elements()["N"][:m.n_elements_])
    assert np.array_equal(cd["PressureError"], err["p_error"]) and np.array_equal(cd["Refine"], err["refine"])
    state = m.element_state()
    assert np.array_equal(cd["Status"], state["status"][:m.n_elements_])
    assert np.array_equal(cd["SplitLevel"], state["split_level"][:m.n_elements_])
    series = json.loads((tmp_path / "wave.pvtu.series").read_text())
    assert series["files"] == [{"name": "wave_t0_125000000s.pvtu", "time": 0.125}]
    w.close()
    m.close()


def test_solve_writes_at_the_reference_output_times(tmp_path):
    zone = meshgen.uniform_zone(8, x_periodic=True, y_periodic=True)
    m = ndg.Mesh2D_t(zone, 3, n_interpolation_points=3)
    m.initial_conditions()
    solver = ndg.Solver2D_t(0.5, [0.0, 0.1, 0.25])
    w = ndg.DataWriter_t(str(tmp_path / "out.pvtu"))
    t, steps = solver.solve(m, data_writer=w)
    # the reference's schedule: step by dt, write after the first step whose
    # end time t has e <= t < e + dt, the last step shortened to land on t_end
    dt = ndg.Solver2D_t.get_delta_t(m)
    times, tt, n = [0.0], 0.0, 0
    while tt < 0.25:
        d = min(dt, 0.25 - tt)
        tt += d
        n += 1
        if any(e <= tt < e + d for e in (0.0, 0.1, 0.25)):
            times.append(tt)
    assert steps == n and t == tt
    got = [f["time"] for f in json.loads((tmp_path / "out.pvtu.series").read_text())["files"]]
    assert got == times
    for f in json.loads((tmp_path / "out_element.pvtu.series").read_text())["files"]:
        assert (tmp_path / f["name"]).exists()
    w.close()
    m.close()


@pytest.mark.parametrize("iterative", [False, True])
def test_pre_condition_matches_reference(iterative):
    zone = meshgen.uniform_zone(16, x_periodic=True, boundary=meshgen.WALL)
    ref, m = _pair(zone, 4, 2, N_max=10, max_split_level=1)
    ref.pre_condition(3, 5, iterative)
    solver = ndg.Solver2D_t(0.5)
    steps = (solver.pre_condition_iterative if iterative else solver.pre_condition)(m, 3, 5)
    assert steps == 15
    assert (m.n_elements_, m.n_elements_total_, m.n_faces_) == (ref.n_elements, ref.n_elements_total, ref.n_faces)
    assert np.array_equal(m.elements()["N"], ref.elements()["N"])
    assert m.n_elements_ > 256 and len(set(m.elements()["N"][:m.n_elements_].tolist())) > 1, "split and p-refined"
    # the initial conditions on the adapted mesh (CUDA's exp against the host's)
    for f in ("p", "u", "v"):
        np.testing.assert_allclose(m.get_field(f), ref.field(f), rtol=1e-14, atol=1e-300)
    m.close()


def test_pre_condition_rejects_a_zero_interval():
    zone = meshgen.uniform_zone(4, boundary=meshgen.WALL)
    m = ndg.Mesh2D_t(zone, 3)
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        ndg.Solver2D_t().pre_condition(m, 2, 0)
    m.close()
