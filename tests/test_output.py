"""Solution output without a GPU.

* The oracle's restatement of Mesh2D_t::get_complete_solution
  (src/meshes/Mesh2D_t.cpp:4251-4296, Element2D_t::interpolate_complete_solution,
  src/entities/Element2D_t.cpp:606-646) against the reference's own code,
  bit for bit: coordinates, fields, time derivatives and analytic errors.
* The file writer in DataWriter_t's role (src/helpers/DataWriter_t.cpp) on
  host arrays: time-stamped names, the point grid (n x n points per element,
  one quad per grid cell with the reference's corner order), the element grid
  (one quad per element through its output-grid corners), array names,
  types, components and values, and the JSON time series files.
"""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from oracle import pyoracle
from oracle.pyoracle import OracleSolver
from tests import meshgen
from tests.vtu import read_grid

needs_ref = pytest.mark.skipif(not pyoracle.ref_available(), reason="reference checker not built (oracle/_ref/libndgref.so)")


@needs_ref
@pytest.mark.parametrize("N", [1, 3, 6, 8])
@pytest.mark.parametrize("kind", ["periodic_jittered", "walls"])
@pytest.mark.parametrize("n_interp", [2, 5])
def test_oracle_output_matches_reference(N, kind, n_interp):
    from oracle.pyoracle import RefSolver
    kw = {"periodic_jittered": dict(x_periodic=True, y_periodic=True, jitter=0.1, seed=2),
          "walls": dict(boundary=meshgen.WALL)}[kind]
    zone = meshgen.uniform_zone(8, **kw)
    ref = RefSolver(zone, N, n_interp=n_interp)
    orc = OracleSolver(zone, N)
    ref.initial_conditions()
    orc.initial_conditions()
    ref.run(6)
    orc.run(6)
    a, b = ref.complete_solution(0.37), orc.complete_solution(n_interp, 0.37)
    for k in pyoracle.OUTPUT_NAMES:
        assert np.array_equal(a[k], b[k]), k


def _synthetic(K, P, seed=0):
    rng = np.random.default_rng(seed)
    n = K * P * P
    arrays = {k: rng.standard_normal(n) for k in ndg.SOLUTION_NAMES}
    arrays.update(N=rng.integers(1, 9, K), status=rng.integers(0, 4, K), rotation=rng.integers(0, 4, K),
                  p_error=rng.random(K), p_sigma=rng.random(K), refine=rng.integers(0, 2, K),
                  coarsen=rng.integers(0, 2, K), split_level=rng.integers(0, 3, K))
    return arrays


def _expected_quads(K, P):
    quads = []
    for e in range(K):
        o = e * P * P
        for i in range(P - 1):
            for j in range(P - 1):
                quads.append([o + (i + 1) * P + j, o + (i + 1) * P + j + 1, o + i * P + j + 1, o + i * P + j])
    return np.array(quads, dtype=np.int64).reshape(-1)


def test_writer_complete_output(tmp_path):
    K, P = 5, 4
    a = _synthetic(K, P)
    w = ndg.DataWriter_t(str(tmp_path / "output.pvtu"))
    # DataWriter_t's constructor creates both series files empty
    for name in ("output.pvtu.series", "output_element.pvtu.series"):
        assert json.loads((tmp_path / name).read_text()) == {"file-series-version": "1.0", "files": []}
    w.write_arrays(0.25, K, P, a, complete=True, rank=3)
    g = read_grid(str(tmp_path / "output_t0_250000000s.pvtu"))
    assert g["piece_file"] == "output_t0_250000000s_0.vtu"
    assert g["n_points"] == K * P * P and g["n_cells"] == K * (P - 1) ** 2
    assert np.array_equal(g["points"][:, 0], a["x"]) and np.array_equal(g["points"][:, 1], a["y"]) and not g["points"][:, 2].any()
    assert np.array_equal(g["connectivity"], _expected_quads(K, P))
    assert np.array_equal(g["offsets"], 4 * np.arange(1, g["n_cells"] + 1)) and (g["types"] == 9).all()
    assert [n for n, _, _ in g["summary_point_data"]] == ["Pressure", "Velocity", "PressureDerivative", "VelocityDerivative",
                                                          "PressureAnalyticalError", "VelocityAnalyticalError"]
    pd = g["point_data"]
    assert np.array_equal(pd["Pressure"], a["p"])
    assert np.array_equal(pd["Velocity"], np.stack([a["u"], a["v"]], axis=1))
    assert np.array_equal(pd["PressureDerivative"], a["dp_dt"])
    assert np.array_equal(pd["VelocityDerivative"], np.stack([a["du_dt"], a["dv_dt"]], axis=1))
    assert np.array_equal(pd["PressureAnalyticalError"], a["p_analytical_error"])
    assert np.array_equal(pd["VelocityAnalyticalError"], np.stack([a["u_analytical_error"], a["v_analytical_error"]], axis=1))

    eg = read_grid(str(tmp_path / "output_element_t0_250000000s.pvtu"))
    assert eg["n_points"] == 4 * K and eg["n_cells"] == K
    corner = [0, (P - 1) * P, (P - 1) * P + P - 1, P - 1]
    want_pts = np.array([[a["x"][e * P * P + c], a["y"][e * P * P + c]] for e in range(K) for c in corner])
    assert np.array_equal(eg["points"][:, :2], want_pts)
    assert np.array_equal(eg["connectivity"], np.arange(4 * K))
    assert [(n, t) for n, t, _ in eg["summary_cell_data"]] == [
        ("N", "Int32"), ("Index", "UInt64"), ("Status", "Int32"), ("Rotation", "Int32"), ("Rank", "Int32"),
        ("PressureError", "Float64"), ("VelocityError", "Float64"), ("PressureSigma", "Float64"),
        ("VelocitySigma", "Float64"), ("Refine", "Int32"), ("Coarsen", "Int32"), ("SplitLevel", "Int32")]
    cd = eg["cell_data"]
    for name, key in (("N", "N"), ("Status", "status"), ("Rotation", "rotation"), ("PressureError", "p_error"),
                      ("PressureSigma", "p_sigma"), ("Refine", "refine"), ("Coarsen", "coarsen"), ("SplitLevel", "split_level")):
        assert np.array_equal(cd[name], a[key]), name
    assert np.array_equal(cd["Index"], np.arange(K)) and (cd["Rank"] == 3).all()
    # velocity errors and decay rates not given: zeros, two components
    assert cd["VelocityError"].shape == (K, 2) and not cd["VelocityError"].any()
    for name in ("output.pvtu.series", "output_element.pvtu.series"):
        s = json.loads((tmp_path / name).read_text())
        stem = "output_element" if "element" in name else "output"
        assert s == {"file-series-version": "1.0", "files": [{"name": f"{stem}_t0_250000000s.pvtu", "time": 0.25}]}
    w.close()


def test_writer_plain_output_and_series_text(tmp_path):
    """write_data: the point grid with Pressure and Velocity only, and only
    the main series grows; the series text is printed as the reference's JSON
    library prints it (two-space indentation, shortest round-trip numbers)."""
    K, P = 3, 2
    a = _synthetic(K, P, seed=1)
    w = ndg.DataWriter_t(str(tmp_path / "run.vtu"))
    times = [0.0, 1e-05, 0.1, 2.0, 123.25]
    for t in times:
        w.write_arrays(t, K, P, {k: a[k] for k in ("x", "y", "p", "u", "v")})
    g = read_grid(str(tmp_path / "run_t0_100000000s.vtu"))
    assert sorted(g["point_data"]) == ["Pressure", "Velocity"] and g["cell_data"] == {}
    assert not (tmp_path / "run_element_t0_100000000s.vtu").exists()
    text = (tmp_path / "run.vtu.series").read_text()
    names = ["run_t0_000000000s.vtu", "run_t0_000010000s.vtu", "run_t0_100000000s.vtu", "run_t2_000000000s.vtu",
             "run_t123_250000000s.vtu"]
    nums = ["0.0", "1e-05", "0.1", "2.0", "123.25"]
    entries = ",\n".join(f'    {{\n      "name": "{n}",\n      "time": {v}\n    }}' for n, v in zip(names, nums))
    assert text == '{\n  "file-series-version": "1.0",\n  "files": [\n' + entries + "\n  ]\n}\n"
    assert json.loads((tmp_path / "run_element.vtu.series").read_text())["files"] == []
    w.close()


def test_writer_rejects_bad_input(tmp_path):
    w = ndg.DataWriter_t(str(tmp_path / "o.pvtu"))
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        w.write_arrays(0.0, 2, 1, {k: np.zeros(2) for k in ("x", "y", "p", "u", "v")})
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        w.write_arrays(0.0, 2, 2, {k: np.zeros(8) for k in ("x", "y", "p")})
    with pytest.raises(ndg.NdgError):
        ndg.DataWriter_t(str(tmp_path / "missing_directory" / "o.pvtu"))
    w.close()


def test_output_and_pre_condition_need_a_gpu_context():
    zone = meshgen.uniform_zone(4, boundary=meshgen.WALL)
    m = ndg.Mesh2D_t(zone, 3, device=-1, n_interpolation_points=3)
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        m.get_solution()
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        ndg.Solver2D_t().pre_condition(m, 1, 2)
    m.close()
