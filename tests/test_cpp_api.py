"""The C++ host API (include/ndg_b200.hpp) compiled into a driver shaped
like the reference's src/main.cu:346-390.

CPU: the header compiles and links against libndg_b200.so; NDG_t's packed
tables equal the oracle's bit for bit and Mesh2D_t's counts equal the
reference reader's. GPU: Solver2D_t::solve takes the reference's steps
(include/solvers/Solver2D_t.tcu:7-135: shortened last step, outputs at the
first step end in [e, e + dt)) and its fields match the reference's CPU path
within the FP64 bar (1e-12 relative L2; the mesh has an inflow side, whose
analytic ghost state uses CUDA's exp).
"""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from oracle.pyoracle import oracle_table
from tests import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-12


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "api_driver")
    libdir = os.path.dirname(ndg.LIB_PATH)
    ndg.lib()  # raises if the library has not been built
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "api_driver.cpp"), "-o", out, "-L", libdir, "-lndg_b200",
           f"-Wl,-rpath,{libdir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


@pytest.fixture(scope="module")
def su2_mesh(tmp_path_factory):
    zone = meshgen.uniform_zone(8, jitter=0.1, seed=5)
    path = str(tmp_path_factory.mktemp("mesh") / "mesh.su2")
    meshgen.write_su2(path, zone, meshgen.su2_markers(zone))
    return path


def test_host_tables_and_counts(driver, su2_mesh):
    N = 6
    res = subprocess.run([driver, "host", su2_mesh, str(N)], check=True, capture_output=True, text=True)
    d = json.loads(res.stdout)
    m = ndg.Mesh2D_t(su2_mesh, N, device=-1)
    assert (d["n_elements"], d["n_elements_total"], d["n_faces"], d["n_nodes"], d["field_size"]) == \
        (m.n_elements_, m.n_elements_total_, m.n_faces_, m.n_nodes_, m.field_size)
    for name, table in (("nodes", 0), ("weights", 1), ("derivative_matrices_hat", 9),
                        ("interpolation_matrices", 10), ("polynomials", 11)):
        want = np.concatenate([oracle_table(N, 2, table, n) for n in range(N + 1)])
        assert np.array_equal(np.array(d[name]), want), name


def _read(path):
    with open(path, "rb") as f:
        steps, n_out, size = np.frombuffer(f.read(24), dtype=np.int64)
        dt = np.frombuffer(f.read(8), dtype=np.float64)[0]
        outs = []
        for _ in range(n_out):
            t = np.frombuffer(f.read(8), dtype=np.float64)[0]
            fields = np.frombuffer(f.read(24 * size), dtype=np.float64).reshape(3, size)
            outs.append((t, fields))
    return int(steps), dt, outs


def _reference_plan(dt_mesh, times):
    """Step ends and output flags of the reference loop."""
    t, t_end, plan = 0.0, times[-1], []
    while t < t_end:
        dt = dt_mesh if t + dt_mesh <= t_end else t_end - t
        t += dt
        plan.append((t, dt, any(e <= t < e + dt for e in times)))
    return plan


@pytest.mark.gpu
def test_solve_matches_reference_steps_and_fields(driver, su2_mesh, tmp_path, ref_available):
    if not ref_available:
        pytest.skip("reference CPU build not present")
    from oracle.pyoracle import RefSolver
    N, cfl = 5, 0.4
    ref = RefSolver(su2_mesh, N, cfl=cfl)
    dt_mesh = ref.delta_t()
    times = [7.5 * dt_mesh, 20 * dt_mesh + 0.3 * dt_mesh]
    out = str(tmp_path / "out.bin")
    subprocess.run([driver, "solve", su2_mesh, str(N), repr(cfl), out] + [repr(t) for t in times],
                   check=True, capture_output=True, text=True)
    steps, dt, outs = _read(out)
    plan = _reference_plan(dt_mesh, times)
    assert dt == dt_mesh
    assert steps == len(plan) == 21
    want_times = [t for t, _, w in plan if w]
    if not plan[-1][2]:
        want_times.append(plan[-1][0])
    assert [t for t, _ in outs] == want_times

    ref.initial_conditions()
    t, k = 0.0, 0
    for t_out, fields in outs:
        while k < len(plan) and t < t_out:
            step_end, step_dt, _ = plan[k]
            if step_dt == dt_mesh:
                t = ref.run(1, t)
            else:
                for m in range(3):
                    ref.stage(m, t, step_dt)
                t = step_end
            k += 1
        assert t == t_out
        for i, f in enumerate(("p", "u", "v")):
            w = ref.field(f)
            assert np.linalg.norm(fields[i] - w) <= TOL * np.linalg.norm(w), (t_out, f)


@pytest.mark.gpu
def test_pre_condition_and_data_writer_through_the_cpp_api(driver, su2_mesh, tmp_path):
    """Solver2D_t::pre_condition then solve with a Helpers::DataWriter_t, the
    reference's driver sequence (src/main.cu:346-390): the writer's series
    lists one complete output per output time, each file readable, and the
    mesh is the pre-conditioned (adapted) one."""
    from tests.vtu import read_grid
    out = tmp_path / "wave.pvtu"
    N, cfl = 3, 0.5
    res = subprocess.run([driver, "write", su2_mesh, str(N), repr(cfl), str(out), "2", "4", "0.0", "0.02", "0.05"],
                         check=True, capture_output=True, text=True)
    d = json.loads(res.stdout)
    assert d["pre_condition_steps"] == 8 and d["steps"] > 0
    series = json.loads((tmp_path / "wave.pvtu.series").read_text())["files"]
    elements = json.loads((tmp_path / "wave_element.pvtu.series").read_text())["files"]
    assert [f["time"] for f in series][0] == 0.0 and series[-1]["time"] == 0.05 and len(series) == len(elements) >= 3
    g = read_grid(str(tmp_path / series[-1]["name"]))
    eg = read_grid(str(tmp_path / elements[-1]["name"]))
    assert eg["n_cells"] == d["n_elements"] and g["n_points"] == 9 * d["n_elements"]
    assert np.isfinite(g["point_data"]["Pressure"]).all() and (eg["cell_data"]["N"] >= N).all()
