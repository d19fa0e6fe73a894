"""CPU tests of the product library (no GPU): the C ABI loads and exports
every declared entry point, the host FP64 tables and the host topology
builder match the oracle bit for bit, and bad input fails with a status
instead of exiting."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from oracle.pyoracle import OracleSolver, oracle_table
from tests import meshgen
from tests.meshgen import su2_markers, write_su2

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "ndg_b200.h")


def declared_symbols() -> list[str]:
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:ndg_status|const char\*)\s+(ndg_\w+)\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = ndg.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
    assert b"sm_100a" in L.ndg_version()


@pytest.mark.parametrize("N", range(0, 17))
def test_tables_bitwise_vs_oracle(N):
    for t, name in enumerate(ndg.TABLES):
        a = ndg.tables_compute(16, 9, name, N)
        b = oracle_table(16, 9, t, N)
        assert np.array_equal(a, b), (name, N)


ZONES = [
    ("periodic", 8, dict(x_periodic=True, y_periodic=True)),
    ("wall", 8, dict(boundary=meshgen.WALL)),
    ("inflow", 4, dict(boundary=meshgen.INFLOW)),
    ("x_periodic", 8, dict(x_periodic=True, boundary=meshgen.OUTFLOW)),
    ("rowmajor_jitter", 6, dict(order="rowmajor", jitter=0.1, x_periodic=True, y_periodic=True)),
    ("hilbert_r32", 32, dict(x_periodic=True, y_periodic=True)),
]


@pytest.mark.parametrize("name,res,kw", ZONES, ids=[z[0] for z in ZONES])
def test_topology_bitwise_vs_oracle(name, res, kw):
    zone = meshgen.uniform_zone(res, **kw)
    m = ndg.Mesh2D_t(zone, 4, device=-1)
    o = OracleSolver(zone, 4)
    assert (m.n_elements_, m.n_elements_total_, m.n_faces_, m.n_nodes_) == (o.n_elements, o.n_elements_total, o.n_faces, o.n_nodes)
    fm, fo = m.faces(), o.faces()
    for k in fo:
        assert np.array_equal(fm[k], fo[k]), k
    em, eo = m.elements(), o.elements()
    for k in eo:
        assert np.array_equal(em[k], eo[k]), k
    for kind in range(7):
        assert np.array_equal(m.boundary(kind), o.boundary(kind)), kind
    assert np.array_equal(m.nodes(), o.nodes())




def test_su2_reader_bitwise_vs_reference_reader(tmp_path, ref_available):
    from oracle import pyoracle
    zone = meshgen.uniform_zone(4)
    path = str(tmp_path / "mesh.su2")
    write_su2(path, zone, su2_markers(zone))
    m = ndg.Mesh2D_t(path, 3, device=-1)
    r = pyoracle.RefSolver(path, 3)
    assert (m.n_elements_, m.n_elements_total_, m.n_faces_) == (r.n_elements, r.n_elements_total, r.n_faces)
    fm, fr = m.faces(), r.faces()
    for k in ("nodes", "elements", "sides", "N", "normal", "tangent", "offset", "scale"):
        assert np.array_equal(fm[k], fr[k]), k
    em, er = m.elements(), r.elements()
    for k in ("nodes", "N", "delta_xy_min", "first_face"):
        assert np.array_equal(em[k], er[k]), k
    for kind in range(7):
        assert np.array_equal(m.boundary(kind), r.boundary(kind)), kind


def test_bad_input_returns_status_not_exit():
    zone = meshgen.uniform_zone(4, x_periodic=True, y_periodic=True)
    with pytest.raises(ndg.NdgError) as e:
        ndg.Mesh2D_t(zone, 5, maximum_N=4, device=-1)
    assert e.value.status == 1
    bad = dict(zone)
    secs = list(bad["sections"])
    name, typ, start, end, conn = secs[0]
    conn = conn.copy()
    conn[0] = 10_000
    secs[0] = (name, typ, start, end, conn)
    bad["sections"] = secs
    with pytest.raises(ndg.NdgError) as e:
        ndg.Mesh2D_t(bad, 3, device=-1)
    assert e.value.status == 2
    with pytest.raises(ndg.NdgError):
        ndg.tables_compute(16, 9, "nodes", 17)
    # GPU-only calls on a host-only context fail with a status.
    m = ndg.Mesh2D_t(zone, 3, device=-1)
    with pytest.raises(ndg.NdgError) as e:
        m.initial_conditions()
    assert e.value.status == 1
    assert ndg.lib().ndg_last_error().decode() != ""


def test_missing_file_and_unknown_extension():
    with pytest.raises(ndg.NdgError):
        ndg.Mesh2D_t("/nonexistent/mesh.su2", 3, device=-1)
    with pytest.raises(ndg.NdgError):
        ndg.Mesh2D_t("mesh.msh", 3, device=-1)
    with pytest.raises(ndg.NdgError) as e:
        ndg.Mesh2D_t("mesh.cgns", 3, device=-1)
    assert e.value.status == 7
    _ = C  # ctypes is used through the package


@pytest.mark.parametrize("res, kw", [(8, dict(x_periodic=True)), (16, dict(jitter=0.1, seed=3)),
                                     (8, dict(order="rowmajor", x_periodic=True, y_periodic=True)), (4, {})])
def test_element_state_bitwise_vs_reference(res, kw, ref_available):
    """Split level, Hilbert status and rotation (Mesh2D_t::compute_element_status)
    and per-side face lists at load, against the reference."""
    if not ref_available:
        pytest.skip("reference CPU build not present")
    from oracle.pyoracle import RefSolver
    zone = meshgen.uniform_zone(res, **kw)
    m = ndg.Mesh2D_t(zone, 3, device=-1)
    r = RefSolver(zone, 3)
    sm, er = m.element_state(), r.elements()
    for k in ("split_level", "status", "rotation", "n_faces_side"):
        assert np.array_equal(sm[k], er[k]), k
    assert np.array_equal(sm["faces"], r.element_faces())


def test_tile_candidates_on_a_host_context():
    """The autotuner's candidate tiles need no GPU to list: powers of two
    that fit 512 threads and 113 KB of shared memory, then the tensor-core
    tiles (TENSOR_TILE + 2, 4, 8) from order 6 up."""
    zone = meshgen.uniform_zone(4, boundary=meshgen.WALL)
    m = ndg.Mesh2D_t(zone, 8, device=-1)
    cand, default = m.tile_candidates()
    T = ndg.TENSOR_TILE
    assert cand == [2, 4, 8, 16, T + 2, T + 4, T + 8] and default == 4
    m4 = ndg.Mesh2D_t(zone, 4, device=-1)
    assert all(t < T for t in m4.tile_candidates()[0])
    m16 = ndg.Mesh2D_t(zone, 16, device=-1)
    cand16, _ = m16.tile_candidates()
    simt16 = [c % T for c in cand16]
    assert cand16 and max(simt16) * 3 * 17 <= 512 and all(c in (2, 4, 8, 16) for c in simt16)


def test_mixed_launch_modes_on_a_host_context():
    """ndg_set_mixed_launch takes 0 (one launch per order group, large
    non-conforming orders split), 1 (one queue launch per stage) and 2 (every
    group split into side fluxes and element tiles); other modes are an
    invalid argument, reported as a status."""
    zone = meshgen.uniform_zone(4, x_periodic=True, y_periodic=True)
    m = ndg.Mesh2D_t(zone, 4, device=-1)
    for mode in (0, 1, 2):
        m.set_mixed_launch(mode)
    for mode in (-1, 3):
        with pytest.raises(ndg.NdgError) as e:
            m.set_mixed_launch(mode)
        assert e.value.status == 1
        assert "mode is 0" in ndg.lib().ndg_last_error().decode()
