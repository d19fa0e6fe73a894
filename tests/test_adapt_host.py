"""h- and p-adaptation of the topology against the reference's own
Mesh2D_t::adapt, on the CPU.

The reference steps, estimates its error and adapts; the library adapts a
host-only mesh with the same per-element refine flags and decay rates
(ndg_adapt_flags). Elements (nodes, orders, split levels, Hilbert statuses
and rotations, minimum lengths, face lists), faces (nodes, elements, sides,
orders, normals, tangents, offsets, scales), boundary and interface lists
and node coordinates must agree bit for bit after every round.
"""
from __future__ import annotations

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from tests import meshgen


def _compare(m, r):
    assert (m.n_elements_, m.n_elements_total_, m.n_faces_, m.n_nodes_) == (r.n_elements, r.n_elements_total, r.n_faces, r.n_nodes)
    em, er = m.elements(), r.elements()
    for k in ("nodes", "N", "delta_xy_min", "first_face"):
        assert np.array_equal(em[k], er[k]), k
    sm = m.element_state()
    for k in ("split_level", "status", "rotation", "n_faces_side"):
        assert np.array_equal(sm[k], er[k]), k
    assert np.array_equal(sm["faces"], r.element_faces())
    fm, fr = m.faces(), r.faces()
    for k in ("nodes", "elements", "sides", "N", "normal", "tangent", "offset", "scale"):
        assert np.array_equal(fm[k], fr[k]), k
    for kind in range(7):
        assert np.array_equal(m.boundary(kind), r.boundary(kind)), kind
    assert np.array_equal(np.ravel(m.nodes()), np.ravel(r.nodes()))


CASES = [
    ("periodic", 8, dict(x_periodic=True, y_periodic=True), 4, 8, 2),
    ("walls", 8, dict(boundary=meshgen.WALL), 4, 8, 2),
    ("x_periodic_walls", 16, dict(x_periodic=True, boundary=meshgen.WALL), 4, 8, 2),
    ("jittered", 16, dict(x_periodic=True, y_periodic=True, jitter=0.1, seed=0), 4, 12, 2),
    ("rowmajor_outflow", 12, dict(order="rowmajor", boundary=meshgen.OUTFLOW), 3, 7, 3),
    ("inflow", 8, dict(boundary=meshgen.INFLOW), 4, 8, 2),
    ("symmetry_y_periodic", 16, dict(y_periodic=True, boundary=meshgen.SYMMETRY), 5, 9, 2),
]


@pytest.mark.parametrize("name,res,kw,N,N_max,splits", CASES, ids=[c[0] for c in CASES])
def test_adapt_rounds_bitwise_vs_reference(name, res, kw, N, N_max, splits, ref_available):
    if not ref_available:
        pytest.skip("reference CPU build not present")
    from oracle.pyoracle import RefSolver
    zone = meshgen.uniform_zone(res, **kw)
    r = RefSolver(zone, N, N_max=N_max, max_split_level=splits, tolerance_min=1e-4, tolerance_max=1e-14)
    m = ndg.Mesh2D_t(zone, N, maximum_N=N_max, max_split_level=splits, tolerance_min=1e-4, tolerance_max=1e-14, device=-1)
    r.initial_conditions()
    split_seen = False
    for _ in range(3):
        r.run(10)
        r.estimate_error()
        e = r.error()
        r.adapt()
        m.adapt(e["refine"], e["p_sigma"])
        _compare(m, r)
        split_seen |= m.n_elements_ > res * res
    assert split_seen
