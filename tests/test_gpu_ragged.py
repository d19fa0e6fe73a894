"""Ragged tiles: element counts that no tile divides and that are odd (the
device field blocks then carry one padding element), for every candidate
tile of the uniform-order stage kernels, in every form, with several
instances sharing the mesh, against the oracle.

The last CTA of a launch holds fewer elements than its tile; its copies,
traces, fluxes and RK updates must stop at the last element, and the
padding element between instances must never leak into a neighbour's
fields. Bars: bit-exact in FP64_STRICT (default tile), 1e-12 relative L2
in FP64 (every tile; the SIMT tiles bit-identical to each other), 1e-6 in
FP32.
"""
from __future__ import annotations

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from oracle.pyoracle import OracleSolver
from tests import meshgen

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("res,N", [(7, 4), (5, 8), (9, 3), (3, 12)])
@pytest.mark.parametrize("kind", ["periodic", "walls"])
def test_odd_element_counts_every_tile(res, N, kind):
    kw = {"periodic": dict(x_periodic=True, y_periodic=True), "walls": dict(boundary=meshgen.WALL)}[kind]
    zone = meshgen.uniform_zone(res, order="rowmajor", jitter=0.1, seed=res, **kw)
    assert (res * res) % 2 == 1
    o = OracleSolver(zone, N)
    o.initial_conditions()
    ic = {f: o.field(f) for f in ("p", "u", "v")}
    steps = 6
    o.run(steps)
    want = {f: o.field(f) for f in ("p", "u", "v")}

    strict = ndg.Mesh2D_t(zone, N, precision=ndg.FP64_STRICT)
    for f in ("p", "u", "v"):
        strict.set_field(f, ic[f])
    ndg.Solver2D_t.run(strict, steps)
    for f in ("p", "u", "v"):
        assert np.array_equal(strict.get_field(f), want[f]), f
    strict.close()

    for precision, tol in ((ndg.FP64, 1e-12), (ndg.FP32, 1e-6)):
        # three instances: the oracle's initial state, its negative, and half of it
        m = ndg.Mesh2D_t(zone, N, precision=precision, n_instances=3)
        cand, _ = m.tile_candidates()
        first = None
        for tile in [0] + cand:
            m.set_tile(tile)
            for f in ("p", "u", "v"):
                m.set_field(f, np.concatenate([ic[f], -ic[f], 0.5 * ic[f]]))
            for f in ("k_p", "k_u", "k_v"):
                m.set_field(f, np.zeros(3 * m.field_size))
            ndg.Solver2D_t.run(m, steps)
            got = {f: m.get_field(f, instance=-1) for f in ("p", "u", "v")}
            for f in ("p", "u", "v"):
                a, b, c = np.split(got[f], 3)
                assert rel_l2(a, want[f]) < tol, (precision, tile, f)
                # the operator is linear: the other instances are exact multiples in FP64
                if precision == ndg.FP64:
                    assert rel_l2(b, -want[f]) < tol and rel_l2(c, 0.5 * want[f]) < tol, (tile, f)
            if first is None:
                first = got
            elif tile < ndg.TENSOR_TILE:  # tensor-core tiles sum in another order: held to tol above
                for f in ("p", "u", "v"):
                    assert np.array_equal(got[f], first[f]), (precision, tile, f)
        m.close()
