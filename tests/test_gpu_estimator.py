"""GPU error estimator against the oracle (src/entities/Element2D_t.cpp:274-343).

The oracle's estimator is pinned bit for bit to the reference's
(tests/test_oracle.py). The device kernel rounds every product and sum as
the reference does; only log/exp come from CUDA, so errors and decay rates
agree to a few ulp and refine/coarsen flags are identical wherever the error
is not within 1e-12 (relative) of a tolerance. Elements whose spectrum
underflows to zero give NaN in both, with no refinement.
"""
from __future__ import annotations

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from oracle.pyoracle import OracleSolver
from tests import meshgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [1, 2, 4, 6, 8, 12, 16])
@pytest.mark.parametrize("steps", [0, 7])
def test_estimator_matches_oracle(N, steps):
    tol_min, tol_max = 1e-4, 1e-9
    zone = meshgen.uniform_zone(8, x_periodic=True, boundary=meshgen.WALL)
    o = OracleSolver(zone, N, tolerance_min=tol_min, tolerance_max=tol_max)
    o.initial_conditions()
    m = ndg.Mesh2D_t(zone, N, tolerance_min=tol_min, tolerance_max=tol_max, precision=ndg.FP64_STRICT)
    for f in ("p", "u", "v"):
        m.set_field(f, o.field(f))
    if steps:
        o.run(steps)
        ndg.Solver2D_t.run(m, steps)
        for f in ("p", "u", "v"):
            assert np.array_equal(m.get_field(f), o.field(f))
    o.estimate_error()
    m.estimate_error()
    want, got = o.error(), m.error()
    for k in ("p_error", "p_sigma"):
        w, g = want[k], got[k]
        assert np.array_equal(np.isnan(w), np.isnan(g)), k
        ok = ~np.isnan(w)
        np.testing.assert_allclose(g[ok], w[ok], rtol=1e-13, atol=0, err_msg=k)
    err = want["p_error"]
    far = np.isnan(err) | ((np.abs(err - tol_min) > 1e-12 * tol_min) & (np.abs(err - tol_max) > 1e-12 * tol_max))
    assert far.sum() > 0.9 * err.size
    for k in ("refine", "coarsen"):
        assert np.array_equal(got[k][far], want[k][far]), k


def test_estimator_all_instances():
    zone = meshgen.uniform_zone(4, x_periodic=True, y_periodic=True)
    o = OracleSolver(zone, 5, tolerance_min=1e-3, tolerance_max=1e-8)
    o.initial_conditions()
    p = o.field("p")
    m = ndg.Mesh2D_t(zone, 5, n_instances=2, tolerance_min=1e-3, tolerance_max=1e-8)
    m.set_field("p", np.concatenate([p, 3.0 * p]))
    m.estimate_error()
    o.estimate_error()
    e0, e1 = m.error(0), m.error(1)
    np.testing.assert_allclose(e0["p_error"], o.error()["p_error"], rtol=1e-13)
    # The estimator is homogeneous of degree 1 in p: the error triples, the rate stays.
    ok = ~np.isnan(e0["p_error"])
    np.testing.assert_allclose(e1["p_error"][ok], 3.0 * e0["p_error"][ok], rtol=1e-12)
    np.testing.assert_allclose(e1["p_sigma"][ok], e0["p_sigma"][ok], rtol=1e-12)
