"""L2 error against the analytic plane wave (ndg_l2_error) against the
oracle's computation of the same norm, sqrt(sum w_i w_j J (q - g)^2), on the
same fields: equal to 1e-13 (they differ in summation order and in the
exponential of the plane wave, CUDA's against the host's), for the uniform
and the mixed-order path; zero (to the exponential's last bit) at t = 0
after the oracle's initial condition."""
from __future__ import annotations

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from oracle.pyoracle import OracleSolver
from tests import meshgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [2, 4, 8])
@pytest.mark.parametrize("kind", ["periodic", "walls_jittered"])
def test_l2_error_matches_oracle(N, kind):
    kw = {"periodic": dict(x_periodic=True, y_periodic=True),
          "walls_jittered": dict(boundary=meshgen.WALL, jitter=0.1, seed=2)}[kind]
    zone = meshgen.uniform_zone(16, **kw)
    o = OracleSolver(zone, N)
    o.initial_conditions()
    m = ndg.Mesh2D_t(zone, N, precision=ndg.FP64_STRICT)
    for f in ("p", "u", "v"):
        m.set_field(f, o.field(f))
    # the oracle's own initial condition is its g at t = 0; the device's g
    # uses CUDA's exp, within an ulp of the host's
    assert np.all(o.l2_error(0.0) == 0.0) and np.all(m.l2_error(0.0) < 1e-14)
    t_o = o.run(12)
    t_m = ndg.Solver2D_t.run(m, 12)
    assert t_o == t_m
    got, want = m.l2_error(t_m), o.l2_error(t_o)
    assert np.all(want > 0)
    np.testing.assert_allclose(got, want, rtol=1e-13)
    m.close()


def test_l2_error_on_a_mixed_order_mesh():
    zone = meshgen.uniform_zone(16, x_periodic=True, y_periodic=True)
    m = ndg.Mesh2D_t(zone, 4, maximum_N=8)
    m.initial_conditions()
    K = m.n_elements_
    rng = np.random.default_rng(1)
    m.adapt((rng.random(K) < 0.4).astype(np.int32), np.full(K, 2.0))
    assert len(set(m.elements()["N"][:m.n_elements_].tolist())) == 2
    t = ndg.Solver2D_t.run(m, 5)
    # the same norm from the nodal fields on the host
    el = m.elements()
    N = el["N"][:m.n_elements_]
    nodes = m.nodes()
    quads = el["nodes"].reshape(-1, 4)[:m.n_elements_]
    fields = {f: m.get_field(f) for f in ("p", "u", "v")}
    s = np.zeros(3)
    off = 0
    kx = ky = 0.707106781186548
    d = 0.120112240878645
    for e in range(m.n_elements_):
        n = int(N[e]) + 1
        xn = ndg.tables_compute(int(N.max()), 2, "nodes", int(N[e]))
        w = ndg.tables_compute(int(N.max()), 2, "weights", int(N[e]))
        px, py = nodes[quads[e], 0], nodes[quads[e], 1]
        for i in range(n):
            for j in range(n):
                xi, eta = xn[i], xn[j]
                x = (px[0] * (1 - xi) * (1 - eta) + px[1] * (xi + 1) * (1 - eta) + px[2] * (xi + 1) * (eta + 1) + px[3] * (1 - xi) * (eta + 1)) / 4
                y = (py[0] * (1 - xi) * (1 - eta) + py[1] * (xi + 1) * (1 - eta) + py[2] * (xi + 1) * (eta + 1) + py[3] * (1 - xi) * (eta + 1)) / 4
                m00 = ((1 - eta) * (px[1] - px[0]) + (1 + eta) * (px[2] - px[3])) / 4
                m01 = ((1 - xi) * (px[3] - px[0]) + (1 + xi) * (px[2] - px[1])) / 4
                m10 = ((1 - eta) * (py[1] - py[0]) + (1 + eta) * (py[2] - py[3])) / 4
                m11 = ((1 - xi) * (py[3] - py[0]) + (1 + xi) * (py[2] - py[1])) / 4
                J = m00 * m11 - m01 * m10
                a = kx * (x + 0.2) + ky * (y + 0.2) - t
                g = np.exp(-a * a / (d * d))
                gv = (g, g * kx, g * ky)
                k = off + i * n + j
                for f, name in enumerate(("p", "u", "v")):
                    s[f] += w[i] * w[j] * J * (fields[name][k] - gv[f]) ** 2
        off += n * n
    np.testing.assert_allclose(m.l2_error(t), np.sqrt(s), rtol=1e-11)
    m.close()
