"""The three launch structures of a stage on a mixed-order mesh: one launch
per order group as concurrent graph branches (the default), one launch
per stage over a queue of every order group's tiles, and the groups split
into a side-flux launch and an element-tile launch (the conforming-element
kernel over the side fluxes). Each computes the same operations, so the
fields must be bit-identical in FP64_STRICT;
in FP64 and FP32 the two compilations may contract multiply-adds
differently, so they are held to 1e-12 and 1e-6 relative L2. Meshes after
p-adaptation (mortar faces between orders) and after element splitting
(nonconforming faces, ghosts on walls). Launch counts of the queue form:
the ghost kernel plus one launch per stage. In the default form each
order's conforming elements (conforming_stage_kernel) and the rest are
groups of their own, so the comparison also pins the conforming kernel to
the general one.
"""
from __future__ import annotations

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from tests import meshgen

pytestmark = pytest.mark.gpu


def _mixed_mesh(kind, precision, n_instances=1):
    if kind == "p_periodic":
        zone = meshgen.uniform_zone(16, x_periodic=True, y_periodic=True, jitter=0.1, seed=1)
        m = ndg.Mesh2D_t(zone, 4, maximum_N=10, n_instances=n_instances, precision=precision)
        m.initial_conditions()
        rng = np.random.default_rng(0)
        for _ in range(3):
            K = m.n_elements_
            m.adapt((rng.random(K) < 0.4).astype(np.int32), np.full(K, 2.0))
    else:
        zone = meshgen.uniform_zone(16, boundary=meshgen.WALL, jitter=0.1, seed=7)
        m = ndg.Mesh2D_t(zone, 4, maximum_N=8, max_split_level=2, n_instances=n_instances, precision=precision)
        m.initial_conditions()
        rng = np.random.default_rng(5)
        for _ in range(2):
            K = m.n_elements_
            refine = (rng.random(K) < 0.3).astype(np.int32)
            sigma = np.where(rng.random(K) < 0.5, 0.5, 2.0)
            m.adapt(refine, sigma)
    return m


@pytest.mark.parametrize("precision", [ndg.FP64_STRICT, ndg.FP64, ndg.FP32])
@pytest.mark.parametrize("kind", ["p_periodic", "hp_walls"])
def test_queue_and_group_launches_agree(kind, precision):
    m = _mixed_mesh(kind, precision)
    N = m.elements()["N"][:m.n_elements_]
    assert len(set(N.tolist())) >= 2
    state = {f: m.get_field(f) for f in ("p", "u", "v", "k_p", "k_u", "k_v")}
    out = []
    for mode in (0, 1, 2):
        m.set_mixed_launch(mode)
        for f, v in state.items():
            m.set_field(f, v)
        launches0 = m.launches()
        ndg.Solver2D_t.run(m, 6)
        out.append(({f: m.get_field(f) for f in ("p", "u", "v")}, m.launches() - launches0))
    (a, _), (b, launches_queue), (c, _) = out
    tol = {ndg.FP64_STRICT: 0.0, ndg.FP64: 1e-12, ndg.FP32: 1e-6}[precision]
    for other in (b, c):
        for f in ("p", "u", "v"):
            assert np.linalg.norm(a[f] - other[f]) <= tol * np.linalg.norm(a[f]), f
            assert np.isfinite(other[f]).all()
    ghosts = 1 if m.n_elements_total_ > m.n_elements_ else 0
    # per step: 3 stages x (ghosts + queue) + the time update; then the first
    # traces, one launch per order's conforming part and per its other part
    assert launches_queue <= 6 * (3 * (1 + ghosts) + 1) + 2 * len(set(N.tolist()))
    m.close()
