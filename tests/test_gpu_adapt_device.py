"""Adaptation decisions on the device (adapt_device.cu) against the host's.

A GPU context decides an adaptation on the device: per-element flags from
the estimate, the new-node flags of splitting elements' sides (find_nodes),
the ghosts' copies (copy_interfaces_error, copy_boundaries_error), the face
splits and the exclusive counts that number new elements, faces and nodes.
A host-only context decides the same adaptation on the host. With the same
flags, three rounds of mixed p- and h-refinement on meshes with every
boundary kind and periodic interfaces must give bit-identical topologies:
elements, orders, split levels, Hilbert statuses, rotations, face lists,
faces, boundary lists and nodes. The lockstep tests against the reference
(tests/test_gpu_hp_config.py, tests/test_gpu_adapt.py) run the device path
too.
"""
from __future__ import annotations

import zlib

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from tests import meshgen

pytestmark = pytest.mark.gpu


def _same_topology(a, b):
    assert (a.n_elements_, a.n_elements_total_, a.n_faces_, a.n_nodes_) == (b.n_elements_, b.n_elements_total_, b.n_faces_, b.n_nodes_)
    ea, eb = a.elements(), b.elements()
    for k in ("nodes", "N", "delta_xy_min", "first_face"):
        assert np.array_equal(ea[k], eb[k]), k
    sa, sb = a.element_state(), b.element_state()
    for k in ("split_level", "status", "rotation", "n_faces_side", "faces"):
        assert np.array_equal(sa[k], sb[k]), k
    fa, fb = a.faces(), b.faces()
    for k in ("nodes", "elements", "sides", "N", "normal", "tangent", "offset", "scale"):
        assert np.array_equal(fa[k], fb[k]), k
    for kind in range(7):
        assert np.array_equal(a.boundary(kind), b.boundary(kind)), kind
    assert np.array_equal(np.ravel(a.nodes()), np.ravel(b.nodes()))


CASES = [
    ("periodic", 8, dict(x_periodic=True, y_periodic=True), 4, 8, 2),
    ("walls_jittered", 16, dict(boundary=meshgen.WALL, jitter=0.1, seed=7), 4, 12, 2),
    ("x_periodic_walls", 16, dict(x_periodic=True, boundary=meshgen.WALL), 4, 8, 2),
    ("rowmajor_outflow", 12, dict(order="rowmajor", boundary=meshgen.OUTFLOW), 3, 7, 3),
    ("inflow", 8, dict(boundary=meshgen.INFLOW), 4, 8, 2),
    ("symmetry_y_periodic", 16, dict(y_periodic=True, boundary=meshgen.SYMMETRY), 5, 9, 2),
]


@pytest.mark.parametrize("name,res,kw,N,N_max,splits", CASES, ids=[c[0] for c in CASES])
def test_device_decisions_equal_host_decisions(name, res, kw, N, N_max, splits):
    zone = meshgen.uniform_zone(res, **kw)
    dev = ndg.Mesh2D_t(zone, N, maximum_N=N_max, max_split_level=splits)
    host = ndg.Mesh2D_t(zone, N, maximum_N=N_max, max_split_level=splits, device=-1)
    dev.initial_conditions()
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    split_seen = False
    for _ in range(3):
        K = dev.n_elements_
        refine = (rng.random(K) < 0.3).astype(np.int32)
        sigma = rng.choice([0.25, 0.999, 1.0, 3.0], size=K)
        dev.adapt(refine, sigma)
        host.adapt(refine, sigma)
        _same_topology(dev, host)
        split_seen |= dev.n_elements_ > res * res
    assert split_seen
    ndg.Solver2D_t.run(dev, 2)
    assert np.isfinite(dev.get_field("p")).all()
    dev.close()
    host.close()


def test_device_decisions_from_the_device_estimate():
    """ndg_adapt: the decisions start from the estimator's device arrays."""
    zone = meshgen.uniform_zone(16, boundary=meshgen.WALL, jitter=0.1, seed=7)
    dev = ndg.Mesh2D_t(zone, 4, maximum_N=12, max_split_level=2, tolerance_min=1e-9, tolerance_max=1e-14)
    host = ndg.Mesh2D_t(zone, 4, maximum_N=12, max_split_level=2, tolerance_min=1e-9, tolerance_max=1e-14, device=-1)
    from tests import hp_lockstep
    ic = hp_lockstep.pulses(zone, 4)
    for f in ("p", "u", "v"):
        dev.set_field(f, ic[f])
    for _ in range(3):
        ndg.Solver2D_t.run(dev, 20)
        dev.estimate_error()
        e = dev.error()
        dev.adapt()
        host.adapt(e["refine"], e["p_sigma"])
        _same_topology(dev, host)
    assert dev.n_elements_ > 256 and len(set(dev.elements()["N"][:dev.n_elements_].tolist())) > 1
    dev.close()
    host.close()
