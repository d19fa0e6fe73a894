"""Tile candidates and the autotuner of the uniform-order stage kernel
(ndg_autotune, ndg_set_tile).

A SIMT tile only groups elements into CTAs; each element's arithmetic is the
same in every such tile, so those candidates must give bit-identical fields
to the default tile, in the FP64 and the FP32 forms, with several instances.
Tensor-core tiles (codes >= TENSOR_TILE) sum the contractions in the tensor
cores' order, so they are held to a tolerance instead: 1e-12 relative L2 in
FP64; in FP32 both tiles lie within the form's 1e-6 of the FP64 result
(3xTF32 against FP32 FMAs), so within 2e-6 of each other. The autotuner must
leave the fields as it found them.
"""
from __future__ import annotations

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from tests import meshgen

pytestmark = pytest.mark.gpu


def _pulses(mesh, zone, N, n_inst, seed=0):
    from tests import adjoint_setup as A
    rng = np.random.default_rng(seed)
    return np.concatenate([A.gaussian_pulse(zone, N, sigma=0.2, centre=rng.uniform(-0.6, 0.6, 2)) for _ in range(n_inst)])


@pytest.mark.parametrize("precision", [ndg.FP64, ndg.FP32])
@pytest.mark.parametrize("N", [3, 6, 8])
def test_every_tile_gives_the_same_fields(N, precision):
    zone = meshgen.uniform_zone(8, boundary=meshgen.WALL)
    n_inst = 3
    results = []
    mesh = ndg.Mesh2D_t(zone, N, n_instances=n_inst, precision=precision)
    p0 = _pulses(mesh, zone, N, n_inst)
    cand, default = mesh.tile_candidates()
    assert default in cand or default > 0
    for tile in [0] + cand:
        mesh.set_tile(tile)
        mesh.set_field("p", p0)
        for f in ("u", "v", "k_p", "k_u", "k_v"):
            mesh.set_field(f, np.zeros_like(p0))
        ndg.Solver2D_t.run(mesh, 5)
        results.append([mesh.get_field(f) for f in ("p", "u", "v")])
    tol = 1e-12 if precision == ndg.FP64 else 2e-6
    for tile, r in zip(cand, results[1:]):
        for a, b in zip(r, results[0]):
            if tile >= ndg.TENSOR_TILE:
                assert np.linalg.norm(a - b) <= tol * np.linalg.norm(b), tile
            else:
                assert np.array_equal(a, b), tile


@pytest.mark.parametrize("precision", [ndg.FP64, ndg.FP32])
def test_autotune_keeps_the_state_and_the_results(precision):
    zone = meshgen.uniform_zone(16, x_periodic=True, y_periodic=True)
    a = ndg.Mesh2D_t(zone, 6, n_instances=4, precision=precision)
    b = ndg.Mesh2D_t(zone, 6, n_instances=4, precision=precision)
    for m in (a, b):
        m.initial_conditions()
        ndg.Solver2D_t.run(m, 3)
    before = [a.get_field(f) for f in ("p", "u", "v", "k_p")]
    tile, ms = a.autotune(5)
    assert ms > 0 and (tile == 0 or tile in a.tile_candidates()[0])
    for x, f in zip(before, ("p", "u", "v", "k_p")):
        assert np.array_equal(a.get_field(f), x), f
    for m in (a, b):
        ndg.Solver2D_t.run(m, 4)
    tol = 0.0 if tile < ndg.TENSOR_TILE else (1e-12 if precision == ndg.FP64 else 2e-6)
    for f in ("p", "u", "v"):
        x, y = a.get_field(f), b.get_field(f)
        assert np.linalg.norm(x - y) <= tol * np.linalg.norm(y), f


def test_strict_form_keeps_its_tile():
    zone = meshgen.uniform_zone(4, boundary=meshgen.WALL)
    m = ndg.Mesh2D_t(zone, 4, precision=ndg.FP64_STRICT)
    with pytest.raises(ndg.NdgError, match="UNSUPPORTED"):
        m.set_tile(4)
    assert m.autotune(2) == (0, 0.0)
