"""Stage kernels whose two contraction passes (the Dhat products of
compute_dg_wave_derivative, src/solvers/Solver2D_t.cpp:66-136) run on the
tensor cores, against the oracle.

FP64 tiles use DMMA (m16n8k4): their products are exact FP64 products summed
in the tensor cores' order, so they are held to the FP64 form's 1e-12
relative L2 against the reference's CPU path. FP32 tiles use 3xTF32 (m16n8k8,
high and low TF32 parts, FP32 accumulation) and are held to the FP32 form's
1e-6. Cases: every tensor-core tile of orders 6 to 16, periodic, walled and
outflow meshes, an odd element count (a ragged last tile) and three
instances.
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


def _tensor_tiles(mesh):
    return [t for t in mesh.tile_candidates()[0] if t >= ndg.TENSOR_TILE]


@pytest.mark.parametrize("precision", [ndg.FP64, ndg.FP32])
@pytest.mark.parametrize("N", [6, 7, 8, 9, 12, 16])
@pytest.mark.parametrize("kind", ["periodic", "wall", "outflow_odd"])
def test_tensor_tiles_against_oracle(N, kind, precision):
    kw = {"periodic": dict(x_periodic=True, y_periodic=True), "wall": dict(x_periodic=True, boundary=meshgen.WALL),
          "outflow_odd": dict(order="rowmajor", boundary=meshgen.OUTFLOW)}[kind]
    res = 7 if kind == "outflow_odd" else 8
    zone = meshgen.uniform_zone(res, **kw)
    o = OracleSolver(zone, N)
    o.initial_conditions()
    ic = {f: o.field(f) for f in ("p", "u", "v")}
    o.run(10)
    want = {f: o.field(f) for f in ("p", "u", "v")}
    m = ndg.Mesh2D_t(zone, N, precision=precision)
    tiles = _tensor_tiles(m)
    if precision == ndg.FP64:
        assert tiles, "no tensor-core tile for this order"
    tol = 1e-12 if precision == ndg.FP64 else 1e-6
    for tile in tiles:
        m.set_tile(tile)
        for f in ("p", "u", "v"):
            m.set_field(f, ic[f])
        for f in ("k_p", "k_u", "k_v"):
            m.set_field(f, np.zeros_like(ic["p"]))
        ndg.Solver2D_t.run(m, 10)
        for f in ("p", "u", "v"):
            err = rel_l2(m.get_field(f), want[f])
            assert err < tol, (tile, f, err)
    m.close()


@pytest.mark.parametrize("precision", [ndg.FP64, ndg.FP32])
def test_tensor_tiles_with_instances(precision):
    """Three instances with different pulses: each instance's fields equal
    those of a one-instance run within the form's tolerance."""
    from ndg_cuda_b200 import workloads as A
    zone = meshgen.uniform_zone(8, boundary=meshgen.WALL)
    N = 8
    rng = np.random.default_rng(3)
    pulses = [A.gaussian_pulse(zone, N, sigma=0.2, centre=rng.uniform(-0.5, 0.5, 2)) for _ in range(3)]
    batch = ndg.Mesh2D_t(zone, N, n_instances=3, precision=precision)
    single = ndg.Mesh2D_t(zone, N, precision=ndg.FP64_STRICT)
    tol = 1e-12 if precision == ndg.FP64 else 1e-6
    for tile in _tensor_tiles(batch):
        batch.set_tile(tile)
        batch.set_field("p", np.concatenate(pulses))
        for f in ("u", "v", "k_p", "k_u", "k_v"):
            batch.set_field(f, np.zeros(3 * pulses[0].size))
        ndg.Solver2D_t.run(batch, 8)
        got = batch.get_field("p").reshape(3, -1)
        for i, p0 in enumerate(pulses):
            single.set_field("p", p0)
            for f in ("u", "v", "k_p", "k_u", "k_v"):
                single.set_field(f, np.zeros_like(p0))
            ndg.Solver2D_t.run(single, 8)
            assert rel_l2(got[i], single.get_field("p")) < tol, (tile, i)
    batch.close()
    single.close()
