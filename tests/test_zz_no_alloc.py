"""ndg_delta_t_from_device (the CFL step from caller-owned device arrays,
computed without allocating) against ndg_get_delta_t, through the C ABI.

The step is a minimum of correctly rounded quotients, so the two entry points
must agree exactly (tolerance 0). Each case calls the new entry point twice
in a row: the second call reuses the shared scratch array that the first one
left behind.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

import ndg_cuda_b200 as ndg
from tests import meshgen

pytestmark = pytest.mark.gpu

MAX_ELEMENTS = 4_194_304


def _call(dxy: torch.Tensor, N: torch.Tensor, n: int, cfl: float) -> tuple[int, float]:
    out = C.c_double(-1.0)
    stream = torch.cuda.current_stream().cuda_stream
    st = ndg.lib().ndg_delta_t_from_device(dxy.data_ptr(), N.data_ptr(), n, cfl, stream or None, C.byref(out))
    return st, out.value


@pytest.mark.parametrize("res, N, cfl, kw", [
    (8, 6, 0.5, dict(x_periodic=True, boundary=meshgen.WALL)),
    (33, 4, 0.3, dict(order="rowmajor", jitter=0.2, seed=3)),         # 1089 elements: a ragged second block
    (64, 8, 0.5, dict(x_periodic=True, y_periodic=True, jitter=0.1, seed=1)),
    (256, 3, 0.7, dict(x_periodic=True, y_periodic=True, jitter=0.25, seed=7)),
])
def test_matches_get_delta_t_twice(res, N, cfl, kw):
    mesh = ndg.Mesh2D_t(meshgen.uniform_zone(res, **kw), N, cfl=cfl)
    want = ndg.Solver2D_t.get_delta_t(mesh)
    el = mesh.elements()
    K = mesh.n_elements_
    dxy = torch.tensor(el["delta_xy_min"][:K], dtype=torch.float64, device="cuda")
    elem_N = torch.tensor(el["N"][:K], dtype=torch.int32, device="cuda")
    for _ in range(2):
        st, got = _call(dxy, elem_N, K, cfl)
        assert st == 0, ndg.lib().ndg_last_error()
        assert got == want
    mesh.close()


def test_largest_size_and_rejection():
    g = torch.Generator(device="cpu").manual_seed(11)
    dxy = (torch.rand(MAX_ELEMENTS, generator=g, dtype=torch.float64) * 0.01 + 1e-4).cuda()
    elem_N = torch.randint(1, 17, (MAX_ELEMENTS,), generator=g, dtype=torch.int32).cuda()
    cfl = 0.45
    # Products and quotients of doubles are correctly rounded in torch too.
    want = float(((cfl * dxy) / (elem_N.double() * elem_N.double())).min())
    for _ in range(2):
        st, got = _call(dxy, elem_N, MAX_ELEMENTS, cfl)
        assert st == 0, ndg.lib().ndg_last_error()
        assert got == want
    st, got = _call(dxy, elem_N, MAX_ELEMENTS + 1, cfl)
    assert st == 1 and got == -1.0
    assert b"scratch limit" in ndg.lib().ndg_last_error()
    st, _ = _call(dxy, elem_N, 0, cfl)
    assert st == 1
    host = np.ones(16)
    out = C.c_double()
    st = ndg.lib().ndg_delta_t_from_device(host.ctypes.data, elem_N.data_ptr(), 16, cfl, None, C.byref(out))
    assert st == 1 and b"not device-accessible" in ndg.lib().ndg_last_error()
