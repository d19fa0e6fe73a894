"""ndg_delta_t_from_device (the CFL step from caller-owned device arrays,
computed without allocating) against ndg_get_delta_t, through the C ABI.

The step is a minimum of correctly rounded quotients, so the two entry points
must agree exactly (tolerance 0). Each case calls the new entry point twice
in a row: the second call reuses the shared scratch array that the first one
left behind.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import textwrap

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


def test_allocates_no_device_memory():
    """The entry point's defining property: free device memory (cudaMemGetInfo,
    which also sees allocations outside torch's allocator) is the same before
    and after a batch of calls, once the first call has loaded the kernels."""
    mesh = ndg.Mesh2D_t(meshgen.uniform_zone(64, x_periodic=True, y_periodic=True, jitter=0.1, seed=2), 5, cfl=0.4)
    want = ndg.Solver2D_t.get_delta_t(mesh)
    el = mesh.elements()
    K = mesh.n_elements_
    dxy = torch.tensor(el["delta_xy_min"][:K], dtype=torch.float64, device="cuda")
    elem_N = torch.tensor(el["N"][:K], dtype=torch.int32, device="cuda")
    mesh.close()
    st, got = _call(dxy, elem_N, K, 0.4)  # warm-up: module load
    assert st == 0 and got == want
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(50):
        st, got = _call(dxy, elem_N, K, 0.4)
        assert st == 0 and got == want
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


_RESET_SCRIPT = textwrap.dedent("""
    import ctypes as C, glob, os, sys
    import numpy as np
    sys.path.insert(0, os.environ["NDG_ROOT"])
    import ndg_cuda_b200 as ndg
    lib = ndg.lib()
    cands = sorted(glob.glob("/usr/local/cuda/lib64/libcudart.so*"))
    rt = C.CDLL(cands[0])
    rt.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    rt.cudaFree.argtypes = [C.c_void_p]
    K = 3000
    rng = np.random.default_rng(5)
    dxy = rng.uniform(1e-3, 2e-2, K)
    N = rng.integers(1, 13, K).astype(np.int32)
    want = float((0.5 * dxy / (N.astype(np.float64) * N)).min())

    def one_call():
        assert rt.cudaSetDevice(0) == 0
        a, b = C.c_void_p(), C.c_void_p()
        assert rt.cudaMalloc(C.byref(a), K * 8) == 0 and rt.cudaMalloc(C.byref(b), K * 4) == 0
        assert rt.cudaMemcpy(a, dxy.ctypes.data, K * 8, 1) == 0 and rt.cudaMemcpy(b, N.ctypes.data, K * 4, 1) == 0
        out = C.c_double(-1.0)
        st = lib.ndg_delta_t_from_device(a, b, K, 0.5, None, C.byref(out))
        msg = lib.ndg_last_error()
        rt.cudaFree(a)
        rt.cudaFree(b)
        return st, out.value, msg

    st, got, msg = one_call()
    assert st == 0 and got == want, (st, got, msg)
    assert rt.cudaDeviceReset() == 0
    st, got, msg = one_call()
    print("after-reset", st, got == want, msg)
""")


def test_call_after_device_reset():
    """A call, a reset of the device's primary context by another CUDA runtime
    in the same process, and a second call: the second call must not reuse a
    device address from the first context. It either returns the right step
    (the library's runtime rebuilt its context) or reports a CUDA error
    status; it never launches on a stale address. Runs in a fresh process so
    the reset touches no other test's state."""
    env = dict(os.environ, NDG_ROOT=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    res = subprocess.run([sys.executable, "-c", _RESET_SCRIPT], env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    line = [ln for ln in res.stdout.splitlines() if ln.startswith("after-reset")][-1].split(" ", 3)
    st, ok = int(line[1]), line[2] == "True"
    assert (st == 0 and ok) or st == 3, line  # NDG_OK with the right step, or NDG_ERR_CUDA
