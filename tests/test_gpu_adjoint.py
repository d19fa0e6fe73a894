"""The discrete adjoint kernels (ndg_adjoint_*) against the CPU FP64 adjoint
of the oracle, the transpose (dot-product) test, central finite
differences and the torch.autograd wrapper.

Tolerances: the GPU contracts to FMAs and the oracle does not, so the
operator agrees to 1e-12 relative L2 and gradients after tens of steps to
1e-10; the dot-product tests hold to 1e-12 relative; finite differences to
1e-7 (p0, where J is quadratic) and 1e-5 (c).
"""
from __future__ import annotations

import numpy as np
import pytest

import ndg_cuda_b200 as ndg
from tests import adjoint_setup as A
from tests import meshgen

pytestmark = pytest.mark.gpu

MESHES = {
    "periodic": dict(x_periodic=True, y_periodic=True),
    "walls": dict(boundary=meshgen.WALL),
    "jittered_outflow": dict(boundary=meshgen.OUTFLOW, jitter=0.1, seed=3),
    "symmetry_x_periodic": dict(x_periodic=True, boundary=meshgen.SYMMETRY),
}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


def _pair(kind, res, N, seed=1, receivers=None):
    zone = meshgen.uniform_zone(res, **MESHES[kind])
    c = A.speed_field(zone, seed=seed)
    xy = np.zeros((0, 2)) if receivers is None else receivers
    mesh = ndg.Mesh2D_t(zone, N)
    adj = ndg.Adjoint2D_t(mesh, xy, speed=c)
    o, el, w = A.oracle_problem(zone, N, c, xy)
    return zone, c, mesh, adj, o, el, w


@pytest.mark.parametrize("N", [3, 7])
@pytest.mark.parametrize("kind", list(MESHES))
def test_operator_and_transpose_vs_oracle(kind, N):
    zone, c, mesh, adj, o, _, _ = _pair(kind, 8, N)
    rng = np.random.default_rng(11)
    n = 3 * mesh.field_size
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    Lx, LTy, dc = adj.operator(x, y)
    assert rel_l2(Lx, o.operator(x)) < 1e-12
    LTy_o, dc_o = o.operator_transpose(x, y)
    assert rel_l2(LTy, LTy_o) < 1e-12
    assert rel_l2(dc, dc_o) < 1e-12
    # the transpose (dot-product) test on the GPU's own operators
    assert _rel(float(Lx @ y), float(x @ LTy)) < 1e-12 * np.linalg.norm(Lx) * np.linalg.norm(y) / abs(float(Lx @ y))


def test_unit_speed_operator_is_the_stage_derivative():
    """With c = 1 the variable-speed operator is the reference's: its L x is
    the time derivative G of the library's FP64 stage on the same state."""
    zone = meshgen.uniform_zone(8, boundary=meshgen.WALL)
    mesh = ndg.Mesh2D_t(zone, 5, keep_derivative=True)
    adj = ndg.Adjoint2D_t(mesh)
    rng = np.random.default_rng(2)
    x = rng.standard_normal(3 * mesh.field_size)
    Lx, _, _ = adj.operator(x, x)
    fs = mesh.field_size
    for i, f in enumerate(("p", "u", "v")):
        mesh.set_field(f, x[i * fs:(i + 1) * fs])
    ndg.Solver2D_t.stage(mesh, 0, 0.0, 0.0)
    for i, f in enumerate(("G_p", "G_u", "G_v")):
        assert rel_l2(Lx[i * fs:(i + 1) * fs], mesh.get_field(f)) < 1e-13, f


@pytest.mark.parametrize("interval", [0, 1, 7])
@pytest.mark.parametrize("kind", ["walls", "periodic", "jittered_outflow"])
def test_gradient_vs_cpu_adjoint(kind, interval):
    N, steps = 4, 24
    zone, c, mesh, adj, o, el, w = _pair(kind, 8, N, seed=4, receivers=A.circle_receivers(12, 0.6))
    p0 = A.gaussian_pulse(zone, N, sigma=0.25)
    rng = np.random.default_rng(3)
    u0 = 0.1 * rng.standard_normal(p0.size)
    dt = adj.delta_t(0.5)
    assert _rel(dt, A.cfl_dt(zone, N, c)) < 1e-14
    target = rng.standard_normal((steps + 1, el.size)) * 0.1
    J, samples = adj.forward(p0, dt, steps, targets=target, u0=u0, checkpoint_interval=interval)
    g = adj.backward()
    ref = o.adjoint_solve(p0, dt, steps, el, w, targets=target, u0=u0)
    assert rel_l2(samples, ref["samples"]) < 1e-12
    assert _rel(J, ref["J"]) < 1e-12
    for k in ("p0", "u0", "v0", "c"):
        assert rel_l2(g[k], ref[k]) < 1e-10, (k, rel_l2(g[k], ref[k]))


def test_checkpoint_interval_does_not_change_the_gradient():
    N, steps = 4, 20
    zone, c, mesh, adj, o, el, w = _pair("walls", 8, N, seed=5, receivers=A.circle_receivers(8, 0.5))
    p0 = A.gaussian_pulse(zone, N, sigma=0.2)
    dt = adj.delta_t(0.5)
    out = []
    for interval in (0, 1, 3, 20):
        adj.forward(p0, dt, steps, checkpoint_interval=interval)
        out.append(adj.backward())
    for g in out[1:]:
        for k in g:
            assert np.array_equal(g[k], out[0][k]), k


def test_full_map_dot_product():
    """F: p0 -> samples (u0 = v0 = 0) against its adjoint F^T r (p0 = 0,
    targets -r/dt), on the GPU."""
    N, steps = 5, 30
    zone, c, mesh, adj, o, el, w = _pair("symmetry_x_periodic", 8, N, seed=6, receivers=A.circle_receivers(16, 0.7))
    dt = adj.delta_t(0.5)
    rng = np.random.default_rng(8)
    x = rng.standard_normal(mesh.field_size)
    _, Fx = adj.forward(x, dt, steps, checkpoint_interval=8)
    r = rng.standard_normal((steps + 1, el.size))
    r[0] = 0.0
    adj.forward(np.zeros_like(x), dt, steps, targets=-r / dt, checkpoint_interval=8)
    g = adj.backward()
    lhs, rhs = float((Fx[1:] * r[1:]).sum()), float(x @ g["p0"])
    assert _rel(lhs, rhs) < 1e-12


def test_gradient_matches_central_differences():
    N, steps = 7, 40
    zone, c, mesh, adj, o, el, w = _pair("walls", 16, N, seed=7, receivers=A.circle_receivers(16, 0.7))
    p0 = A.gaussian_pulse(zone, N, sigma=0.1)
    dt = adj.delta_t(0.5)
    # targets from a run with a perturbed speed
    adj.set_speed(c * (1 + 0.05 * np.cos(2 * A.element_centres(zone)[:, 1])))
    _, target = adj.forward(p0, dt, steps)
    adj.set_speed(c)
    J, _ = adj.forward(p0, dt, steps, targets=target, checkpoint_interval=10)
    g = adj.backward()
    rng = np.random.default_rng(4)
    dp = rng.standard_normal(p0.size)
    eps = 1e-4
    Jp, _ = adj.forward(p0 + eps * dp, dt, steps, targets=target)
    Jm, _ = adj.forward(p0 - eps * dp, dt, steps, targets=target)
    assert _rel((Jp - Jm) / (2 * eps), float(g["p0"] @ dp)) < 1e-7
    dcv = rng.standard_normal(c.size)
    eps = 1e-6
    adj.set_speed(c + eps * dcv)
    Jp, _ = adj.forward(p0, dt, steps, targets=target)
    adj.set_speed(c - eps * dcv)
    Jm, _ = adj.forward(p0, dt, steps, targets=target)
    assert _rel((Jp - Jm) / (2 * eps), float(g["c"] @ dcv)) < 1e-5


def test_torch_autograd_wrapper():
    import torch
    from ndg_cuda_b200.autograd import receiver_misfit
    N, steps = 2, 6
    zone = meshgen.uniform_zone(4, x_periodic=True, y_periodic=True)
    c0 = A.speed_field(zone, seed=3)
    mesh = ndg.Mesh2D_t(zone, N)
    adj = ndg.Adjoint2D_t(mesh, A.circle_receivers(4, 0.5), speed=c0)
    dt = adj.delta_t(0.4)
    target = np.random.default_rng(1).standard_normal((steps + 1, 4)) * 0.1
    p = torch.tensor(A.gaussian_pulse(zone, N, sigma=0.4), dtype=torch.float64, requires_grad=True)
    c = torch.tensor(c0, dtype=torch.float64, requires_grad=True)

    def f(p_, c_):
        return receiver_misfit(adj, p_, c_, dt, steps, targets=target, checkpoint_interval=4)

    J = f(p, c)
    J.backward()
    g = (p.grad.clone(), c.grad.clone())
    adj.set_speed(c0)
    adj.forward(p.detach().numpy(), dt, steps, targets=target)
    direct = adj.backward()
    assert np.array_equal(g[0].numpy(), direct["p0"]) and np.array_equal(g[1].numpy(), direct["c"])
    assert torch.autograd.gradcheck(f, (p, c), eps=1e-6, atol=1e-9, rtol=1e-5)


def test_rejections():
    zone = meshgen.uniform_zone(4, boundary=meshgen.INFLOW)
    mesh = ndg.Mesh2D_t(zone, 3)
    with pytest.raises(ndg.NdgError, match="UNSUPPORTED"):
        ndg.Adjoint2D_t(mesh)
    zone = meshgen.uniform_zone(4, boundary=meshgen.WALL)
    mesh = ndg.Mesh2D_t(zone, 3, maximum_N=5)
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        ndg.Adjoint2D_t(mesh, np.array([[2.0, 0.0]]))
    adj = ndg.Adjoint2D_t(mesh, np.array([[0.1, 0.2]]))
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        adj.set_speed(np.zeros(mesh.n_elements_))
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        adj.backward()  # no forward yet
    K = mesh.n_elements_
    mesh.adapt(np.ones(K, np.int32), np.full(K, 2.0))  # p-refinement: the mesh changes
    with pytest.raises(ndg.NdgError, match="INVALID_ARG"):
        adj.forward(np.zeros(adj.field_size), 0.01, 2)


# FP32 form: the operator's arithmetic in FP32 (states, RK updates and
# gradient accumulation in FP64). Its gradient is compared with the FP64
# references: the oracle's CPU adjoint and central differences of the FP64
# forward, at FP32 accuracy.
@pytest.mark.parametrize("kind", ["walls", "periodic", "jittered_outflow"])
def test_fp32_operator_and_transpose(kind):
    zone = meshgen.uniform_zone(8, **MESHES[kind])
    c = A.speed_field(zone, seed=1)
    mesh = ndg.Mesh2D_t(zone, 6)
    adj = ndg.Adjoint2D_t(mesh, speed=c, precision=ndg.FP32)
    o, _, _ = A.oracle_problem(zone, 6, c, np.zeros((0, 2)))
    rng = np.random.default_rng(12)
    n = 3 * mesh.field_size
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    Lx, LTy, dc = adj.operator(x, y)
    LTy_o, dc_o = o.operator_transpose(x, y)
    assert rel_l2(Lx, o.operator(x)) < 1e-6
    assert rel_l2(LTy, LTy_o) < 1e-6
    assert rel_l2(dc, dc_o) < 1e-5
    assert abs(float(Lx @ y) - float(x @ LTy)) < 1e-6 * np.linalg.norm(Lx) * np.linalg.norm(y)


@pytest.mark.parametrize("kind", ["walls", "periodic"])
def test_fp32_gradient_vs_cpu_fp64_adjoint_and_differences(kind):
    N, steps = 5, 40
    zone = meshgen.uniform_zone(16, **MESHES[kind])
    c = A.speed_field(zone, seed=8)
    xy = A.circle_receivers(16, 0.7)
    mesh = ndg.Mesh2D_t(zone, N)
    a64 = ndg.Adjoint2D_t(mesh, xy, speed=c)
    a32 = ndg.Adjoint2D_t(mesh, xy, speed=c, precision=ndg.FP32)
    o, el, w = A.oracle_problem(zone, N, c, xy)
    p0 = A.gaussian_pulse(zone, N, sigma=0.15, centre=(0.4, 0.1))
    dt = a64.delta_t(0.5)
    a64.set_speed(c * (1 + 0.05 * np.sin(3 * A.element_centres(zone)[:, 0])))
    _, target = a64.forward(p0, dt, steps)
    a64.set_speed(c)
    J32, s32 = a32.forward(p0, dt, steps, targets=target, checkpoint_interval=9)
    g32 = a32.backward()
    ref = o.adjoint_solve(p0, dt, steps, el, w, targets=target)
    assert rel_l2(s32, ref["samples"]) < 1e-6
    assert abs(J32 - ref["J"]) < 1e-4 * ref["J"]
    for k in ("p0", "c"):
        assert rel_l2(g32[k], ref[k]) < 1e-4, (k, rel_l2(g32[k], ref[k]))
    # central differences of the FP64 forward along random directions
    rng = np.random.default_rng(6)
    dp = rng.standard_normal(p0.size)
    eps = 1e-4
    Jp, _ = a64.forward(p0 + eps * dp, dt, steps, targets=target)
    Jm, _ = a64.forward(p0 - eps * dp, dt, steps, targets=target)
    assert _rel((Jp - Jm) / (2 * eps), float(g32["p0"] @ dp)) < 1e-4
    dcv = rng.standard_normal(c.size)
    eps = 1e-6
    a64.set_speed(c + eps * dcv)
    Jp, _ = a64.forward(p0, dt, steps, targets=target)
    a64.set_speed(c - eps * dcv)
    Jm, _ = a64.forward(p0, dt, steps, targets=target)
    assert _rel((Jp - Jm) / (2 * eps), float(g32["c"] @ dcv)) < 1e-4
