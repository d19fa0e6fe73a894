"""Run one workload of the library for a few steps, for profilers:

    python -m ndg_cuda_b200.cases stage   --res 256 --order 8 --steps 3 [--fp32] [--tile E]
    python -m ndg_cuda_b200.cases batched --res 64 --order 6 --instances 64 --steps 3 [--fp32]
    python -m ndg_cuda_b200.cases adjoint --res 96 --order 7 --steps 20 --interval 10 [--fp32]
    python -m ndg_cuda_b200.cases mixed   --res 128 --order 4 --rounds 3 --steps 2
    python -m ndg_cuda_b200.cases tiles   --res 256 --order 8 [--fp32]
    python -m ndg_cuda_b200.cases hp      --res 128 --order 4 --steps 600 [--fp32]

`stage`: the reference plane wave on a periodic res x res mesh (RK3 steps).
`batched`: independent radial pulses on one walled mesh, one launch per stage.
`adjoint`: forward solve with receivers and its gradient (recomputation and
adjoint sweep) on a walled mesh with a per-element wave speed.
`mixed`: a jittered periodic mesh whose orders are raised by 2 on a seeded
40% of the elements in each of `rounds` p-adaptations (orders 4 to 10 for
order 4 and 3 rounds), then steps on the mixed-order path.
`tiles`: the plane wave on a periodic res x res mesh; every candidate tile
of the stage kernel (SIMT and tensor-core codes) and the default, timed by
CUDA events (best of the second and third RK stages, two rounds, 20 launches
each); one line per tile in µs per launch.
`hp`: the hp-adaptive refining run (walled res x res mesh, interior nodes
jittered by 0.1 h with seed 7, orders up to 12, two split levels, the
Legendre-decay estimate and adapt every 20 steps at threshold 1e-9, two
crossing pulses) for `steps` steps; then the final mesh's stage time by
CUDA events on a stream of its own, and 3 steps inside a profiler range
(cudaProfilerStart/Stop: `ncu --profile-from-start off` captures only them).
Inputs are the seeded synthetic ones of ndg_cuda_b200.workloads.
"""
from __future__ import annotations

import argparse

import numpy as np

from . import FP32, FP64, Adjoint2D_t, Mesh2D_t, Solver2D_t, meshgen, workloads


def _zone(res: int, **kw) -> dict:
    order = "hilbert" if res > 0 and not (res & (res - 1)) else "rowmajor"
    return meshgen.uniform_zone(res, order=order, **kw)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("case", choices=["stage", "batched", "adjoint", "mixed", "tiles", "hp"])
    ap.add_argument("--res", type=int, default=64)
    ap.add_argument("--order", type=int, default=6)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--instances", type=int, default=1)
    ap.add_argument("--interval", type=int, default=0, help="adjoint checkpoint interval (0: one interval)")
    ap.add_argument("--rounds", type=int, default=3, help="p-adaptation rounds of the mixed case")
    ap.add_argument("--tile", type=int, default=0, help="elements per CTA of the stage kernel (0: default)")
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--launch", type=int, default=0, choices=[0, 1, 2],
                    help="mixed case: 0 one launch per order group, 1 one queue launch per stage, "
                    "2 order groups split into side fluxes and element tiles")
    ap.add_argument("--time", type=int, default=0, help="mixed case: then time this many steps (wall clock after a synchronise)")
    args = ap.parse_args(argv)
    prec = FP32 if args.fp32 else FP64
    if args.case == "stage":
        mesh = Mesh2D_t(_zone(args.res, x_periodic=True, y_periodic=True), args.order, precision=prec)
        if args.tile:
            mesh.set_tile(args.tile)
        mesh.initial_conditions()
        Solver2D_t.run(mesh, args.steps)
        print("p[0] =", mesh.get_field("p")[0])
    elif args.case == "batched":
        zone = _zone(args.res, boundary=meshgen.WALL)
        rng = np.random.default_rng(64)
        centres = rng.uniform(-0.8, 0.8, size=(args.instances, 2))
        p0 = np.concatenate([workloads.gaussian_pulse(zone, args.order, sigma=0.05, centre=c) for c in centres])
        mesh = Mesh2D_t(zone, args.order, n_instances=args.instances, precision=prec)
        if args.tile:
            mesh.set_tile(args.tile)
        mesh.set_field("p", p0)
        Solver2D_t.run(mesh, args.steps)
        print("p[0] =", mesh.get_field("p")[0])
    elif args.case == "tiles":
        mesh = Mesh2D_t(_zone(args.res, x_periodic=True, y_periodic=True), args.order, precision=prec)
        mesh.initial_conditions()
        cand, _ = mesh.tile_candidates()
        best: dict[int, float] = {}
        for _ in range(2):
            for t in [0] + cand:
                mesh.set_tile(t)
                Solver2D_t.run(mesh, 1)
                ms = min(mesh.time_stage(1, 20), mesh.time_stage(2, 20))
                best[t] = min(best.get(t, ms), ms)
        for t, ms in best.items():
            print(f"tile {t:4d}: {1e3 * ms:8.1f} us per launch")
    elif args.case == "mixed":
        zone = _zone(args.res, x_periodic=True, y_periodic=True, jitter=0.1, seed=1)
        mesh = Mesh2D_t(zone, args.order, maximum_N=args.order + 2 * args.rounds, precision=prec)
        mesh.initial_conditions()
        rng = np.random.default_rng(0)
        for _ in range(args.rounds):
            K = mesh.n_elements_
            mesh.adapt((rng.random(K) < 0.4).astype(np.int32), np.full(K, 2.0))
        mesh.set_mixed_launch(args.launch)
        Solver2D_t.run(mesh, args.steps)
        print("p[0] =", mesh.get_field("p")[0])
        if args.time:
            import time
            for _ in range(2):
                mesh.synchronize()
                t0 = time.perf_counter()
                Solver2D_t.run(mesh, args.time)
                mesh.synchronize()
                print(f"launch mode {args.launch}: {1e3 * (time.perf_counter() - t0) / args.time:.4f} ms per RK3 step")
    elif args.case == "hp":
        import torch
        zone = meshgen.uniform_zone(args.res, boundary=meshgen.WALL, jitter=0.1, seed=7)
        stream = torch.cuda.Stream()
        mesh = Mesh2D_t(zone, args.order, maximum_N=12, max_split_level=2, tolerance_min=1e-9, tolerance_max=1e-14, cfl=0.5,
                        stream=stream.cuda_stream, precision=prec)
        k1, k2 = np.array([1.0, 1.0]) / np.sqrt(2), np.array([-1.0, 1.0]) / np.sqrt(2)
        pa = workloads.gaussian_pulse(zone, args.order, sigma=0.1, centre=(-0.4, -0.4))
        pb = workloads.gaussian_pulse(zone, args.order, sigma=0.1, centre=(0.4, -0.4))
        mesh.set_field("p", pa + pb)
        mesh.set_field("u", k1[0] * pa + k2[0] * pb)
        mesh.set_field("v", k1[1] * pa + k2[1] * pb)
        for _ in range(args.steps // 20):
            Solver2D_t.run(mesh, 20)
            mesh.estimate_error()
            e = mesh.error()
            mesh.adapt(e["refine"], e["p_sigma"])
        N = mesh.elements()["N"][:mesh.n_elements_]
        print("final mesh:", mesh.n_elements_, "elements, orders", {int(k): int(c) for k, c in zip(*np.unique(N, return_counts=True))})
        Solver2D_t.run(mesh, 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(2):
            e0.record(stream)
            Solver2D_t.run(mesh, 20)
            e1.record(stream)
            torch.cuda.synchronize()
            print(f"final mesh: {1e3 * e0.elapsed_time(e1) / 60:.1f} us per RK stage")
        torch.cuda.profiler.start()
        Solver2D_t.run(mesh, 3)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
    else:
        zone = _zone(args.res, boundary=meshgen.WALL)
        c = workloads.speed_field(zone, seed=0)
        mesh = Mesh2D_t(zone, args.order)
        adj = Adjoint2D_t(mesh, workloads.circle_receivers(16, 0.7), speed=c, precision=prec)
        p0 = workloads.gaussian_pulse(zone, args.order, sigma=0.1, centre=(0.45, 0.0))
        dt = adj.delta_t(0.5)
        J, _ = adj.forward(p0, dt, args.steps, checkpoint_interval=args.interval)
        g = adj.backward()
        print("J =", J, "|grad c| =", float(np.linalg.norm(g["c"])))


if __name__ == "__main__":
    main()
