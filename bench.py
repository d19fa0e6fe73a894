#!/usr/bin/env python
"""Benchmark of the DG wave-equation RK3 step on B200 (one JSON line on rank 0).

Workload (the reference's 256 x 256, N = 8 configuration): uniform periodic
quad mesh of [-1, 1]^2, Legendre-Gauss N = 8, the reference plane-wave
initial condition, CFL 0.5, FP64. One benchmark step is one low-storage RK3
time step (three stages) over the whole mesh.

Metric: DOF-stage updates/s = DOF x 3 x steps / seconds, DOF = 3 K (N+1)^2
(p, u, v). `value` is device-resident (inputs already in HBM); `e2e` is the
same metric through the C ABI with host buffers: every e2e step uploads the
state from pinned host memory, runs the configuration's 2000 RK3 steps and
downloads the state. The working set (q, RK register, trace buffers:
~370 MB) is larger than the 126 MB L2, so no L2 flush is inserted.

`--impl reference` times the reference's own CPU path (oracle/_ref) on the
host cores on the same configuration, a bounded number of steps: one
independent replica per core (its stepping is single-threaded), rates
summed.

Multi-GPU (torchrun): the path runs as independent replicas, one per GPU
(no data-path collective); value sums the ranks' DOF-stages over the
slowest rank's time.
"""
from __future__ import annotations

import argparse
import json

import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RES, ORDER, CFL, CONFIG_STEPS = 256, 8, 0.5, 2000
BYTES_PER_DOF_STAGE = 32  # read + write of q and of the RK register, FP64
# Adjoint workload: 96 x 96 walls, N = 7, 16 receivers, 1000 steps, checkpoints every 50.
ADJ_RES, ADJ_N, ADJ_STEPS, ADJ_INTERVAL, ADJ_RECEIVERS = 96, 7, 1000, 50, 16
# hp-adaptive workload: 128 x 128 jittered walled mesh, N 4 -> 12, 2 split levels, adapt every 20 steps.
HP_RES, HP_N0, HP_NMAX, HP_SPLITS, HP_INTERVAL, HP_STEPS = 128, 4, 12, 2, 20, 3000
# Batched workload: 64 instances on one 64 x 64 walled mesh, N = 6, 1000 steps.
BATCH_RES, BATCH_N, BATCH_INSTANCES, BATCH_STEPS = 64, 6, 64, 1000
# The reference's published order sweep (thesis/Chapter_results/code/plots.py:152-153,
# setup thesis/Chapter_results/results.tex:64-97 and 664-676): a 64 x 64 mesh on a
# unit square, the plane wave with boundaries held to the analytic solution, CFL
# 0.5, 1000 RK3 iterations with an error estimate and adaptation every 100 that
# never refines; ms per iteration on one A100 40 GB and on one AMD Milan 7413 core.
SWEEP_RES, SWEEP_STEPS, SWEEP_INTERVAL = 64, 1000, 100
SWEEP_A100_MS = {4: 2.149, 6: 4.136, 8: 8.075, 10: 12.71, 12: 18.22, 14: 26.06, 16: 33.39}
SWEEP_CPU_CORE_MS = {4: 40.11, 6: 71.50, 8: 108.4, 10: 166.6, 12: 257.5, 14: 349.0, 16: 490.1}
# The reference's published full runs of the same plane wave to t = 2 s with no
# adaptivity (thesis/Chapter_results/code/plots.py:22 and 101-104; setup
# thesis/Chapter_results/results.tex:23-35, 164-171, 323-333): mesh, order,
# published steps, published wall seconds, hardware.
PUBLISHED_RUNS = [(128, 10, 51200, 1136.14, "A100 40 GB"), (32, 10, 12800, 48.36, "A100 40 GB"),
                  (256, 4, 16384, 4036.09, "V100 SXM2 16 GB")]
# adjoint stage: lq and lk read and written, the stage input qs read (FP64);
# forward stage keeping its input: q, k read and written, q written once more
ADJ_BYTES_PER_DOF_STAGE = 40


def workload_zone():
    from ndg_cuda_b200 import meshgen
    return meshgen.uniform_zone(RES, x_periodic=True, y_periodic=True)


def dof_count() -> int:
    return 3 * RES * RES * (ORDER + 1) ** 2


def config(extra: dict | None = None) -> dict:
    c = {"workload": f"dg_wave_rk3_periodic_{RES}x{RES}_N{ORDER}_plane_wave", "mesh": f"{RES}x{RES} uniform periodic quads on [-1,1]^2",
         "order_N": ORDER, "dof": dof_count(), "cfl": CFL, "rk_stages_per_step": 3, "precision_form": "fp64",
         "l2_policy": "working set > L2 (126 MB): q+k 255 MB, traces 113 MB; no flush", "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# Clocks during the timed region.
class ClockSampler:
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100", "-i", str(self.index)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def physical_gpu_index(local: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local < len(ids) and ids[local].isdigit():
            return int(ids[local])
    return local


def measured_hbm_peak() -> tuple[float, str]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(tile: int = 0) -> float | None:
    """DRAM bytes per stage-kernel launch of the tile in use (0: the default)
    from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_traffic.txt")
    key = f"N{ORDER}_res{RES}" + (f"_tile{tile}" if tile else "")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 2 and parts[0] == key:
                    return float(parts[1])
    except (OSError, ValueError):
        pass
    return None


def stage_roofline(mesh, dof: int, peak: float, n_launches: int = 30) -> dict:
    """Event-timed launches of each RK stage's kernel on its own. Stage 0 reads
    no RK register, so it moves 24 B per DOF where stages 1 and 2 move 32; the
    stated convention (32 B per DOF-stage for every stage) is kept for the
    headline, and the bytes each stage actually moves are shown beside it.
    The sum of the three is the stage kernels' share of one RK3 step."""
    per = []
    for m in range(3):
        ms = mesh.time_stage(m, n_launches)
        moved = (24 if m == 0 else 32) * dof
        per.append({"stage": m, "kernel_ms": ms, "bytes_moved": moved, "frac_moved": moved / (ms / 1e3) / 1e9 / peak,
                    "frac_convention": BYTES_PER_DOF_STAGE * dof / (ms / 1e3) / 1e9 / peak})
    total = sum(p["kernel_ms"] for p in per)
    return {"per_stage": per, "sum_ms": total, "mean_ms": total / 3}


# ---------------------------------------------------------------------------
def cpu_reference_rate(budget_s: float, max_steps: int, warmup: int) -> dict:
    """The reference's own CPU path (oracle/_ref/libndgref.so; the plain-C
    oracle when it is absent) on the workload, timed on this host."""
    from oracle import pyoracle
    zone = workload_zone()
    kind = "reference" if pyoracle.ref_available() else "port"
    solver = pyoracle.RefSolver(zone, ORDER, cfl=CFL) if kind == "reference" else pyoracle.OracleSolver(zone, ORDER, cfl=CFL)
    solver.initial_conditions()
    t = 0.0
    for _ in range(warmup):
        t = solver.run(1, t)
    done, start = 0, time.perf_counter()
    while done < max_steps:
        t = solver.run(1, t)
        done += 1
        if time.perf_counter() - start > budget_s:
            break
    elapsed = time.perf_counter() - start
    rate = dof_count() * 3 * done / elapsed
    return {"value": rate, "unit": "DOF-stage updates/s", "cores": 1, "kind": kind, "steps": done, "seconds": elapsed,
            "sample": f"{done} RK3 steps of the {RES}x{RES} N={ORDER} workload on 1 host core (the reference CPU path is single-threaded)"}


def _reference_replica(task) -> dict:
    """One replica of the reference's CPU path, pinned to one host core (runs in a spawned process)."""
    budget, max_steps, warmup, core = task
    try:
        os.sched_setaffinity(0, {core})
    except (AttributeError, OSError):
        pass
    return cpu_reference_rate(budget, max_steps, warmup)


def _available_memory_kb() -> float | None:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return float(line.split()[1])
    except OSError:
        pass
    return None


def config1_leg(local: int, stream) -> dict:
    """The reference's own CPU-runnable case (16 x 16 periodic, N = 4, 200 RK3
    steps of the plane wave): the L2 error against the analytic solution of
    the reference's CPU path (its restatement in the oracle, bit-identical to
    it) and of the device path in every form, from the same initial fields."""
    import numpy as np

    import ndg_cuda_b200 as ndg
    from ndg_cuda_b200 import meshgen
    from oracle.pyoracle import OracleSolver
    zone = meshgen.uniform_zone(16, x_periodic=True, y_periodic=True)
    o = OracleSolver(zone, 4, cfl=CFL)
    o.initial_conditions()
    ic = {f: o.field(f) for f in ("p", "u", "v")}
    t_ref = o.run(200)
    out = {"workload": "dg_wave_rk3_periodic_16x16_N4_plane_wave_200_steps", "time": t_ref,
           "l2_vs_analytic": {"reference_cpu": dict(zip("puv", map(float, o.l2_error(t_ref))))}, "rel_l2_vs_reference": {}}
    import torch
    out["device_rate"] = {}
    for name, prec in (("fp64_strict", ndg.FP64_STRICT), ("fp64", ndg.FP64), ("fp32", ndg.FP32)):
        m = ndg.Mesh2D_t(zone, 4, cfl=CFL, device=local, stream=stream.cuda_stream, precision=prec)
        for f in ("p", "u", "v"):
            m.set_field(f, ic[f])
        t = ndg.Solver2D_t.run(m, 200)
        out["l2_vs_analytic"][name] = dict(zip("puv", map(float, m.l2_error(t))))
        # the configuration's 200 steps timed on the device (CUDA events; the
        # step graphs are built by the run above)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ndg.Solver2D_t.run(m, 200, t)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out["device_rate"][name] = {"ms_200_steps": ms, "value": ndg.dof_count(m) * 3 * 200 / (ms / 1e3), "unit": "DOF-stage updates/s"}
        for f in ("p", "u", "v"):
            m.set_field(f, ic[f])
        ndg.Solver2D_t.run(m, 200)
        out["rel_l2_vs_reference"][name] = {f: float(np.linalg.norm(m.get_field(f) - o.field(f)) / np.linalg.norm(o.field(f)))
                                            for f in ("p", "u", "v")}
        m.close()
    return out


def run_reference_arm(args) -> None:
    """The reference's CPU path on all the host cores it can use: its stepping
    is single-threaded and its MPI domain decomposition is not built here, so
    one independent replica of the workload runs per core (spawned processes,
    each pinned to a core, as many as the host memory holds at about 1.6 GB
    each) and their rates add up. That sum bounds from above what one
    parallel run of the same work could reach."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    budget = float(os.environ.get("NDG_REF_BUDGET_S", "60"))
    cores = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else list(range(os.cpu_count() or 1))
    mem = _available_memory_kb()
    n_rep = len(cores) if mem is None else max(1, min(len(cores), int(mem / 1.6e6)))
    n_rep = int(os.environ.get("NDG_REF_REPLICAS", n_rep))
    warmup = args.warmup
    tasks = [(budget, max(args.steps, 1), warmup, cores[i % len(cores)]) for i in range(n_rep)]
    with mp.get_context("spawn").Pool(n_rep) as pool:
        reps = pool.map(_reference_replica, tasks)
    value = sum(r["value"] for r in reps)
    steps = [r["steps"] for r in reps]
    per_step_s = sorted(r["seconds"] / r["steps"] for r in reps)[len(reps) // 2]
    kind = reps[0]["kind"]
    sample = (f"{n_rep} independent replicas of the {RES}x{RES} N={ORDER} workload, one per host core, "
              f"{min(steps)}-{max(steps)} RK3 steps each (the reference CPU path is single-threaded; replicas stand in "
              f"for its MPI decomposition, which is not built)")
    line = {"impl": "reference", "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage updates/s",
            "n_gpus": args.gpus, "steps": min(steps), "warmup": warmup,
            "ms_per_step": 1e3 * per_step_s, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference plane-wave initial condition)",
            "config": config(),
            "cpu_baseline": {"value": value, "unit": "DOF-stage updates/s", "cores": n_rep, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "DOF-stage updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def hp_run(local: int, stream, tolerance: float, steps: int, precision: int = 0, replay=None) -> dict:
    """One adaptive run: RK3 steps on the device, then the error estimate and
    Mesh2D_t::adapt every HP_INTERVAL steps (the reference loop). With
    `replay` (the flags of an earlier run) the mesh is adapted with those
    flags instead, so that two forms step on the same meshes."""
    import numpy as np
    import torch
    import ndg_cuda_b200 as ndg
    from ndg_cuda_b200 import meshgen
    from ndg_cuda_b200 import workloads as A
    zone = meshgen.uniform_zone(HP_RES, boundary=meshgen.WALL, jitter=0.1, seed=7)
    m = ndg.Mesh2D_t(zone, HP_N0, maximum_N=HP_NMAX, max_split_level=HP_SPLITS, tolerance_min=tolerance, tolerance_max=1e-14,
                     cfl=CFL, device=local, stream=stream.cuda_stream, precision=precision)
    k1, k2 = np.array([1.0, 1.0]) / np.sqrt(2), np.array([-1.0, 1.0]) / np.sqrt(2)
    pa = A.gaussian_pulse(zone, HP_N0, sigma=0.1, centre=(-0.4, -0.4))
    pb = A.gaussian_pulse(zone, HP_N0, sigma=0.1, centre=(0.4, -0.4))
    m.set_field("p", pa + pb)
    m.set_field("u", k1[0] * pa + k2[0] * pb)
    m.set_field("v", k1[1] * pa + k2[1] * pb)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ms = adapt_s = 0.0
    dof_stages = 0
    refined = 0
    flags = []
    launches0 = m.launches()
    wall0 = time.perf_counter()
    for it in range(steps // HP_INTERVAL):
        ndg.Solver2D_t.run(m, 0)  # traces and step graphs of the current mesh, outside the timed region
        e0.record(stream)
        ndg.Solver2D_t.run(m, HP_INTERVAL)
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms += e0.elapsed_time(e1)
        dof_stages += ndg.dof_count(m) * 3 * HP_INTERVAL
        a0 = time.perf_counter()
        if replay is None:
            m.estimate_error()
            e = m.error()
            flags.append((e["refine"], e["p_sigma"]))
        else:
            flags.append(replay[it])
        refined += int(flags[-1][0].sum())
        m.adapt(*flags[-1])
        adapt_s += time.perf_counter() - a0
    wall = time.perf_counter() - wall0
    N = m.elements()["N"][:m.n_elements_]
    split = m.element_state()["split_level"][:m.n_elements_]
    out = {"tolerance_min": tolerance, "steps": steps, "adaptations": steps // HP_INTERVAL, "refine_flags_total": refined,
           "final_elements": m.n_elements_, "final_orders": {str(int(k)): int((N == k).sum()) for k in np.unique(N)},
           "final_split_levels": {str(int(k)): int((split == k).sum()) for k in np.unique(split)},
           "final_dof": ndg.dof_count(m), "device_stepping_ms": step_ms, "value": dof_stages / (step_ms / 1e3),
           "unit": "DOF-stage updates/s", "adapt_wall_s": adapt_s, "wall_s": wall, "gpu_launches": m.launches() - launches0,
           "path": "mixed-order" if len(set(N.tolist())) > 1 or m.n_elements_ != HP_RES * HP_RES else "uniform (nothing refined)",
           "precision": "fp32" if precision == ndg.FP32 else "fp64"}
    fields = {f: m.get_field(f) for f in ("p", "u", "v")}
    m.close()
    return out, flags, fields


def order_sweep_leg(local: int, stream) -> dict:
    """The reference's published order sweep, run the same way here: per
    order, 1000 RK3 steps with an error estimate and an adaptation every 100
    (maximum order and split level held at the start, so that nothing
    refines, as in the published runs). ms per iteration is the host wall
    time of the whole loop (estimates, flag downloads and adaptation calls
    included) over the iterations; the device time of the same loop is
    reported beside it."""
    import torch
    import ndg_cuda_b200 as ndg
    from ndg_cuda_b200 import meshgen
    zone = meshgen.uniform_zone(SWEEP_RES, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, boundary=meshgen.INFLOW)
    orders = {}
    for N in sorted(SWEEP_A100_MS):
        m = ndg.Mesh2D_t(zone, N, maximum_N=N, max_split_level=0, cfl=CFL, device=local, stream=stream.cuda_stream)
        m.initial_conditions()
        tile, _ = m.autotune(10)
        ndg.Solver2D_t.run(m, 5)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        e0.record(stream)
        for _ in range(SWEEP_STEPS // SWEEP_INTERVAL):
            ndg.Solver2D_t.run(m, SWEEP_INTERVAL)
            m.estimate_error()
            m.adapt()
        e1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        ms = 1e3 * wall / SWEEP_STEPS
        dof = ndg.dof_count(m)
        orders[str(N)] = {"ms_per_iteration": ms, "device_ms_per_iteration": e0.elapsed_time(e1) / SWEEP_STEPS,
                          "dof": dof, "value": dof * 3 * SWEEP_STEPS / wall, "unit": "DOF-stage updates/s",
                          "reference_a100_ms": SWEEP_A100_MS[N], "speedup_vs_reference_a100": SWEEP_A100_MS[N] / ms,
                          "reference_cpu_core_ms": SWEEP_CPU_CORE_MS[N], "elements_after": m.n_elements_,
                          "tile_elements_per_cta": tile or m.tile_candidates()[1]}
        m.close()
    return {"workload": f"dg_wave_rk3_inflow_{SWEEP_RES}x{SWEEP_RES}_unit_square_plane_wave_N4to16",
            "setup": (f"{SWEEP_RES}x{SWEEP_RES} quads on [0,1]^2, boundaries held to the analytic plane wave, CFL {CFL}, FP64, "
                      f"{SWEEP_STEPS} RK3 steps with an error estimate and adaptation every {SWEEP_INTERVAL} (nothing refines)"),
            "reference_numbers": "published ms per iteration of the reference (thesis plots.py:152-153): one A100 40 GB, one AMD Milan 7413 core",
            "orders": orders}


def published_runs_leg(local: int, stream) -> dict:
    """The reference's published full runs, end to end: the plane wave on a
    unit square with boundaries held to the analytic solution, CFL 0.5, from
    t = 0 to t = 2 s through Solver2D_t.solve (the last step shortened to land
    on t = 2), no adaptivity. Wall time from the initial condition on the
    device to the final state, and the L2 error against the analytic
    solution at t = 2."""
    import torch
    import ndg_cuda_b200 as ndg
    from ndg_cuda_b200 import meshgen
    runs = []
    for res, N, ref_steps, ref_s, hardware in PUBLISHED_RUNS:
        zone = meshgen.uniform_zone(res, x_min=0.0, x_max=1.0, y_min=0.0, y_max=1.0, boundary=meshgen.INFLOW)
        m = ndg.Mesh2D_t(zone, N, cfl=CFL, device=local, stream=stream.cuda_stream)
        m.initial_conditions()
        tile, _ = m.autotune(10)
        solver = ndg.Solver2D_t(CFL, output_times=(2.0,))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        e0.record(stream)
        m.initial_conditions()
        t, steps = solver.solve(m)
        e1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
        dof = ndg.dof_count(m)
        runs.append({"mesh": f"{res}x{res}", "N": N, "dof": dof, "steps": steps, "reference_steps": ref_steps, "time": t,
                     "wall_s": wall, "device_s": e0.elapsed_time(e1) / 1e3, "value": dof * 3 * steps / wall,
                     "unit": "DOF-stage updates/s", "reference_wall_s": ref_s, "reference_hardware": hardware,
                     "speedup_vs_reference": ref_s / wall, "l2_vs_analytic": dict(zip("puv", map(float, m.l2_error(t)))),
                     "tile_elements_per_cta": tile or m.tile_candidates()[1]})
        m.close()
    return {"setup": f"unit square, boundaries held to the analytic plane wave, CFL {CFL}, FP64, t = 0 to 2 s, no adaptivity",
            "reference_numbers": "published wall times of the reference (thesis plots.py:22, 101-104)", "runs": runs}


# Threshold of the refining runs: the configuration's 1e-4 never refines on
# this mesh; at 1e-9 p-refinement fires in the first adaptation and element
# splitting reaches split level 2 by the second.
HP_REFINING_TOL, HP_REFINING_STEPS = 1e-9, 600


def hp_leg(local: int, stream) -> dict:
    import numpy as np
    import ndg_cuda_b200 as ndg
    as_configured, _, _ = hp_run(local, stream, 1e-4, HP_STEPS)
    refining, flags, f64 = hp_run(local, stream, HP_REFINING_TOL, HP_REFINING_STEPS)
    refining32, _, f32 = hp_run(local, stream, HP_REFINING_TOL, HP_REFINING_STEPS, precision=ndg.FP32, replay=flags)
    refining32["rel_l2_vs_fp64"] = {f: float(np.linalg.norm(f32[f] - f64[f]) / max(np.linalg.norm(f64[f]), 1e-300)) for f in f64}
    refining32["note"] = "the same meshes as the FP64 run (its refine flags replayed); FP32 traces, fluxes, mortar and volume arithmetic, FP64 q, k and RK update"
    # Roofline of the mixed-order path: the whole stage (ghost kernel and the
    # order groups' kernels) at the 32 B per DOF-stage of the uniform path's
    # convention, over the run's device stepping time.
    peak, peak_src = measured_hbm_peak()
    for run in (as_configured, refining, refining32):
        achieved = run["value"] * BYTES_PER_DOF_STAGE / 1e9
        run["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                           "peak_source": peak_src, "scope": "whole stage: ghost traces and every order group's kernel, 32 B per DOF-stage"}
    # Parity at the configuration's scale: three adaptation rounds in
    # lockstep with the reference's CPU path (outside every timed region).
    lockstep = hp_lockstep_check(local, stream)
    adapt_cost = adapt_cost_leg(local, stream)
    return {"workload": f"hp_adaptive_wave_rk3_walls_{HP_RES}x{HP_RES}_jitter0.1_N{HP_N0}to{HP_NMAX}",
            "setup": (f"{HP_RES}x{HP_RES} walled quads, interior nodes jittered by U(-0.1h, 0.1h) (seed 7), N {HP_N0} up to {HP_NMAX}, "
                      f"up to {HP_SPLITS} splits, estimate + adapt every {HP_INTERVAL} steps (Legendre decay), two crossing "
                      f"Gaussian pulses sigma 0.1 from (-0.4,-0.4) and (0.4,-0.4) moving along (1,1) and (-1,1), CFL {CFL}, FP64"),
            "as_configured": as_configured,
            "refining": refining,
            "refining_fp32": refining32,
            "launch_structure": ("one CUDA graph per RK3 step; per stage a ghost-trace kernel, then per order group the fused kernel, "
                                 "or, where at least half its elements are conforming, the conforming-element kernel for those and "
                                 "the fused kernel for the rest (an order of at least 2,048 elements with no conforming part "
                                 "runs split: its side fluxes, then the conforming-element kernel over them); "
                                 "the groups forked onto side streams as parallel graph branches"),
            "note": ("at the configuration's threshold 1e-4 the estimate never exceeds it on this mesh (largest error at N=4 "
                     "is 3.4e-6), so nothing refines; the 1e-9 runs exercise p-refinement, splitting to level 2 and the mortar path"),
            "flags_parity": lockstep["flags_parity"],
            "lockstep": lockstep,
            "adapt_cost": adapt_cost}


def adapt_cost_leg(local: int, stream) -> dict:
    """Wall time of one adaptation (Mesh2D_t::adapt: decisions and counts on
    the device, topology rebuild on the host, device plan and field
    transfer) on the hp mesh family at 128 x 128 and 512 x 512: seeded flags
    on 10% of the elements, half of them splitting, three rounds each."""
    import numpy as np
    import ndg_cuda_b200 as ndg
    from ndg_cuda_b200 import meshgen
    out = {}
    for res in (HP_RES, 4 * HP_RES):
        zone = meshgen.uniform_zone(res, boundary=meshgen.WALL, jitter=0.1, seed=7)
        m = ndg.Mesh2D_t(zone, HP_N0, maximum_N=HP_NMAX, max_split_level=HP_SPLITS, cfl=CFL, device=local, stream=stream.cuda_stream)
        m.initial_conditions()
        ndg.Solver2D_t.run(m, 1)
        rng = np.random.default_rng(res)
        rounds = []
        for _ in range(3):
            K = m.n_elements_
            refine = (rng.random(K) < 0.1).astype(np.int32)
            sigma = np.where(rng.random(K) < 0.5, 0.5, 2.0)
            m.synchronize()
            t0 = time.perf_counter()
            m.adapt(refine, sigma)
            m.synchronize()
            rounds.append({"elements_before": K, "elements_after": m.n_elements_, "faces_after": m.n_faces_,
                           "ms": 1e3 * (time.perf_counter() - t0), "phases_ms": m.adapt_timings()})
        out[f"{res}x{res}"] = {"rounds": rounds, "ms_per_adaptation": statistics.median(r["ms"] for r in rounds)}
        m.close()
    return out


def hp_lockstep_check(local: int, stream) -> dict:
    """Refine flags, p/h decisions, topology and fields of the library against
    the reference's own CPU adapt on the hp mesh (tests/hp_lockstep.py), in
    FP64_STRICT and FP64; a summary of every comparison."""
    from oracle import pyoracle
    if not pyoracle.ref_available():
        return {"flags_parity": None, "skipped": "the reference CPU build (oracle/_ref/libndgref.so) is absent"}
    from tests import hp_lockstep
    t0 = time.perf_counter()
    rep = hp_lockstep.run(rounds=3, extra_steps=5, device=local, stream=stream.cuda_stream)
    rounds = [{"round": r["round"], "elements_before": r["elements_before"], "elements_after": r["elements_after"],
               "refine": r["refine"], "p_refine": r["p_refine"], "h_refine": r["h_refine"],
               "orders_after": r["orders_after"], "split_levels_after": r["split_levels_after"],
               "forms": {k: {"refine_flags_equal": v["refine_flags_equal"], "p_h_decisions_equal": v["p_h_decisions_equal"],
                             "topology_mismatches": v["topology_mismatches"],
                             "fields_bitwise": v["fields_after_adapt"]["bitwise"],
                             "fields_max_rel_l2": max(v["fields_after_adapt"]["rel_l2"].values())}
                         for k, v in r["forms"].items()}} for r in rep["rounds"]]
    extra = rep.get("fields_after_extra_steps", {})
    return {"flags_parity": rep["flags_parity"], "tolerance_min": rep["tolerance_min"], "mesh": rep["mesh"],
            "split_levels_reached": rep["split_levels_reached"], "rounds": rounds,
            "after_5_more_steps": {k: {"bitwise": v["bitwise"], "max_rel_l2": max(v["rel_l2"].values())}
                                   for k, v in extra.items() if isinstance(v, dict)},
            "checked": "refine flags and p/h decisions from each side's own estimate, every ndg_mesh_get_* array bitwise, fields bitwise (fp64_strict) / < 1e-12 rel L2 (fp64)",
            "seconds": time.perf_counter() - t0}


def batched_leg(local: int, stream, peak: float, dist) -> dict:
    """Many independent runs on one mesh in one launch per stage (instances
    as the grid's second dimension), the RK3 step as a CUDA graph, the tile
    chosen by the autotuner per form; FP64 against the FP32 form."""
    import numpy as np
    import torch
    import ndg_cuda_b200 as ndg
    from ndg_cuda_b200 import workloads as A
    from ndg_cuda_b200 import meshgen
    zone = meshgen.uniform_zone(BATCH_RES, boundary=meshgen.WALL)
    rng = np.random.default_rng(64)
    centres = rng.uniform(-0.8, 0.8, size=(BATCH_INSTANCES, 2))
    p0 = np.concatenate([A.gaussian_pulse(zone, BATCH_N, sigma=0.05, centre=c) for c in centres])
    zeros = np.zeros_like(p0)
    out = {"workload": f"batched_wave_rk3_walls_{BATCH_RES}x{BATCH_RES}_N{BATCH_N}_{BATCH_INSTANCES}_instances",
           "setup": (f"{BATCH_INSTANCES} independent runs on one {BATCH_RES}x{BATCH_RES} walled mesh, N={BATCH_N}, each a radial "
                     f"Gaussian pressure pulse sigma 0.05 at a seeded uniform centre in [-0.8,0.8]^2 (u = v = 0), "
                     f"{BATCH_STEPS} RK3 steps at CFL {CFL}; one launch per stage for all instances, the step as a CUDA graph")}
    meshes = {}
    for name, prec in (("fp64", ndg.FP64), ("fp32", ndg.FP32)):
        m = ndg.Mesh2D_t(zone, BATCH_N, cfl=CFL, n_instances=BATCH_INSTANCES, device=local, stream=stream.cuda_stream, precision=prec)
        meshes[name] = m

        def reset(m=m):
            m.set_field("p", p0)
            for f in ("u", "v", "k_p", "k_u", "k_v"):
                m.set_field(f, zeros)

        reset()
        tile, tile_ms = m.autotune(20)
        reset()
        ndg.Solver2D_t.run(m, 3)
        reset()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist is not None:
            dist.barrier()
        e0.record(stream)
        ndg.Solver2D_t.run(m, BATCH_STEPS)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if dist is not None:
            dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        ms = float(ms.item())
        dof = ndg.dof_count(m)
        world = dist.get_world_size() if dist is not None else 1
        st = stage_roofline(m, dof, peak, 20)
        stage_ms = st["mean_ms"]
        out[name] = {"value": world * dof * 3 * BATCH_STEPS / (ms / 1e3), "unit": "DOF-stage updates/s", "ms_per_step": ms / BATCH_STEPS,
                     "kernel_ms": stage_ms, "roofline_frac": BYTES_PER_DOF_STAGE * dof / (stage_ms / 1e3) / 1e9 / peak,
                     "per_stage": st["per_stage"], "kernel_ms_per_step": st["sum_ms"],
                     "tile": {"elements_per_cta": tile if tile else m.tile_candidates()[1], "autotuner_choice": "candidate" if tile else "default",
                              "candidates": m.tile_candidates()[0], "tuned_ms_per_launch": tile_ms}}
        out["dof"] = dof
    # FP32 against FP64 after the configuration's steps from the same state
    for m in meshes.values():
        m.set_field("p", p0)
        for f in ("u", "v", "k_p", "k_u", "k_v"):
            m.set_field(f, zeros)
        ndg.Solver2D_t.run(m, BATCH_STEPS)
    err = {}
    for f in ("p", "u", "v"):
        a64, a32 = meshes["fp64"].get_field(f), meshes["fp32"].get_field(f)
        err[f] = float(np.linalg.norm(a32 - a64) / max(np.linalg.norm(a64), 1e-300))
    out["fp32_rel_l2_vs_fp64"] = err
    for m in meshes.values():
        m.close()
    return out


def adjoint_leg(local: int, stream, peak: float, cpu_sample: bool) -> dict:
    """Gradient of a receiver misfit with respect to the initial pressure and a
    per-element wave speed (the library's discrete adjoint): forward solve
    with checkpoints, then recomputation + adjoint sweep, timed on the device
    (CUDA events inside the library) and end to end through the API with
    host buffers."""
    import numpy as np
    import ndg_cuda_b200 as ndg
    from ndg_cuda_b200 import workloads as A
    from ndg_cuda_b200 import meshgen
    zone = meshgen.uniform_zone(ADJ_RES, order="rowmajor", boundary=meshgen.WALL)
    c = A.speed_field(zone, seed=0)
    mesh = ndg.Mesh2D_t(zone, ADJ_N, device=local, stream=stream.cuda_stream)
    adj = ndg.Adjoint2D_t(mesh, A.circle_receivers(ADJ_RECEIVERS, 0.7), speed=c)
    p0 = A.gaussian_pulse(zone, ADJ_N, sigma=0.1, centre=(0.45, 0.0))
    dt = adj.delta_t(CFL)
    # targets: the same run with a perturbed speed
    adj.set_speed(c * (1 + 0.05 * np.sin(4 * A.element_centres(zone)[:, 0])))
    _, target = adj.forward(p0, dt, ADJ_STEPS, checkpoint_interval=ADJ_INTERVAL)
    adj.set_speed(c)
    adj.forward(p0, dt, ADJ_STEPS, targets=target, checkpoint_interval=ADJ_INTERVAL)
    adj.backward()  # warm-up
    reps, fwd, bwd, wall_f, wall_b = 3, [], [], [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        J, _ = adj.forward(p0, dt, ADJ_STEPS, targets=target, checkpoint_interval=ADJ_INTERVAL)
        t1 = time.perf_counter()
        g = adj.backward()
        t2 = time.perf_counter()
        tm = adj.timings()
        fwd.append(tm["forward_ms"])
        bwd.append(tm["backward_ms"])
        wall_f.append(1e3 * (t1 - t0))
        wall_b.append(1e3 * (t2 - t1))
    kernel = {"speed_stage": adj.time_stage(0, 30), "speed_stage_keeping_input": adj.time_stage(1, 30), "adjoint_stage": adj.time_stage(2, 30)}
    dof = 3 * mesh.field_size
    f_ms, b_ms = statistics.median(fwd), statistics.median(bwd)
    roof = {}
    for name, ms in kernel.items():
        bytes_ = (BYTES_PER_DOF_STAGE if name == "speed_stage" else ADJ_BYTES_PER_DOF_STAGE) * dof
        roof[name] = {"achieved_GBs": bytes_ / (ms / 1e3) / 1e9, "frac": bytes_ / (ms / 1e3) / 1e9 / peak,
                      "algorithmic_bytes_per_launch": bytes_}
    out = {"workload": f"adjoint_wave_rk3_walls_{ADJ_RES}x{ADJ_RES}_N{ADJ_N}_{ADJ_STEPS}_steps",
           "setup": (f"{ADJ_RES}x{ADJ_RES} uniform quads with walls, N={ADJ_N}, c = 1 + 0.2 tanh(8 seeded Gaussian bumps, sigma 0.3), "
                     f"{ADJ_RECEIVERS} receivers on a circle r=0.7, Gaussian pressure pulse sigma 0.1 at (0.45, 0), targets from "
                     f"c (1 + 0.05 sin 4x), {ADJ_STEPS} RK3 steps at CFL {CFL}, checkpoints every {ADJ_INTERVAL} steps"),
           "dof": dof, "steps": ADJ_STEPS, "checkpoint_interval": ADJ_INTERVAL, "dtype": "f64",
           "forward_ms": f_ms, "backward_ms": b_ms, "adjoint_over_forward": b_ms / f_ms,
           "forward_dof_stage_per_s": dof * 3 * ADJ_STEPS / (f_ms / 1e3),
           "backward_dof_stage_per_s": dof * 3 * ADJ_STEPS / (b_ms / 1e3),
           "wall_time_per_unit_time_s": {"forward": f_ms / 1e3 / (ADJ_STEPS * dt), "forward_plus_gradient": (f_ms + b_ms) / 1e3 / (ADJ_STEPS * dt)},
           "e2e_forward_ms": statistics.median(wall_f), "e2e_backward_ms": statistics.median(wall_b),
           "e2e_note": "host buffers: p0 and targets uploaded, samples and the four gradients downloaded inside the timed calls",
           "kernel_ms": kernel, "roofline": roof, "launches": {"forward": tm["forward_launches"], "backward": tm["backward_launches"]},
           "misfit": J, "grad_norm": {"p0": float(np.linalg.norm(g["p0"])), "c": float(np.linalg.norm(g["c"]))}}
    # FP32 form of the same gradient (operator arithmetic in FP32)
    a32 = ndg.Adjoint2D_t(mesh, A.circle_receivers(ADJ_RECEIVERS, 0.7), speed=c, precision=ndg.FP32)
    a32.forward(p0, dt, ADJ_STEPS, targets=target, checkpoint_interval=ADJ_INTERVAL)
    a32.backward()  # warm-up
    f32, b32 = [], []
    for _ in range(reps):
        J32, _ = a32.forward(p0, dt, ADJ_STEPS, targets=target, checkpoint_interval=ADJ_INTERVAL)
        g32 = a32.backward()
        t32 = a32.timings()
        f32.append(t32["forward_ms"])
        b32.append(t32["backward_ms"])
    k32 = {"speed_stage": a32.time_stage(0, 30), "adjoint_stage": a32.time_stage(2, 30)}
    rel = {k: float(np.linalg.norm(g32[k] - g[k]) / max(np.linalg.norm(g[k]), 1e-300)) for k in ("p0", "c")}
    out["fp32"] = {"forward_ms": statistics.median(f32), "backward_ms": statistics.median(b32),
                   "adjoint_over_forward": statistics.median(b32) / statistics.median(f32), "kernel_ms": k32,
                   "misfit_rel_diff_vs_fp64": abs(J32 - J) / max(abs(J), 1e-300), "gradient_rel_l2_vs_fp64": rel,
                   "arithmetic": "traces, fluxes, metrics, volume term and their transposes in FP32; states, RK updates, misfit and gradient accumulation in FP64"}
    a32.close()
    if cpu_sample:
        # the oracle's CPU FP64 adjoint on a bounded sample of the same problem
        from tests import adjoint_setup
        o, el, w = adjoint_setup.oracle_problem(zone, ADJ_N, c, A.circle_receivers(ADJ_RECEIVERS, 0.7))
        n_cpu = 4
        t0 = time.perf_counter()
        o.adjoint_solve(p0, dt, n_cpu, el, w, targets=target[:n_cpu + 1])
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": dof * 3 * n_cpu / sec, "unit": "DOF-stage updates/s (forward + adjoint)", "cores": 1, "kind": "port",
                               "sample": f"{n_cpu} steps forward and adjoint of the same problem with the oracle's CPU FP64 adjoint, 1 core",
                               "seconds": sec}
    adj.close()
    mesh.close()
    return out


def job_rate(local_ms: float, local_units: float, dist, device: str) -> tuple[float, float]:
    """Replicas: the slowest rank's device time (max over ranks) and the
    whole-job rate, the units all ranks processed over that time. `dist` is
    torch.distributed (or None for one process); tensors live on `device`
    (cuda for NCCL, cpu for gloo)."""
    import torch
    ms = torch.tensor([local_ms], dtype=torch.float64, device=device)
    units = torch.tensor([local_units], dtype=torch.float64, device=device)
    if dist is not None and dist.is_initialized():
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        dist.all_reduce(units, op=dist.ReduceOp.SUM)
    ms_max = float(ms.item())
    return ms_max, float(units.item()) / (ms_max / 1e3)


def run_ours(args) -> None:
    import torch
    import ndg_cuda_b200 as ndg

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    zone = workload_zone()
    mesh = ndg.Mesh2D_t(zone, ORDER, cfl=CFL, device=local, stream=stream.cuda_stream)
    mesh.initial_conditions()
    dof = ndg.dof_count(mesh)
    assert dof == dof_count()
    if args.tile is None:
        tile, _ = mesh.autotune(20)  # fields are restored by the tuner
    else:
        tile = args.tile  # fixed by hand (profiler runs, where the tuner's timings are distorted)
        mesh.set_tile(tile)

    ndg.Solver2D_t.run(mesh, args.warmup)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(physical_gpu_index(local)) as clocks:
        barrier()
        launches0 = mesh.launches()
        start.record(stream)
        ndg.Solver2D_t.run(mesh, args.steps)
        stop.record(stream)
        torch.cuda.synchronize()
        launches = mesh.launches() - launches0
        barrier()
    ms_max, value = job_rate(start.elapsed_time(stop), dof * 3 * args.steps, dist, "cuda")
    dt_step = ndg.Solver2D_t.get_delta_t(mesh)  # simulated time per RK3 step

    # Roofline of the dominant kernel: the fused stage kernel, timed per launch
    # for each of the three RK stages (the first reads no RK register).
    stages = stage_roofline(mesh, dof, measured_hbm_peak()[0])
    stage_ms = stages["mean_ms"]
    achieved = BYTES_PER_DOF_STAGE * dof / (stage_ms / 1e3) / 1e9
    peak, peak_kind = measured_hbm_peak()
    traffic = profiled_traffic(tile)

    # End to end through the C ABI with pinned host buffers.
    e2e_steps = 0 if args.no_e2e else 2
    host = {f: torch.empty(mesh.field_size, dtype=torch.float64, pin_memory=True) for f in ("p", "u", "v")}
    for f in host:
        host[f].copy_(torch.from_numpy(mesh.get_field(f)))
    L = ndg.lib()

    def e2e_call():
        for i, f in enumerate(("p", "u", "v")):
            ndg._check(L.ndg_set_field(mesh.handle, 0, i, host[f].data_ptr()))
        ndg.Solver2D_t.run(mesh, CONFIG_STEPS)
        for i, f in enumerate(("p", "u", "v")):
            ndg._check(L.ndg_get_field(mesh.handle, 0, i, host[f].data_ptr()))

    if e2e_steps:
        e2e_call()  # warm-up
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    wall0 = time.perf_counter()
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_call()
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    e2e_ms = e0.elapsed_time(e1)
    e2e_t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * dof * 3 * CONFIG_STEPS * e2e_steps / (float(e2e_t.item()) / 1e3) if e2e_steps else None
    state_bytes = 3 * mesh.field_size * 8

    # FP32 form on the same workload: throughput, kernel time, and its error
    # against this FP64 run after the configuration's 2000 steps from the
    # same initial condition.
    fp32 = None
    if not args.no_fp32:
        m32 = ndg.Mesh2D_t(zone, ORDER, cfl=CFL, device=local, stream=stream.cuda_stream, precision=ndg.FP32)
        m32.initial_conditions()
        tile32, _ = m32.autotune(20)
        ndg.Solver2D_t.run(m32, args.warmup)
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        ndg.Solver2D_t.run(m32, args.steps)
        f1.record(stream)
        torch.cuda.synchronize()
        f_ms = torch.tensor([f0.elapsed_time(f1)], dtype=torch.float64, device="cuda")
        if dist is not None:
            dist.all_reduce(f_ms, op=dist.ReduceOp.MAX)
        st32 = stage_roofline(m32, dof, peak)
        stage32_ms = st32["mean_ms"]
        m32.initial_conditions()
        mesh.initial_conditions()
        t32 = ndg.Solver2D_t.run(m32, CONFIG_STEPS)
        t64 = ndg.Solver2D_t.run(mesh, CONFIG_STEPS)
        l2_analytic = {"time": t64, "fp64": dict(zip("puv", map(float, mesh.l2_error(t64)))),
                       "fp32": dict(zip("puv", map(float, m32.l2_error(t32))))}
        err = {}
        for f in ("p", "u", "v"):
            a64, a32 = mesh.get_field(f), m32.get_field(f)
            err[f] = float(((a32 - a64) ** 2).sum() ** 0.5 / max((a64 ** 2).sum() ** 0.5, 1e-300))
        fp32 = {"value": world * dof * 3 * args.steps / (float(f_ms.item()) / 1e3), "unit": "DOF-stage updates/s",
                "ms_per_step": float(f_ms.item()) / args.steps, "kernel": f"stage_kernel_f32<{ORDER}>", "kernel_ms": stage32_ms,
                "per_stage": st32["per_stage"], "kernel_ms_per_step": st32["sum_ms"],
                "roofline_frac": BYTES_PER_DOF_STAGE * dof / (stage32_ms / 1e3) / 1e9 / peak,
                "rel_l2_vs_fp64": err, "steps_compared": CONFIG_STEPS, "tile_elements_per_cta": tile32 or m32.tile_candidates()[1],
                "l2_vs_analytic": l2_analytic,
                "wall_time_per_unit_time_s": float(f_ms.item()) / args.steps / 1e3 / dt_step,
                "arithmetic": "traces, fluxes, metrics and volume term in FP32; q, k and the RK update in FP64"}
        m32.close()

    hp = None
    if not args.no_hp and world == 1:
        hp = hp_leg(local, stream)

    config1 = config1_leg(local, stream) if not args.no_fp32 and world == 1 else None

    sweep = order_sweep_leg(local, stream) if not args.no_sweep and world == 1 else None
    published = published_runs_leg(local, stream) if not args.no_sweep and world == 1 else None

    batched = None
    if not args.no_batched:
        batched = batched_leg(local, stream, peak, dist)

    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_leg(local, stream, peak, rank == 0 and world == 1 and not args.no_cpu_baseline)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rate(float(os.environ.get("NDG_CPU_BUDGET_S", "15")), 1000, 1)

    if rank == 0:
        line = {"metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (reference plane-wave initial condition on a generated mesh)",
                "config": config(),
                "simulated_time_per_step": dt_step,
                "wall_time_per_unit_time_s": {"device_fp64": ms_max / args.steps / 1e3 / dt_step,
                                              "e2e_fp64": (float(e2e_t.item()) / 1e3 / (CONFIG_STEPS * e2e_steps) / dt_step) if e2e_steps else None},
                "e2e": {"value": e2e_value, "unit": "DOF-stage updates/s", "h2d_bytes_per_step": state_bytes,
                        "d2h_bytes_per_step": state_bytes, "rk3_steps_per_e2e_step": CONFIG_STEPS, "e2e_steps": e2e_steps,
                        "host_wall_s": wall},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                             "traffic": traffic, "kernel": f"stage_kernel<{ORDER}, false, {tile}>", "kernel_ms": stage_ms,
                             "per_stage": stages["per_stage"], "kernel_ms_per_step": stages["sum_ms"],
                             "ms_per_step_device": ms_max / args.steps,
                             "tile_elements_per_cta": tile or mesh.tile_candidates()[1],
                             "tile_source": "autotuner" if args.tile is None else "--tile",
                             "algorithmic_bytes_per_launch": BYTES_PER_DOF_STAGE * dof, "peak_source": peak_kind},
                "cpu_baseline": None if cpu is None else {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "fp32": fp32,
                "config1_analytic": config1,
                "hp_adaptive": hp,
                "order_sweep": sweep,
                "published_runs": published,
                "batched": batched,
                "adjoint": adjoint,
                "gpu_launches": launches,
                "clocks": clocks.summary()}
        print(json.dumps(line), flush=True)
    mesh.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=CONFIG_STEPS)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU reference timing (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end host-buffer leg (profiling runs)")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-form leg (profiling runs)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint leg (profiling runs)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-instances leg (profiling runs)")
    ap.add_argument("--no-hp", action="store_true", help="skip the hp-adaptive leg (profiling runs)")
    ap.add_argument("--no-sweep", action="store_true", help="skip the legs on the reference's published cases (order sweep, full runs)")
    ap.add_argument("--tile", type=int, default=None,
                    help="elements per CTA of the main leg's stage kernel instead of the autotuner's choice (profiling runs)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

