"""The hp-adaptive configuration run in lockstep with the reference's own CPU
path (Mesh2D_t::adapt, src/meshes/Mesh2D_t.cpp:1644-2268; hp_adapt :5186-5659;
split_faces :5661-5985), at the configuration's own scale.

Workload: a 128 x 128 walled quad mesh with interior nodes jittered by
U(-0.1h, 0.1h) (seed 7), N = 4 initially, p-refinement up to N = 12, up to two
split levels (2:1 mortar faces), an error estimate and adaptation every 20
steps, two crossing Gaussian pulses of width 0.1. The configured threshold
1e-4 never refines on this mesh (the largest estimate at N = 4 is 3.4e-6), so
the lockstep uses 1e-9, where p-refinement fires in the first round and
element splitting reaches split level 2 by the second.

Each side estimates and adapts on its own: the library from its device
estimate, the reference from its CPU estimate. Per round the refine flags and
the p/h decisions, then every topology array the C ABI returns
(ndg_mesh_get_*) must agree bit for bit, and the fields after the transfer
bit for bit in FP64_STRICT and within 1e-12 relative L2 in FP64.

Used by tests/test_gpu_hp_config.py and by bench.py's hp leg (as a checker,
outside every timed region).
"""
from __future__ import annotations

import numpy as np

import ndg_cuda_b200 as ndg
from ndg_cuda_b200 import meshgen
from ndg_cuda_b200 import workloads as A

RES, N0, N_MAX, SPLITS, INTERVAL, SEED, JITTER = 128, 4, 12, 2, 20, 7, 0.1
LOCKSTEP_TOLERANCE = 1e-9
FIELD_TOL = 1e-12


def zone(res: int = RES) -> dict:
    return meshgen.uniform_zone(res, boundary=meshgen.WALL, jitter=JITTER, seed=SEED)


def pulses(z: dict, N: int) -> dict:
    """Two Gaussian pulses of width 0.1 from (-0.4, -0.4) and (0.4, -0.4),
    moving along (1, 1) and (-1, 1): p = pa + pb, (u, v) = k_a pa + k_b pb."""
    k1, k2 = np.array([1.0, 1.0]) / np.sqrt(2), np.array([-1.0, 1.0]) / np.sqrt(2)
    pa = A.gaussian_pulse(z, N, sigma=0.1, centre=(-0.4, -0.4))
    pb = A.gaussian_pulse(z, N, sigma=0.1, centre=(0.4, -0.4))
    return {"p": pa + pb, "u": k1[0] * pa + k2[0] * pb, "v": k1[1] * pa + k2[1] * pb}


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def topology_diff(m, r) -> list[str]:
    """Names of the topology arrays where the library's mesh and the
    reference's differ (empty: bit-identical)."""
    bad = []
    if (m.n_elements_, m.n_elements_total_, m.n_faces_, m.n_nodes_) != (r.n_elements, r.n_elements_total, r.n_faces, r.n_nodes):
        return ["counts"]
    em, er = m.elements(), r.elements()
    for k in ("nodes", "N", "delta_xy_min", "first_face"):
        if not np.array_equal(em[k], er[k]):
            bad.append("elements." + k)
    sm = m.element_state()
    for k in ("split_level", "status", "rotation", "n_faces_side"):
        if not np.array_equal(sm[k], er[k]):
            bad.append("elements." + k)
    if not np.array_equal(sm["faces"], r.element_faces()):
        bad.append("elements.faces")
    fm, fr = m.faces(), r.faces()
    for k in ("nodes", "elements", "sides", "N", "normal", "tangent", "offset", "scale"):
        if not np.array_equal(fm[k], fr[k]):
            bad.append("faces." + k)
    for kind in range(7):
        if not np.array_equal(m.boundary(kind), r.boundary(kind)):
            bad.append(f"boundary.{kind}")
    if not np.array_equal(np.ravel(m.nodes()), np.ravel(r.nodes())):
        bad.append("nodes")
    return bad


def _decisions(err: dict, el: dict, K: int) -> tuple[np.ndarray, np.ndarray]:
    """would_p_refine and would_h_refine (src/entities/Element2D_t.cpp:802-812)."""
    refine = err["refine"][:K] == 1
    N, split = el["N"][:K], el["split_level"][:K]
    sigma = err["p_sigma"][:K]
    return refine & (sigma >= 1.0) & (N + 2 <= N_MAX), refine & (sigma < 1.0) & (split < SPLITS)


def run(rounds: int = 3, extra_steps: int = 5, tolerance: float = LOCKSTEP_TOLERANCE, res: int = RES,
        precisions=(("fp64_strict", ndg.FP64_STRICT), ("fp64", ndg.FP64)), device: int = 0, stream=None) -> dict:
    """Steps, estimates and adapts the reference's CPU path and one library
    mesh per precision side by side; returns a report of every comparison."""
    from oracle.pyoracle import RefSolver
    z = zone(res)
    ref = RefSolver(z, N0, N_max=N_MAX, max_split_level=SPLITS, tolerance_min=tolerance, tolerance_max=1e-14)
    meshes = {name: ndg.Mesh2D_t(z, N0, maximum_N=N_MAX, max_split_level=SPLITS, tolerance_min=tolerance, tolerance_max=1e-14,
                                 precision=prec, device=device, stream=stream) for name, prec in precisions}
    ic = pulses(z, N0)
    for f in ("p", "u", "v"):
        ref.set_field(f, ic[f])
        for m in meshes.values():
            m.set_field(f, ic[f])

    def field_errors() -> dict:
        out = {}
        want = {f: ref.field(f) for f in ("p", "u", "v")}
        for name, m in meshes.items():
            got = {f: m.get_field(f) for f in ("p", "u", "v")}
            out[name] = {"bitwise": all(np.array_equal(got[f], want[f]) for f in got),
                         "rel_l2": {f: rel_l2(got[f], want[f]) for f in got}}
        return out

    report = {"tolerance_min": tolerance, "mesh": f"{res}x{res} walls, jitter {JITTER} (seed {SEED})", "rounds": []}
    t = 0.0
    for rnd in range(rounds):
        t_ref = ref.run(INTERVAL, t)
        for m in meshes.values():
            t_m = ndg.Solver2D_t.run(m, INTERVAL, t)
            assert t_m == t_ref
        t = t_ref
        ref.estimate_error()
        e_ref = ref.error()
        el_ref = ref.elements()
        K = ref.n_elements
        p_ref, h_ref = _decisions(e_ref, {"N": el_ref["N"], "split_level": el_ref["split_level"]}, K)
        entry = {"round": rnd, "elements_before": K, "refine": int((e_ref["refine"] == 1).sum()),
                 "p_refine": int(p_ref.sum()), "h_refine": int(h_ref.sum()), "forms": {}}
        for name, m in meshes.items():
            m.estimate_error()
            e = m.error()
            st = m.element_state()
            p_m, h_m = _decisions(e, {"N": m.elements()["N"], "split_level": st["split_level"]}, K)
            entry["forms"][name] = {"refine_flags_equal": bool(np.array_equal(e["refine"], e_ref["refine"])),
                                    "p_h_decisions_equal": bool(np.array_equal(p_m, p_ref) and np.array_equal(h_m, h_ref)),
                                    "p_error_max_rel_diff": float(np.nanmax(np.abs(e["p_error"] - e_ref["p_error"]) /
                                                                            np.maximum(np.abs(e_ref["p_error"]), 1e-300)))}
        ref.adapt()
        for name, m in meshes.items():
            m.adapt()
            entry["forms"][name]["topology_mismatches"] = topology_diff(m, ref)
        fe = field_errors()
        for name in meshes:
            entry["forms"][name]["fields_after_adapt"] = fe[name]
        el = ref.elements()
        Kn = ref.n_elements
        entry["elements_after"] = Kn
        entry["orders_after"] = {str(int(k)): int(c) for k, c in zip(*np.unique(el["N"][:Kn], return_counts=True))}
        entry["split_levels_after"] = {str(int(k)): int(c) for k, c in zip(*np.unique(el["split_level"][:Kn], return_counts=True))}
        report["rounds"].append(entry)
    if extra_steps:
        t_ref = ref.run(extra_steps, t)
        for m in meshes.values():
            ndg.Solver2D_t.run(m, extra_steps, t)
        report["fields_after_extra_steps"] = {"steps": extra_steps, **field_errors()}
    for m in meshes.values():
        m.close()
    ok = True
    for entry in report["rounds"]:
        for name, fm in entry["forms"].items():
            ok &= fm["refine_flags_equal"] and fm["p_h_decisions_equal"] and not fm["topology_mismatches"]
            ok &= fm["fields_after_adapt"]["bitwise"] if name == "fp64_strict" else max(fm["fields_after_adapt"]["rel_l2"].values()) < FIELD_TOL
    if extra_steps:
        for name in meshes:
            fe = report["fields_after_extra_steps"][name]
            ok &= fe["bitwise"] if name == "fp64_strict" else max(fe["rel_l2"].values()) < FIELD_TOL
    last = report["rounds"][-1]["split_levels_after"] if report["rounds"] else {}
    report["split_levels_reached"] = sorted(int(k) for k in last)
    report["flags_parity"] = bool(ok)
    return report
