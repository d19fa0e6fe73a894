"""ctypes bindings for the two CPU checkers under oracle/.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
benchmark's CPU-baseline leg. The product never imports this module.

* `RefSolver` drives the reference's own CPU path compiled from its sources
  (oracle/_ref/libndgref.so, built by oracle/Makefile where the reference
  sources are present).
* `OracleSolver` drives the plain-C restatement (oracle/_ref/libndgoracle.so).

Both take a zone in the layout of tests/meshgen.py and expose the same calls.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libndgref.so")
ORACLE_LIB = os.path.join(HERE, "_ref", "libndgoracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build(reference_dir: str | None = None) -> None:
    """Builds the checkers (make -C oracle); the reference part only when its sources exist."""
    cmd = ["make", "-s", "-C", HERE]
    if reference_dir:
        cmd.append(f"REF={reference_dir}")
    subprocess.run(cmd, check=True)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


_ref = None
_orc = None


def _load_ref():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_LIB)
        lib.ndgref_zone_reset.argtypes = [C.c_long, _dp, _dp]
        lib.ndgref_zone_add_section.argtypes = [C.c_char_p, C.c_int, C.c_long, C.c_long, _lp, C.c_long]
        lib.ndgref_zone_add_boco.argtypes = [C.c_char_p, C.c_int, _lp, C.c_long]
        lib.ndgref_zone_add_conn.argtypes = [C.c_char_p, _lp, _lp, C.c_long]
        lib.ndgref_create.argtypes = [C.c_int, C.c_int, C.c_long, C.c_int, C.c_long, C.c_double, C.c_double, C.c_double]
        lib.ndgref_create_file.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_long, C.c_double]
        lib.ndgref_table.argtypes = [C.c_int, C.c_long, C.c_int, C.c_int, _dp]
        lib.ndgref_counts.argtypes = [C.POINTER(C.c_long)] * 4
        lib.ndgref_get_delta_t.restype = C.c_double
        lib.ndgref_stage.argtypes = [C.c_int, C.c_double, C.c_double]
        lib.ndgref_run.argtypes = [C.c_long, C.c_double]
        lib.ndgref_run.restype = C.c_double
        lib.ndgref_element_N.argtypes = [_ip]
        lib.ndgref_get_field.argtypes = [C.c_int, _dp]
        lib.ndgref_get_field.restype = C.c_long
        lib.ndgref_set_field.argtypes = [C.c_int, _dp]
        lib.ndgref_set_field.restype = C.c_long
        lib.ndgref_get_faces.argtypes = [_lp, _lp, _lp, _ip, _dp, _dp, _dp, _dp]
        lib.ndgref_get_elements.argtypes = [_lp, _ip, _ip, _ip, _ip, _dp, _lp, _ip]
        lib.ndgref_get_nodes.argtypes = [_dp]
        lib.ndgref_get_boundary.argtypes = [C.c_int, C.c_void_p]
        lib.ndgref_get_boundary.restype = C.c_long
        lib.ndgref_get_error.argtypes = [_dp, _dp, _ip, _ip]
        lib.ndgref_get_element_faces.argtypes = [C.c_void_p]
        lib.ndgref_get_element_faces.restype = C.c_long
        lib.ndgref_complete_solution.argtypes = [C.c_double, C.POINTER(C.c_void_p)]
        lib.ndgref_pre_condition.argtypes = [C.c_long, C.c_long, C.c_int]
        _ref = lib
    return _ref


def _load_oracle():
    global _orc
    if _orc is None:
        lib = C.CDLL(ORACLE_LIB)
        lib.ndgo_table.argtypes = [C.c_int, C.c_int64, C.c_int, C.c_int, _dp]
        lib.ndgo_create.restype = C.c_void_p
        lib.ndgo_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int64, _dp, _dp,
                                    C.c_int, _ip, _lp, _lp, _lp,
                                    C.c_int, _ip, _lp, _lp,
                                    C.c_int, _lp, _lp, _lp]
        lib.ndgo_destroy.argtypes = [C.c_void_p]
        lib.ndgo_counts.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 4
        lib.ndgo_initial_conditions.argtypes = [C.c_void_p]
        lib.ndgo_get_delta_t.argtypes = [C.c_void_p]
        lib.ndgo_get_delta_t.restype = C.c_double
        lib.ndgo_stage.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        lib.ndgo_run.argtypes = [C.c_void_p, C.c_int64, C.c_double]
        lib.ndgo_run.restype = C.c_double
        lib.ndgo_get_field.argtypes = [C.c_void_p, C.c_int, _dp]
        lib.ndgo_get_field.restype = C.c_int64
        lib.ndgo_set_field.argtypes = [C.c_void_p, C.c_int, _dp]
        lib.ndgo_set_field.restype = C.c_int64
        lib.ndgo_element_N.argtypes = [C.c_void_p, _ip]
        lib.ndgo_get_faces.argtypes = [C.c_void_p, _lp, _lp, _lp, _ip, _dp, _dp, _dp, _dp]
        lib.ndgo_get_elements.argtypes = [C.c_void_p, _lp, _ip, _dp, _lp]
        lib.ndgo_get_nodes.argtypes = [C.c_void_p, _dp]
        lib.ndgo_get_boundary.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        lib.ndgo_get_boundary.restype = C.c_int64
        lib.ndgo_estimate_error.argtypes = [C.c_void_p, C.c_double, C.c_double]
        lib.ndgo_get_error.argtypes = [C.c_void_p, _dp, _dp, _ip, _ip]
        lib.ndgo_set_speed.argtypes = [C.c_void_p, C.c_void_p]
        lib.ndgo_operator.argtypes = [C.c_void_p, _dp, _dp]
        lib.ndgo_operator.restype = C.c_int
        lib.ndgo_operator_transpose.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        lib.ndgo_operator_transpose.restype = C.c_int
        lib.ndgo_adjoint_solve.argtypes = [C.c_void_p, _dp, C.c_void_p, C.c_void_p, C.c_double, C.c_int64,
                                           C.c_int, _lp, _dp, C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        lib.ndgo_adjoint_solve.restype = C.c_double
        lib.ndgo_complete_solution.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.POINTER(C.c_void_p)]
        lib.ndgo_complete_solution.restype = C.c_int
        lib.ndgo_l2_error.argtypes = [C.c_void_p, C.c_double, _dp]
        _orc = lib
    return _orc


FIELDS = {"p": 0, "u": 1, "v": 2, "Gp": 3, "Gu": 4, "Gv": 5, "kp": 6, "ku": 7, "kv": 8}
# arrays of Mesh2D_t::get_complete_solution, in the checkers' output order
OUTPUT_NAMES = ("x", "y", "p", "u", "v", "dp_dt", "du_dt", "dv_dt",
                "p_analytical_error", "u_analytical_error", "v_analytical_error")


def _output_arrays(count: int) -> tuple[dict, C.Array]:
    arrays = {k: np.zeros(count) for k in OUTPUT_NAMES}
    ptrs = (C.c_void_p * len(OUTPUT_NAMES))(*[a.ctypes.data for a in arrays.values()])
    return arrays, ptrs


class _Base:
    n_elements: int
    n_elements_total: int
    n_faces: int
    n_nodes: int

    def field(self, name: str) -> np.ndarray:
        raise NotImplementedError

    def solution(self) -> np.ndarray:
        """(3, n_elements, (N+1)^2) for uniform N."""
        n2 = self.field("p").size // self.n_elements
        return np.stack([self.field(f).reshape(self.n_elements, n2) for f in ("p", "u", "v")])


class RefSolver(_Base):
    """The reference's own SEM::Host path (one process holds one instance)."""

    def __init__(self, zone: dict | str, N: int, N_max: int | None = None, cfl: float = 0.5, n_interp: int = 2,
                 max_split_level: int = 0, adaptivity_interval: int = 0,
                 tolerance_min: float = 1e-6, tolerance_max: float = 1e-14):
        lib = _load_ref()
        self.lib = lib
        self.n_interp = n_interp
        if isinstance(zone, str):
            lib.ndgref_create_file(zone.encode(), N, N_max if N_max is not None else N, n_interp, cfl)
            self._refresh_counts()
            return
        lib.ndgref_zone_reset(len(zone["x"]), np.ascontiguousarray(zone["x"]), np.ascontiguousarray(zone["y"]))
        for name, typ, start, end, conn in zone["sections"]:
            conn = np.ascontiguousarray(conn, dtype=np.int64)
            lib.ndgref_zone_add_section(name.encode(), typ, start, end, conn, conn.size)
        for name, bc, pts in zone["bocos"]:
            pts = np.ascontiguousarray(pts, dtype=np.int64)
            lib.ndgref_zone_add_boco(name.encode(), bc, pts, pts.size)
        for name, pts, donors in zone["conns"]:
            pts = np.ascontiguousarray(pts, dtype=np.int64)
            donors = np.ascontiguousarray(donors, dtype=np.int64)
            lib.ndgref_zone_add_conn(name.encode(), pts, donors, pts.size)
        lib.ndgref_create(N, N_max if N_max is not None else N, n_interp, max_split_level, adaptivity_interval,
                          tolerance_min, tolerance_max, cfl)
        self._refresh_counts()

    def _refresh_counts(self):
        vals = [C.c_long() for _ in range(4)]
        self.lib.ndgref_counts(*[C.byref(v) for v in vals])
        self.n_elements, self.n_elements_total, self.n_faces, self.n_nodes = (v.value for v in vals)

    def initial_conditions(self):
        self.lib.ndgref_initial_conditions()

    def delta_t(self) -> float:
        return self.lib.ndgref_get_delta_t()

    def stage(self, m: int, time: float, dt: float):
        self.lib.ndgref_stage(m, time, dt)

    def run(self, n_steps: int, time: float = 0.0) -> float:
        return self.lib.ndgref_run(n_steps, time)

    def element_N(self) -> np.ndarray:
        N = np.empty(self.n_elements, dtype=np.int32)
        self.lib.ndgref_element_N(N)
        return N

    def _field_size(self) -> int:
        N = self.element_N().astype(np.int64)
        return int(((N + 1) ** 2).sum())

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self._field_size())
        self.lib.ndgref_get_field(FIELDS[name], out)
        return out

    def set_field(self, name: str, values: np.ndarray):
        values = np.ascontiguousarray(values, dtype=np.float64).ravel()
        assert values.size == self._field_size()
        self.lib.ndgref_set_field(FIELDS[name], values)

    def faces(self) -> dict:
        F = self.n_faces
        d = {k: np.empty(2 * F, dtype=np.int64) for k in ("nodes", "elements", "sides")}
        d["N"] = np.empty(F, dtype=np.int32)
        for k in ("normal", "tangent", "offset", "scale"):
            d[k] = np.empty(2 * F)
        self.lib.ndgref_get_faces(d["nodes"], d["elements"], d["sides"], d["N"], d["normal"], d["tangent"], d["offset"], d["scale"])
        return d

    def elements(self) -> dict:
        E = self.n_elements_total
        d = {"nodes": np.empty(4 * E, dtype=np.int64), "N": np.empty(E, dtype=np.int32),
             "split_level": np.empty(E, dtype=np.int32), "status": np.empty(E, dtype=np.int32),
             "rotation": np.empty(E, dtype=np.int32), "delta_xy_min": np.empty(E),
             "first_face": np.empty(4 * E, dtype=np.int64), "n_faces_side": np.empty(4 * E, dtype=np.int32)}
        self.lib.ndgref_get_elements(d["nodes"], d["N"], d["split_level"], d["status"], d["rotation"],
                                     d["delta_xy_min"], d["first_face"], d["n_faces_side"])
        return d

    def element_faces(self) -> np.ndarray:
        n = self.lib.ndgref_get_element_faces(None)
        out = np.empty(max(n, 1), dtype=np.int64)
        self.lib.ndgref_get_element_faces(out.ctypes.data)
        return out[:n]

    def nodes(self) -> np.ndarray:
        out = np.empty(2 * self.n_nodes)
        self.lib.ndgref_get_nodes(out)
        return out.reshape(-1, 2)

    def boundary(self, kind: int) -> np.ndarray:
        n = self.lib.ndgref_get_boundary(kind, None)
        out = np.empty(n, dtype=np.int64)
        if n:
            self.lib.ndgref_get_boundary(kind, out.ctypes.data)
        return out

    def estimate_error(self):
        self.lib.ndgref_estimate_error()

    def error(self) -> dict:
        n = self.n_elements
        d = {"p_error": np.empty(n), "p_sigma": np.empty(n), "refine": np.empty(n, dtype=np.int32),
             "coarsen": np.empty(n, dtype=np.int32)}
        self.lib.ndgref_get_error(d["p_error"], d["p_sigma"], d["refine"], d["coarsen"])
        return d

    def adapt(self):
        self.lib.ndgref_adapt()
        self._refresh_counts()

    def complete_solution(self, time: float) -> dict:
        """Mesh2D_t::get_complete_solution at `time` (the reference's own code)."""
        arrays, ptrs = _output_arrays(self.n_elements * self.n_interp * self.n_interp)
        self.lib.ndgref_complete_solution(time, ptrs)
        return arrays

    def pre_condition(self, n_adaptivity_steps: int, pre_condition_interval: int, iterative: bool = False):
        """Solver2D_t::pre_condition / pre_condition_iterative (prints the reference's progress bar)."""
        self.lib.ndgref_pre_condition(n_adaptivity_steps, pre_condition_interval, 1 if iterative else 0)
        self._refresh_counts()


def ref_table(N_max: int, n_interp: int, table: int, N: int) -> np.ndarray:
    lib = _load_ref()
    out = np.empty(max((N + 1) * max(N + 1, n_interp), 1))
    cnt = lib.ndgref_table(N_max, n_interp, table, N, out)
    return out[:cnt].copy()


def oracle_table(N_max: int, n_interp: int, table: int, N: int) -> np.ndarray:
    lib = _load_oracle()
    out = np.empty(max((N + 1) * max(N + 1, n_interp), 1))
    cnt = lib.ndgo_table(N_max, n_interp, table, N, out)
    return out[:cnt].copy()


def _flatten(zone: dict) -> dict:
    secs = zone["sections"]
    cat = lambda xs, dt: np.concatenate([np.asarray(v, dtype=dt) for v in xs]) if xs else np.zeros(0, dt)  # noqa: E731
    return {
        "x": np.ascontiguousarray(zone["x"], dtype=np.float64),
        "y": np.ascontiguousarray(zone["y"], dtype=np.float64),
        "sec_type": np.array([s[1] for s in secs], dtype=np.int32),
        "sec_start": np.array([s[2] for s in secs], dtype=np.int64),
        "sec_end": np.array([s[3] for s in secs], dtype=np.int64),
        "sec_conn": cat([s[4] for s in secs], np.int64),
        "boco_type": np.array([b[1] for b in zone["bocos"]], dtype=np.int32),
        "boco_count": np.array([len(b[2]) for b in zone["bocos"]], dtype=np.int64),
        "boco_points": cat([b[2] for b in zone["bocos"]], np.int64),
        "conn_count": np.array([len(c[1]) for c in zone["conns"]], dtype=np.int64),
        "conn_points": cat([c[1] for c in zone["conns"]], np.int64),
        "conn_donors": cat([c[2] for c in zone["conns"]], np.int64),
    }


class OracleSolver(_Base):
    """The plain-C restatement (oracle/ndg_oracle.c)."""

    def __init__(self, zone: dict, N: int, N_max: int | None = None, cfl: float = 0.5,
                 tolerance_min: float = 1e-6, tolerance_max: float = 1e-14):
        lib = _load_oracle()
        self.lib = lib
        self.tolerance = (tolerance_min, tolerance_max)
        z = _flatten(zone)
        self._keep = z
        self.ctx = lib.ndgo_create(N, N_max if N_max is not None else N, cfl, len(z["x"]), z["x"], z["y"],
                                   len(z["sec_type"]), z["sec_type"], z["sec_start"], z["sec_end"], z["sec_conn"],
                                   len(z["boco_type"]), z["boco_type"], z["boco_count"], z["boco_points"],
                                   len(z["conn_count"]), z["conn_count"], z["conn_points"], z["conn_donors"])
        if not self.ctx:
            raise ValueError("oracle rejected the zone")
        vals = [C.c_int64() for _ in range(4)]
        lib.ndgo_counts(self.ctx, *[C.byref(v) for v in vals])
        self.n_elements, self.n_elements_total, self.n_faces, self.n_nodes = (v.value for v in vals)

    def __del__(self):
        if getattr(self, "ctx", None):
            self.lib.ndgo_destroy(self.ctx)
            self.ctx = None

    def initial_conditions(self):
        self.lib.ndgo_initial_conditions(self.ctx)

    def delta_t(self) -> float:
        return self.lib.ndgo_get_delta_t(self.ctx)

    def stage(self, m: int, time: float, dt: float):
        self.lib.ndgo_stage(self.ctx, m, time, dt)

    def run(self, n_steps: int, time: float = 0.0) -> float:
        return self.lib.ndgo_run(self.ctx, n_steps, time)

    def element_N(self) -> np.ndarray:
        N = np.empty(self.n_elements, dtype=np.int32)
        self.lib.ndgo_element_N(self.ctx, N)
        return N

    def _field_size(self) -> int:
        N = self.element_N().astype(np.int64)
        return int(((N + 1) ** 2).sum())

    def field(self, name: str) -> np.ndarray:
        out = np.empty(self._field_size())
        self.lib.ndgo_get_field(self.ctx, FIELDS[name], out)
        return out

    def set_field(self, name: str, values: np.ndarray):
        values = np.ascontiguousarray(values, dtype=np.float64).ravel()
        assert values.size == self._field_size()
        self.lib.ndgo_set_field(self.ctx, FIELDS[name], values)

    def faces(self) -> dict:
        F = self.n_faces
        d = {k: np.empty(2 * F, dtype=np.int64) for k in ("nodes", "elements", "sides")}
        d["N"] = np.empty(F, dtype=np.int32)
        for k in ("normal", "tangent", "offset", "scale"):
            d[k] = np.empty(2 * F)
        self.lib.ndgo_get_faces(self.ctx, d["nodes"], d["elements"], d["sides"], d["N"], d["normal"], d["tangent"],
                                d["offset"], d["scale"])
        return d

    def elements(self) -> dict:
        E = self.n_elements_total
        d = {"nodes": np.empty(4 * E, dtype=np.int64), "N": np.empty(E, dtype=np.int32),
             "delta_xy_min": np.empty(E), "first_face": np.empty(4 * E, dtype=np.int64)}
        self.lib.ndgo_get_elements(self.ctx, d["nodes"], d["N"], d["delta_xy_min"], d["first_face"])
        return d

    def nodes(self) -> np.ndarray:
        out = np.empty(2 * self.n_nodes)
        self.lib.ndgo_get_nodes(self.ctx, out)
        return out.reshape(-1, 2)

    def boundary(self, kind: int) -> np.ndarray:
        n = self.lib.ndgo_get_boundary(self.ctx, kind, None)
        out = np.empty(n, dtype=np.int64)
        if n:
            self.lib.ndgo_get_boundary(self.ctx, kind, out.ctypes.data)
        return out

    def estimate_error(self):
        self.lib.ndgo_estimate_error(self.ctx, *self.tolerance)

    def l2_error(self, time: float) -> np.ndarray:
        """L2 error of p, u, v against the plane wave at `time`."""
        out = np.zeros(3)
        self.lib.ndgo_l2_error(self.ctx, time, out)
        return out

    def complete_solution(self, n_interp: int, time: float) -> dict:
        """Restatement of Mesh2D_t::get_complete_solution on n_interp^2 points per element."""
        arrays, ptrs = _output_arrays(self.n_elements * n_interp * n_interp)
        if self.lib.ndgo_complete_solution(self.ctx, n_interp, time, ptrs) != 0:
            raise ValueError("bad output request")
        return arrays

    def error(self) -> dict:
        n = self.n_elements
        d = {"p_error": np.empty(n), "p_sigma": np.empty(n), "refine": np.empty(n, dtype=np.int32),
             "coarsen": np.empty(n, dtype=np.int32)}
        self.lib.ndgo_get_error(self.ctx, d["p_error"], d["p_sigma"], d["refine"], d["coarsen"])
        return d

    # Variable-speed operator and its discrete adjoint (CPU reference gradient).
    def set_speed(self, speed):
        if speed is None:
            self.lib.ndgo_set_speed(self.ctx, None)
            return
        self._speed = np.ascontiguousarray(speed, dtype=np.float64).ravel()
        assert self._speed.size == self.n_elements
        self.lib.ndgo_set_speed(self.ctx, self._speed.ctypes.data)

    def operator(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        out = np.empty_like(x)
        if self.lib.ndgo_operator(self.ctx, x, out) != 0:
            raise ValueError("operator failed")
        return out

    def operator_transpose(self, x, y) -> tuple[np.ndarray, np.ndarray]:
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.ascontiguousarray(y, dtype=np.float64).ravel()
        lty, dc = np.empty_like(y), np.empty(self.n_elements)
        if self.lib.ndgo_operator_transpose(self.ctx, x, y, lty, dc) != 0:
            raise ValueError("the transpose covers conforming faces of one order")
        return lty, dc

    def adjoint_solve(self, p0, dt: float, n_steps: int, rec_elem, rec_w, targets=None, u0=None, v0=None) -> dict:
        """Forward solve with receivers, misfit J and its gradient (p0, u0, v0, c)."""
        fs = self._field_size()
        p0 = np.ascontiguousarray(p0, dtype=np.float64).ravel()
        u0 = None if u0 is None else np.ascontiguousarray(u0, dtype=np.float64).ravel()
        v0 = None if v0 is None else np.ascontiguousarray(v0, dtype=np.float64).ravel()
        rec_elem = np.ascontiguousarray(rec_elem, dtype=np.int64).ravel()
        rec_w = np.ascontiguousarray(rec_w, dtype=np.float64).ravel()
        R = rec_elem.size
        tg = None if targets is None else np.ascontiguousarray(targets, dtype=np.float64).reshape(n_steps + 1, R)
        samples = np.empty((n_steps + 1, max(R, 1)))
        g = {k: np.empty(fs) for k in ("p0", "u0", "v0")}
        g["c"] = np.empty(self.n_elements)
        J = self.lib.ndgo_adjoint_solve(self.ctx, p0, None if u0 is None else u0.ctypes.data, None if v0 is None else v0.ctypes.data,
                                        dt, n_steps, R, rec_elem if R else np.zeros(1, np.int64), rec_w if R else np.zeros(1),
                                        None if tg is None else tg.ctypes.data, samples, g["p0"], g["u0"], g["v0"], g["c"])
        g["J"] = J
        g["samples"] = samples[:, :R]
        return g
