"""ndg_cuda_b200: B200-native DG spectral-element solver for the 2D wave equation.

Python host side of the library. It mirrors the reference's host API for the
hot path -- NDG_t (polynomial tables), Mesh2D_t (mesh, initial conditions,
fields) and Solver2D_t (CFL step, RK3 stepping, solve) -- over the C ABI of
include/ndg_b200.h, which ctypes binds from the in-tree
ndg_cuda_b200/libndg_b200.so. There is no fallback: if the library is missing
or a call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = ["NdgError", "lib", "NDG_t", "Mesh2D_t", "Solver2D_t", "Adjoint2D_t", "DataWriter_t", "Zone", "LIB_PATH",
           "FP64", "FP64_STRICT", "FP32", "tables_compute"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libndg_b200.so")

FP64, FP64_STRICT, FP32 = 0, 1, 2
# Tile codes at or above TENSOR_TILE select the stage kernel whose contraction
# passes run on the tensor cores, with (code - TENSOR_TILE) elements per CTA.
TENSOR_TILE = 100
_STATUS = {0: "OK", 1: "INVALID_ARG", 2: "MESH", 3: "CUDA", 4: "NONFINITE", 5: "OOM", 6: "TIMEOUT", 7: "UNSUPPORTED"}
FIELDS = {"p": 0, "u": 1, "v": 2, "G_p": 3, "G_u": 4, "G_v": 5, "k_p": 6, "k_u": 7, "k_v": 8}
TABLES = ["nodes", "weights", "barycentric_weights", "lagrange_interpolant_left", "lagrange_interpolant_right",
          "lagrange_interpolant_derivative_left", "lagrange_interpolant_derivative_right", "derivative_matrices",
          "g_hat_derivative_matrices", "derivative_matrices_hat", "interpolation_matrices", "polynomials"]


class NdgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, status)}: {message}")
        self.status = status


class _Zone(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("x", C.c_void_p), ("y", C.c_void_p),
                ("n_sections", C.c_int32), ("section_type", C.c_void_p), ("section_start", C.c_void_p),
                ("section_end", C.c_void_p), ("section_connectivity", C.c_void_p),
                ("n_bocos", C.c_int32), ("boco_type", C.c_void_p), ("boco_count", C.c_void_p), ("boco_points", C.c_void_p),
                ("n_conns", C.c_int32), ("conn_count", C.c_void_p), ("conn_points", C.c_void_p), ("conn_donors", C.c_void_p)]


class _Params(C.Structure):
    _fields_ = [("initial_N", C.c_int32), ("maximum_N", C.c_int32), ("n_interpolation_points", C.c_int64),
                ("max_split_level", C.c_int32), ("adaptivity_interval", C.c_int64),
                ("tolerance_min", C.c_double), ("tolerance_max", C.c_double), ("cfl", C.c_double)]


# arrays of ndg_get_solution / ndg_solution_output, in its field order
SOLUTION_NAMES = ("x", "y", "p", "u", "v", "dp_dt", "du_dt", "dv_dt",
                  "p_analytical_error", "u_analytical_error", "v_analytical_error")


class _SolutionOutput(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in SOLUTION_NAMES]


class _OutputArrays(C.Structure):
    _fields_ = ([("complete", C.c_int32)] + [(k, C.c_void_p) for k in SOLUTION_NAMES]
                + [("N", C.c_void_p), ("status", C.c_void_p), ("rotation", C.c_void_p), ("rank", C.c_int32)]
                + [(k, C.c_void_p) for k in ("p_error", "u_error", "v_error", "p_sigma", "u_sigma", "v_sigma",
                                             "refine", "coarsen", "split_level")])


_lib = None


def lib() -> C.CDLL:
    """Loads libndg_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise NdgError(3, f"{LIB_PATH} is missing; build it with python -m ndg_cuda_b200.build")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    sigs = {
        "ndg_last_error": ([], C.c_char_p), "ndg_version": ([], C.c_char_p),
        "ndg_ctx_create": ([i32, vp, C.POINTER(vp)], C.c_int),
        "ndg_ctx_destroy": ([vp], C.c_int),
        "ndg_ctx_set_precision": ([vp, i32], C.c_int),
        "ndg_ctx_keep_derivative": ([vp, i32], C.c_int),
        "ndg_set_mixed_launch": ([vp, i32], C.c_int),
        "ndg_adapt_timings": ([vp, C.POINTER(dbl)], C.c_int),
        "ndg_ctx_synchronize": ([vp], C.c_int),
        "ndg_tables_build": ([vp, i32, i64], C.c_int),
        "ndg_tables_get": ([vp, i32, i32, vp, i64, C.POINTER(i64)], C.c_int),
        "ndg_tables_compute": ([i32, i64, i32, i32, vp, i64, C.POINTER(i64)], C.c_int),
        "ndg_mesh_load_zone": ([vp, C.POINTER(_Zone), C.POINTER(_Params), i32], C.c_int),
        "ndg_mesh_load_file": ([vp, C.c_char_p, C.POINTER(_Params), i32], C.c_int),
        "ndg_mesh_counts": ([vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)], C.c_int),
        "ndg_mesh_get_faces": ([vp] * 9, C.c_int),
        "ndg_mesh_get_elements": ([vp] * 5, C.c_int),
        "ndg_mesh_get_boundary": ([vp, i32, vp, i64, C.POINTER(i64)], C.c_int),
        "ndg_mesh_get_nodes": ([vp, vp], C.c_int),
        "ndg_mesh_get_element_state": ([vp, vp, vp, vp, vp], C.c_int),
        "ndg_mesh_get_element_faces": ([vp, vp, i64, C.POINTER(i64)], C.c_int),
        "ndg_mesh_field_size": ([vp, C.POINTER(i64)], C.c_int),
        "ndg_initial_conditions": ([vp], C.c_int),
        "ndg_set_field": ([vp, i32, i32, vp], C.c_int),
        "ndg_get_field": ([vp, i32, i32, vp], C.c_int),
        "ndg_get_delta_t": ([vp, C.POINTER(dbl)], C.c_int),
        "ndg_set_cfl": ([vp, dbl], C.c_int),
        "ndg_stage": ([vp, i32, dbl, dbl], C.c_int),
        "ndg_run": ([vp, i64, C.POINTER(dbl)], C.c_int),
        "ndg_solve": ([vp, dbl, C.POINTER(dbl), C.POINTER(i64)], C.c_int),
        "ndg_launch_count": ([vp, C.POINTER(i64)], C.c_int),
        "ndg_time_stage": ([vp, i32, i32, C.POINTER(dbl)], C.c_int),
        "ndg_estimate_error": ([vp], C.c_int),
        "ndg_get_error": ([vp, i32, vp, vp, vp, vp], C.c_int),
        "ndg_adapt": ([vp], C.c_int),
        "ndg_get_solution": ([vp, i32, dbl, C.POINTER(_SolutionOutput)], C.c_int),
        "ndg_writer_create": ([C.c_char_p, C.POINTER(vp)], C.c_int),
        "ndg_writer_destroy": ([vp], C.c_int),
        "ndg_writer_write_arrays": ([vp, dbl, i64, i64, C.POINTER(_OutputArrays)], C.c_int),
        "ndg_writer_write": ([vp, vp, i32, dbl, i32], C.c_int),
        "ndg_pre_condition": ([vp, i64, i64, i32, C.POINTER(i64)], C.c_int),
        "ndg_l2_error": ([vp, i32, dbl, vp], C.c_int),
        "ndg_adapt_flags": ([vp, vp, vp], C.c_int),
        "ndg_delta_t_from_device": ([vp, vp, i64, dbl, vp, C.POINTER(dbl)], C.c_int),
        "ndg_autotune": ([vp, i32, C.POINTER(i32), C.POINTER(dbl)], C.c_int),
        "ndg_set_tile": ([vp, i32], C.c_int),
        "ndg_tile_candidates": ([vp, vp, i32, C.POINTER(i32), C.POINTER(i32)], C.c_int),
        "ndg_adjoint_create": ([vp, i32, vp, C.POINTER(vp)], C.c_int),
        "ndg_adjoint_destroy": ([vp], C.c_int),
        "ndg_adjoint_set_speed": ([vp, vp], C.c_int),
        "ndg_adjoint_set_precision": ([vp, i32], C.c_int),
        "ndg_adjoint_delta_t": ([vp, dbl, C.POINTER(dbl)], C.c_int),
        "ndg_adjoint_receivers": ([vp, vp, vp], C.c_int),
        "ndg_adjoint_forward": ([vp, vp, vp, vp, vp, dbl, i64, i64, vp, C.POINTER(dbl)], C.c_int),
        "ndg_adjoint_backward": ([vp, vp, vp, vp, vp], C.c_int),
        "ndg_adjoint_operator": ([vp, vp, vp, vp, vp, vp], C.c_int),
        "ndg_adjoint_timings": ([vp, C.POINTER(dbl), C.POINTER(dbl), C.POINTER(i64), C.POINTER(i64)], C.c_int),
        "ndg_adjoint_time_stage": ([vp, i32, i32, C.POINTER(dbl)], C.c_int),
    }
    for name, (args, res) in sigs.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _check(status: int) -> None:
    if status != 0:
        raise NdgError(status, lib().ndg_last_error().decode())


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def tables_compute(N_max: int, n_interpolation_points: int, table: str | int, N: int) -> np.ndarray:
    """One NDG_t table computed on the host (no GPU needed)."""
    t = TABLES.index(table) if isinstance(table, str) else table
    count = C.c_int64()
    _check(lib().ndg_tables_compute(N_max, n_interpolation_points, t, N, None, 0, C.byref(count)))
    out = np.empty(count.value)
    _check(lib().ndg_tables_compute(N_max, n_interpolation_points, t, N, _ptr(out), out.size, C.byref(count)))
    return out


class Zone:
    """One unstructured 2D zone in CGNS terms (the input of Mesh2D_t).

    `sections` are (name, type, start, end, connectivity) with type 0 = QUAD_4
    and 1 = BAR_2; `bocos` are (name, bc, points); `conns` are
    (name, points, donor_points); all element and node numbers 1-based.
    """

    def __init__(self, x, y, sections, bocos=(), conns=()):
        self.x = np.ascontiguousarray(x, dtype=np.float64)
        self.y = np.ascontiguousarray(y, dtype=np.float64)
        self.sections = list(sections)
        self.bocos = list(bocos)
        self.conns = list(conns)

    @classmethod
    def from_dict(cls, d: dict) -> "Zone":
        return cls(d["x"], d["y"], d["sections"], d["bocos"], d["conns"])

    def _struct(self) -> tuple[_Zone, list]:
        keep = []

        def arr(values, dtype):
            a = np.ascontiguousarray(np.asarray(values, dtype=dtype)) if len(values) else np.zeros(1, dtype=dtype)
            keep.append(a)
            return _ptr(a)

        z = _Zone()
        z.n_nodes = self.x.size
        z.x, z.y = _ptr(self.x), _ptr(self.y)
        z.n_sections = len(self.sections)
        z.section_type = arr([s[1] for s in self.sections], np.int32)
        z.section_start = arr([s[2] for s in self.sections], np.int64)
        z.section_end = arr([s[3] for s in self.sections], np.int64)
        z.section_connectivity = arr(np.concatenate([np.asarray(s[4], np.int64) for s in self.sections]), np.int64)
        z.n_bocos = len(self.bocos)
        z.boco_type = arr([b[1] for b in self.bocos], np.int32)
        z.boco_count = arr([len(b[2]) for b in self.bocos], np.int64)
        z.boco_points = arr(np.concatenate([np.asarray(b[2], np.int64) for b in self.bocos]) if self.bocos else [], np.int64)
        z.n_conns = len(self.conns)
        z.conn_count = arr([len(c[1]) for c in self.conns], np.int64)
        z.conn_points = arr(np.concatenate([np.asarray(c[1], np.int64) for c in self.conns]) if self.conns else [], np.int64)
        z.conn_donors = arr(np.concatenate([np.asarray(c[2], np.int64) for c in self.conns]) if self.conns else [], np.int64)
        return z, keep


class _Context:
    def __init__(self, device: int, stream: int | None = None):
        h = C.c_void_p()
        _check(lib().ndg_ctx_create(device, stream, C.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            lib().ndg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NDG_t:
    """Polynomial tables of NDG_t<LegendrePolynomial_t>(N_max, n_interpolation_points)
    (include/entities/NDG_t.cuh:11-29), one numpy array per order."""

    def __init__(self, N_max: int, n_interpolation_points: int, device: int = 0):
        self.N_max_ = N_max
        self.N_interpolation_points_ = n_interpolation_points
        self._ctx = _Context(device)
        _check(lib().ndg_tables_build(self._ctx.h, N_max, n_interpolation_points))
        for i, name in enumerate(TABLES):
            setattr(self, name + "_", [self._get(i, N) for N in range(N_max + 1)])

    def _get(self, table: int, N: int) -> np.ndarray:
        count = C.c_int64()
        _check(lib().ndg_tables_get(self._ctx.h, table, N, None, 0, C.byref(count)))
        out = np.empty(count.value)
        _check(lib().ndg_tables_get(self._ctx.h, table, N, _ptr(out), out.size, C.byref(count)))
        return out


class Mesh2D_t:
    """Mesh2D_t(zone, initial_N, maximum_N, ...) on one GPU
    (include/meshes/Mesh2D_t.cuh:23-182): reference numbering of elements,
    faces, ghosts and boundaries; device fields p, u, v, G and the RK register.

    `mesh` is a Zone, a zone dict (tests/meshgen.py layout) or a .su2 path.
    `n_instances` independent solutions share the mesh (batched runs).
    device < 0 builds the topology only (no GPU).
    """

    def __init__(self, mesh, initial_N: int, maximum_N: int | None = None, n_interpolation_points: int = 2,
                 max_split_level: int = 0, adaptivity_interval: int = 0, tolerance_min: float = 1e-6,
                 tolerance_max: float = 1e-14, cfl: float = 0.5, n_instances: int = 1, device: int = 0,
                 precision: int = FP64, keep_derivative: bool = False, stream: int | None = None):
        self.initial_N_ = initial_N
        self.maximum_N_ = maximum_N if maximum_N is not None else initial_N
        self.adaptivity_interval_ = adaptivity_interval
        self.n_interpolation_points_ = n_interpolation_points
        self.keep_derivative_ = keep_derivative
        self.n_instances = n_instances
        self._ctx = _Context(device, stream)
        h = self._ctx.h
        if precision != FP64:
            _check(lib().ndg_ctx_set_precision(h, precision))
        if keep_derivative:
            _check(lib().ndg_ctx_keep_derivative(h, 1))
        p = _Params(initial_N, self.maximum_N_, n_interpolation_points, max_split_level, adaptivity_interval,
                    tolerance_min, tolerance_max, cfl)
        if isinstance(mesh, (str, os.PathLike)):
            _check(lib().ndg_mesh_load_file(h, os.fspath(mesh).encode(), C.byref(p), n_instances))
        else:
            zone = mesh if isinstance(mesh, Zone) else Zone.from_dict(mesh)
            z, keep = zone._struct()
            _check(lib().ndg_mesh_load_zone(h, C.byref(z), C.byref(p), n_instances))
            del keep
        counts = [C.c_int64() for _ in range(4)]
        _check(lib().ndg_mesh_counts(h, *[C.byref(c) for c in counts]))
        self.n_elements_, self.n_elements_total_, self.n_faces_, self.n_nodes_ = (c.value for c in counts)
        fs = C.c_int64()
        _check(lib().ndg_mesh_field_size(h, C.byref(fs)))
        self.field_size = fs.value

    @property
    def handle(self):
        return self._ctx.h

    def set_precision(self, precision: int) -> None:
        _check(lib().ndg_ctx_set_precision(self._ctx.h, precision))

    def adapt_timings(self) -> dict:
        """Host wall time (ms) of the last adaptation by phase."""
        ms = (C.c_double * 4)()
        _check(lib().ndg_adapt_timings(self._ctx.h, ms))
        return dict(zip(("device_decisions", "topology", "transfer", "plan"), ms))

    def set_mixed_launch(self, mode: int) -> None:
        """Mixed-order meshes: 0 one launch per order group, groups of at least 2,048 elements whose
        order has no conforming part split into a side-flux launch and an element-tile launch
        (default); 1 one queue launch per stage;
        2 as 0 with every group that is not all conforming elements split."""
        _check(lib().ndg_set_mixed_launch(self._ctx.h, mode))

    # Mesh2D_t::initial_conditions (src/meshes/Mesh2D_t.cu:5030)
    def initial_conditions(self) -> None:
        _check(lib().ndg_initial_conditions(self._ctx.h))

    def set_field(self, name: str, values: np.ndarray, instance: int = -1) -> None:
        values = np.ascontiguousarray(values, dtype=np.float64).ravel()
        expected = self.field_size * (self.n_instances if instance < 0 else 1)
        if values.size != expected:
            raise ValueError(f"expected {expected} values, got {values.size}")
        _check(lib().ndg_set_field(self._ctx.h, instance, FIELDS[name], _ptr(values)))

    def get_field(self, name: str, instance: int = -1) -> np.ndarray:
        out = np.empty(self.field_size * (self.n_instances if instance < 0 else 1))
        _check(lib().ndg_get_field(self._ctx.h, instance, FIELDS[name], _ptr(out)))
        return out

    # Mesh2D_t::estimate_error (src/meshes/Mesh2D_t.cu:5158)
    def estimate_error(self) -> None:
        _check(lib().ndg_estimate_error(self._ctx.h))

    def error(self, instance: int = 0) -> dict:
        """p_error_, p_sigma_, refine_, coarsen_ of every element of one instance."""
        K = self.n_elements_
        d = {"p_error": np.empty(K), "p_sigma": np.empty(K), "refine": np.empty(K, dtype=np.int32),
             "coarsen": np.empty(K, dtype=np.int32)}
        _check(lib().ndg_get_error(self._ctx.h, instance, *[_ptr(d[k]) for k in ("p_error", "p_sigma", "refine", "coarsen")]))
        return d

    def adapt(self, refine: np.ndarray | None = None, p_sigma: np.ndarray | None = None) -> None:
        """Mesh2D_t::adapt: from the last error estimate, or from the given
        per-element refine flags and decay rates."""
        if refine is None:
            _check(lib().ndg_adapt(self._ctx.h))
        else:
            r = np.ascontiguousarray(refine, dtype=np.int32)
            sg = np.ascontiguousarray(p_sigma, dtype=np.float64)
            _check(lib().ndg_adapt_flags(self._ctx.h, _ptr(r), _ptr(sg)))
        self._refresh_counts()

    def _refresh_counts(self) -> None:
        counts = [C.c_int64() for _ in range(4)]
        _check(lib().ndg_mesh_counts(self._ctx.h, *[C.byref(c) for c in counts]))
        self.n_elements_, self.n_elements_total_, self.n_faces_, self.n_nodes_ = (c.value for c in counts)
        fs = C.c_int64()
        _check(lib().ndg_mesh_field_size(self._ctx.h, C.byref(fs)))
        self.field_size = fs.value

    def synchronize(self) -> None:
        _check(lib().ndg_ctx_synchronize(self._ctx.h))

    def time_stage(self, m: int, n_launches: int) -> float:
        """Mean duration in ms of the stage-m kernel over n_launches launches (advances the state)."""
        ms = C.c_double()
        _check(lib().ndg_time_stage(self._ctx.h, m, n_launches, C.byref(ms)))
        return ms.value

    def autotune(self, n_launches: int = 20) -> tuple[int, float]:
        """Times every candidate tile of the stage kernel on this mesh and
        keeps the fastest: (elements per CTA, 0 = default; ms per launch)."""
        e, ms = C.c_int32(), C.c_double()
        _check(lib().ndg_autotune(self._ctx.h, n_launches, C.byref(e), C.byref(ms)))
        return e.value, ms.value

    def set_tile(self, elements_per_block: int) -> None:
        _check(lib().ndg_set_tile(self._ctx.h, elements_per_block))

    def tile_candidates(self) -> tuple[list[int], int]:
        out = (C.c_int32 * 16)()
        n, d = C.c_int32(), C.c_int32()
        _check(lib().ndg_tile_candidates(self._ctx.h, C.cast(out, C.c_void_p), 16, C.byref(n), C.byref(d)))
        return list(out[:n.value]), d.value

    def launches(self) -> int:
        n = C.c_int64()
        _check(lib().ndg_launch_count(self._ctx.h, C.byref(n)))
        return n.value

    # Topology views with the reference's numbering.
    def faces(self) -> dict:
        F = self.n_faces_
        d = {k: np.empty(2 * F, dtype=np.int64) for k in ("nodes", "elements", "sides")}
        d["N"] = np.empty(F, dtype=np.int32)
        for k in ("normal", "tangent", "offset", "scale"):
            d[k] = np.empty(2 * F)
        _check(lib().ndg_mesh_get_faces(self._ctx.h, *[_ptr(d[k]) for k in ("nodes", "elements", "sides", "N", "normal", "tangent", "offset", "scale")]))
        return d

    def elements(self) -> dict:
        E = self.n_elements_total_
        d = {"nodes": np.empty(4 * E, dtype=np.int64), "N": np.empty(E, dtype=np.int32), "delta_xy_min": np.empty(E),
             "first_face": np.empty(4 * E, dtype=np.int64)}
        _check(lib().ndg_mesh_get_elements(self._ctx.h, *[_ptr(d[k]) for k in ("nodes", "N", "delta_xy_min", "first_face")]))
        return d

    def element_state(self) -> dict:
        """split_level, status, rotation and faces per side of every element,
        with the face lists concatenated side by side."""
        E = self.n_elements_total_
        d = {"split_level": np.empty(E, dtype=np.int32), "status": np.empty(E, dtype=np.int32),
             "rotation": np.empty(E, dtype=np.int32), "n_faces_side": np.empty(4 * E, dtype=np.int32)}
        _check(lib().ndg_mesh_get_element_state(self._ctx.h, *[_ptr(d[k]) for k in ("split_level", "status", "rotation", "n_faces_side")]))
        cnt = C.c_int64()
        _check(lib().ndg_mesh_get_element_faces(self._ctx.h, None, 0, C.byref(cnt)))
        d["faces"] = np.empty(max(cnt.value, 1), dtype=np.int64)
        _check(lib().ndg_mesh_get_element_faces(self._ctx.h, _ptr(d["faces"]), d["faces"].size, C.byref(cnt)))
        d["faces"] = d["faces"][:cnt.value]
        return d

    def boundary(self, kind: int) -> np.ndarray:
        cnt = C.c_int64()
        _check(lib().ndg_mesh_get_boundary(self._ctx.h, kind, None, 0, C.byref(cnt)))
        out = np.empty(max(cnt.value, 1), dtype=np.int64)
        _check(lib().ndg_mesh_get_boundary(self._ctx.h, kind, _ptr(out), out.size, C.byref(cnt)))
        return out[:cnt.value]

    def nodes(self) -> np.ndarray:
        out = np.empty(2 * self.n_nodes_)
        _check(lib().ndg_mesh_get_nodes(self._ctx.h, _ptr(out)))
        return out.reshape(-1, 2)

    # Mesh2D_t::get_solution / get_complete_solution (src/meshes/Mesh2D_t.cpp:4237-4296)
    def get_solution(self, time: float = 0.0, complete: bool = False, instance: int = 0) -> dict:
        """Fields on the n_interpolation_points^2 output grid of every element
        (ndg_get_solution): x, y, p, u, v, and with `complete` the analytic
        errors at `time` and, when the mesh keeps them, the time derivatives.
        Element e's point (i, j) is entry e n^2 + i n + j."""
        names = ["x", "y", "p", "u", "v"]
        if complete:
            if self.keep_derivative_:
                names += ["dp_dt", "du_dt", "dv_dt"]
            names += ["p_analytical_error", "u_analytical_error", "v_analytical_error"]
        P = self.n_interpolation_points_
        arrays = {k: np.empty(self.n_elements_ * P * P) for k in names}
        o = _SolutionOutput(**{k: arrays[k].ctypes.data for k in names})
        _check(lib().ndg_get_solution(self._ctx.h, instance, float(time), C.byref(o)))
        return arrays

    def get_complete_solution(self, time: float, instance: int = 0) -> dict:
        return self.get_solution(time, complete=True, instance=instance)

    def l2_error(self, time: float, instance: int = 0) -> np.ndarray:
        """L2 error of p, u, v against the reference plane wave at `time`
        (ndg_l2_error): sqrt(sum w_i w_j J (q - g)^2) per field."""
        out = np.zeros(3)
        _check(lib().ndg_l2_error(self._ctx.h, instance, float(time), _ptr(out)))
        return out

    # Mesh2D_t::write_data / write_complete_data (src/meshes/Mesh2D_t.cpp:1601-1642)
    def write_data(self, time: float, data_writer: "DataWriter_t", instance: int = 0) -> None:
        _check(lib().ndg_writer_write(data_writer.handle, self._ctx.h, instance, float(time), 0))

    def write_complete_data(self, time: float, data_writer: "DataWriter_t", instance: int = 0) -> None:
        _check(lib().ndg_writer_write(data_writer.handle, self._ctx.h, instance, float(time), 1))

    def close(self) -> None:
        self._ctx.close()


class DataWriter_t:
    """DataWriter_t(output_filename) (include/helpers/DataWriter_t.h,
    src/helpers/DataWriter_t.cpp), without VTK: per output time a parallel
    unstructured grid <stem>_t<time>s<ext> with its piece <...>_0.vtu, the
    element grid <stem>_element_t<time>s<ext> for complete outputs, and the
    time series files <output_filename>.series and <stem>_element<ext>.series
    (created empty here)."""

    def __init__(self, output_filename):
        h = C.c_void_p()
        _check(lib().ndg_writer_create(os.fspath(output_filename).encode(), C.byref(h)))
        self.handle = h.value

    def write_arrays(self, time: float, n_elements: int, n_interp: int, arrays: dict, complete: bool = False,
                     rank: int = 0) -> None:
        """Writes host arrays (the names of Mesh2D_t.get_solution, plus the
        element arrays N, status, rotation, p_error, u_error, v_error, p_sigma,
        u_sigma, v_sigma, refine, coarsen, split_level); missing ones are
        zeros. Needs no GPU."""
        keep = {}
        fields = {}
        for k, v in arrays.items():
            dt = np.int32 if k in ("N", "status", "rotation", "refine", "coarsen", "split_level") else np.float64
            keep[k] = np.ascontiguousarray(v, dtype=dt)
            fields[k] = keep[k].ctypes.data
        a = _OutputArrays(complete=1 if complete else 0, rank=rank, **fields)
        _check(lib().ndg_writer_write_arrays(self.handle, float(time), n_elements, n_interp, C.byref(a)))
        del keep

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib().ndg_writer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver2D_t:
    """Solver2D_t(CFL, output_times, viscosity) (include/solvers/Solver2D_t.cuh:14-65):
    the CFL step and the low-storage RK3 time loop on the GPU."""

    def __init__(self, CFL: float = 0.5, output_times=(1.0,), viscosity: float = 0.0):
        self.CFL_ = CFL
        self.output_times_ = list(output_times)
        self.viscosity_ = viscosity

    @staticmethod
    def get_delta_t(mesh: Mesh2D_t) -> float:
        dt = C.c_double()
        _check(lib().ndg_get_delta_t(mesh.handle, C.byref(dt)))
        return dt.value

    @staticmethod
    def stage(mesh: Mesh2D_t, m: int, time: float, dt: float) -> None:
        _check(lib().ndg_stage(mesh.handle, m, time, dt))

    @staticmethod
    def run(mesh: Mesh2D_t, n_steps: int, time: float = 0.0) -> float:
        t = C.c_double(time)
        _check(lib().ndg_run(mesh.handle, n_steps, C.byref(t)))
        return t.value

    def solve(self, mesh: Mesh2D_t, time: float = 0.0, data_writer: DataWriter_t | None = None,
              output=None) -> tuple[float, int]:
        """Steps to output_times_[-1] with the reference's shortened last step,
        at this solver's CFL. With a data_writer (write_complete_data) or an
        output(time, mesh) callback, outputs come where the reference's
        Solver2D_t::solve (include/solvers/Solver2D_t.tpp:7-133) writes them:
        at the start if the start time is an output time, after the first step
        whose end time t has e <= t < e + dt for an output time e (after an
        error estimate), and at the end if the last step wrote none."""
        _check(lib().ndg_set_cfl(mesh.handle, float(self.CFL_)))
        if data_writer is None and output is None:
            t = C.c_double(time)
            n = C.c_int64()
            _check(lib().ndg_solve(mesh.handle, float(self.output_times_[-1]), C.byref(t), C.byref(n)))
            mesh._refresh_counts()  # the mesh may have been adapted
            return t.value, n.value
        emit = output if output is not None else (lambda tt, m: m.write_complete_data(tt, data_writer))
        t_end = float(self.output_times_[-1])
        dt_mesh = self.get_delta_t(mesh)
        for e in self.output_times_:
            if e <= time < e + dt_mesh:
                emit(time, mesh)
        steps, pending, t_run, wrote_last = 0, 0, time, False

        def flush():
            nonlocal pending, t_run
            if pending:
                t_run = self.run(mesh, pending, t_run)
            pending = 0

        while time < t_end:
            dt = dt_mesh
            last = time + dt > t_end
            if last:
                dt = t_end - time
                flush()
                for m in range(3):
                    self.stage(mesh, m, time, dt)
                t_run = time + dt
            else:
                pending += 1
            time += dt
            steps += 1
            wrote_last = any(e <= time < e + dt for e in self.output_times_)
            if wrote_last:
                flush()
                mesh.estimate_error()
                emit(time, mesh)
            if mesh.adaptivity_interval_ > 0 and steps % mesh.adaptivity_interval_ == 0:
                flush()
                mesh.estimate_error()
                mesh.adapt()
                dt_mesh = self.get_delta_t(mesh)
        flush()
        if not wrote_last:
            mesh.estimate_error()
            emit(time, mesh)
        return time, steps

    def _pre_condition(self, mesh: Mesh2D_t, n_adaptivity_steps: int, pre_condition_interval: int, iterative: int) -> int:
        n = C.c_int64()
        _check(lib().ndg_set_cfl(mesh.handle, float(self.CFL_)))
        _check(lib().ndg_pre_condition(mesh.handle, n_adaptivity_steps, pre_condition_interval, iterative, C.byref(n)))
        mesh._refresh_counts()
        return n.value

    # Solver2D_t::pre_condition / pre_condition_iterative (include/solvers/Solver2D_t.tpp:136-334)
    def pre_condition(self, mesh: Mesh2D_t, n_adaptivity_steps: int, pre_condition_interval: int) -> int:
        """Steps and adapts n_adaptivity_steps times, every
        pre_condition_interval steps, then sets the initial conditions on the
        adapted mesh. Returns the number of steps."""
        return self._pre_condition(mesh, n_adaptivity_steps, pre_condition_interval, 0)

    def pre_condition_iterative(self, mesh: Mesh2D_t, n_adaptivity_steps: int, pre_condition_interval: int) -> int:
        """As pre_condition, with the initial conditions set again (and the
        time restarted) after every adaptation."""
        return self._pre_condition(mesh, n_adaptivity_steps, pre_condition_interval, 1)


class Adjoint2D_t:
    """Discrete adjoint of the variable-speed wave operator on a mesh of one
    order (ndg_adjoint_*): forward solve with receivers and a misfit, its
    exact gradient with respect to the initial fields and the per-element
    wave speed, and the operator with its transpose.

    The mesh must not be adapted while the adjoint exists."""

    def __init__(self, mesh: Mesh2D_t, receivers_xy=None, speed=None, precision: int = FP64):
        xy = np.ascontiguousarray(np.zeros((0, 2)) if receivers_xy is None else receivers_xy, dtype=np.float64).reshape(-1, 2)
        self.mesh = mesh
        self.n_receivers = xy.shape[0]
        self.n_elements = mesh.n_elements_
        self.field_size = mesh.field_size
        h = C.c_void_p()
        _check(lib().ndg_adjoint_create(mesh.handle, self.n_receivers, _ptr(xy) if xy.size else None, C.byref(h)))
        self.h = h
        self.serial = 0  # changes with every forward solve and speed update
        if precision != FP64:
            _check(lib().ndg_adjoint_set_precision(h, precision))
        if speed is not None:
            self.set_speed(speed)

    def set_speed(self, c) -> None:
        c = np.ascontiguousarray(c, dtype=np.float64).ravel()
        if c.size != self.n_elements:
            raise ValueError(f"expected {self.n_elements} speeds, got {c.size}")
        _check(lib().ndg_adjoint_set_speed(self.h, _ptr(c)))
        self.serial += 1

    def delta_t(self, cfl: float) -> float:
        dt = C.c_double()
        _check(lib().ndg_adjoint_delta_t(self.h, cfl, C.byref(dt)))
        return dt.value

    def receivers(self) -> tuple[np.ndarray, np.ndarray]:
        """Element and (xi, eta) of every receiver."""
        el = np.empty(max(self.n_receivers, 1), dtype=np.int64)
        xe = np.empty(max(2 * self.n_receivers, 1))
        _check(lib().ndg_adjoint_receivers(self.h, _ptr(el), _ptr(xe)))
        return el[:self.n_receivers], xe[:2 * self.n_receivers].reshape(-1, 2)

    def _field(self, a):
        if a is None:
            return None, None
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        if a.size != self.field_size:
            raise ValueError(f"expected {self.field_size} values, got {a.size}")
        return a, _ptr(a)

    def forward(self, p0, dt: float, n_steps: int, targets=None, u0=None, v0=None, checkpoint_interval: int = 0) -> tuple[float, np.ndarray]:
        """Misfit J and the receivers' pressure, shape (n_steps + 1, n_receivers)."""
        p0, pp = self._field(p0)
        u0, pu = self._field(u0)
        v0, pv = self._field(v0)
        R = self.n_receivers
        tg = None
        if targets is not None:
            tg = np.ascontiguousarray(targets, dtype=np.float64).reshape(n_steps + 1, R)
        samples = np.empty((n_steps + 1, max(R, 1)))
        J = C.c_double()
        self.serial += 1
        _check(lib().ndg_adjoint_forward(self.h, pp, pu, pv, None if tg is None else _ptr(tg), dt, n_steps, checkpoint_interval,
                                         _ptr(samples), C.byref(J)))
        return J.value, samples[:, :R]

    def backward(self) -> dict:
        """Gradients of the last forward's misfit: p0, u0, v0 and c."""
        g = {k: np.empty(self.field_size) for k in ("p0", "u0", "v0")}
        g["c"] = np.empty(self.n_elements)
        _check(lib().ndg_adjoint_backward(self.h, *[_ptr(g[k]) for k in ("p0", "u0", "v0", "c")]))
        return g

    def operator(self, x, y) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(L(c) x, L(c)^T y, d(y . L(c) x)/dc) for states of 3 field_size values."""
        x = np.ascontiguousarray(x, dtype=np.float64).ravel()
        y = np.ascontiguousarray(y, dtype=np.float64).ravel()
        if x.size != 3 * self.field_size or y.size != 3 * self.field_size:
            raise ValueError("x and y hold p, u and v")
        Lx, LTy, dc = np.empty_like(x), np.empty_like(y), np.empty(self.n_elements)
        _check(lib().ndg_adjoint_operator(self.h, _ptr(x), _ptr(y), _ptr(Lx), _ptr(LTy), _ptr(dc)))
        return Lx, LTy, dc

    def timings(self) -> dict:
        f, b = C.c_double(), C.c_double()
        lf, lb = C.c_int64(), C.c_int64()
        _check(lib().ndg_adjoint_timings(self.h, C.byref(f), C.byref(b), C.byref(lf), C.byref(lb)))
        return {"forward_ms": f.value, "backward_ms": b.value, "forward_launches": lf.value, "backward_launches": lb.value}

    def time_stage(self, which: int, n_launches: int) -> float:
        """Mean kernel duration in ms: 0 forward stage, 1 forward stage
        keeping its input, 2 adjoint stage (after a forward and a backward)."""
        ms = C.c_double()
        _check(lib().ndg_adjoint_time_stage(self.h, which, n_launches, C.byref(ms)))
        return ms.value

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().ndg_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def delta_t_from_device(delta_xy_min: int, elem_N: int, n_elements: int, cfl: float, stream: int = 0) -> float:
    """CFL step from device arrays (float64 delta_xy_min, int32 N per element)
    given by address, without allocating: ndg_delta_t_from_device."""
    dt = C.c_double()
    _check(lib().ndg_delta_t_from_device(delta_xy_min, elem_N, n_elements, cfl, stream or None, C.byref(dt)))
    return dt.value


def dof_count(mesh: Mesh2D_t) -> int:
    """Degrees of freedom 3 * sum (N+1)^2 over elements and instances."""
    return 3 * mesh.field_size * mesh.n_instances


