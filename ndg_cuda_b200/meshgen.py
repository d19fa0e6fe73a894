"""Uniform quad zones in the reference's CGNS layout (the tests, the
benchmark and the workload cases build their meshes with it).

Restates the reference's extras/mesh_generator/main.cpp:159-392: nodes on an
(res+1)^2 lattice numbered x-major, QUAD_4 elements in Hilbert order (or
row-major, for resolutions that are not powers of two), then four BAR_2 ghost
sections (bottom, right, top, left), boundary conditions on the non-periodic
sides and Abutting1to1 self-connectivity on the periodic ones.

A zone is a plain dict of numpy arrays and lists; the library
(`Mesh2D_t(zone, ...)`) and the CPU checkers take exactly this description.
"""
from __future__ import annotations

import numpy as np

WALL, SYMMETRY, INFLOW, OUTFLOW, NULL = 0, 1, 2, 3, 4
QUAD_4, BAR_2 = 0, 1


def hilbert_d2xy(n: int, d: int) -> tuple[int, int]:
    """Hilbert index -> (x, y) on an n x n grid (src/functions/Hilbert.cpp:17-29)."""
    x = y = 0
    s = 1
    while s < n:
        rx = 1 & (d // 2)
        ry = 1 & (d ^ rx)
        if ry == 0:
            if rx == 1:
                x = s - 1 - x
                y = s - 1 - y
            x, y = y, x
        x += s * rx
        y += s * ry
        d //= 4
        s *= 2
    return x, y


def uniform_zone(res: int, x_min: float = -1.0, x_max: float = 1.0, y_min: float = -1.0, y_max: float = 1.0,
                 boundary: int = WALL, x_periodic: bool = False, y_periodic: bool = False,
                 order: str = "hilbert", jitter: float = 0.0, seed: int = 0) -> dict:
    """One zone of res x res quads (extras/mesh_generator/main.cpp:159-392).

    `order` is "hilbert" (the reference generator; res must be a power of two)
    or "rowmajor". `jitter` moves interior nodes by U(-jitter*h, jitter*h) per
    axis, drawn from numpy's PCG64 with `seed`; nodes on the domain boundary
    stay put so periodic seams keep matching.
    """
    if order == "hilbert" and (res <= 0 or res & (res - 1)):
        raise ValueError("Hilbert element order needs a power-of-two resolution")
    xr = yr = res
    xnr, ynr = xr + 1, yr + 1
    n_el = xr * yr
    x = np.empty(xnr * ynr)
    y = np.empty(xnr * ynr)
    for i in range(xnr):
        for j in range(ynr):
            x[i * ynr + j] = x_min + i * (x_max - x_min) / (xnr - 1)
            y[i * ynr + j] = y_min + j * (y_max - y_min) / (ynr - 1)
    if jitter > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        hx = (x_max - x_min) / xr
        hy = (y_max - y_min) / yr
        dx = rng.uniform(-jitter * hx, jitter * hx, size=(xnr, ynr))
        dy = rng.uniform(-jitter * hy, jitter * hy, size=(xnr, ynr))
        for i in range(1, xnr - 1):
            for j in range(1, ynr - 1):
                x[i * ynr + j] += dx[i, j]
                y[i * ynr + j] += dy[i, j]

    quads = np.empty(4 * n_el, dtype=np.int64)
    for i in range(n_el):
        if order == "hilbert":
            ex, ey = hilbert_d2xy(res, i)
        else:
            ex, ey = i % xr, i // xr
        quads[4 * i + 0] = ynr * (ex + 1) + ey + 1
        quads[4 * i + 1] = ynr * (ex + 1) + ey + 2
        quads[4 * i + 2] = ynr * ex + ey + 2
        quads[4 * i + 3] = ynr * ex + ey + 1

    bottom = np.empty(2 * xr, dtype=np.int64)
    for i in range(xr):
        bottom[2 * i] = (i + 1) * ynr + 1
        bottom[2 * i + 1] = i * ynr + 1
    right = np.empty(2 * yr, dtype=np.int64)
    for j in range(yr):
        right[2 * j] = ynr * (xnr - 1) + j + 2
        right[2 * j + 1] = ynr * (xnr - 1) + j + 1
    top = np.empty(2 * xr, dtype=np.int64)
    for i in range(xr):
        top[2 * i] = (xr - i) * ynr
        top[2 * i + 1] = (xr - i + 1) * ynr
    left = np.empty(2 * yr, dtype=np.int64)
    for j in range(yr):
        left[2 * j] = yr - j
        left[2 * j + 1] = yr - j + 1

    b_start, b_end = n_el + 1, n_el + xr
    r_start, r_end = n_el + xr + 1, n_el + xr + yr
    t_start, t_end = n_el + xr + yr + 1, n_el + 2 * xr + yr
    l_start, l_end = n_el + 2 * xr + yr + 1, n_el + 2 * xr + 2 * yr
    sections = [
        ("Elements", QUAD_4, 1, n_el, quads),
        ("BottomElements", BAR_2, b_start, b_end, bottom),
        ("RightElements", BAR_2, r_start, r_end, right),
        ("TopElements", BAR_2, t_start, t_end, top),
        ("LeftElements", BAR_2, l_start, l_end, left),
    ]
    bocos = []
    if not y_periodic:
        bocos.append(("BottomBoundary", boundary, np.arange(b_start, b_start + xr, dtype=np.int64)))
        bocos.append(("TopBoundary", boundary, np.arange(t_start, t_start + xr, dtype=np.int64)))
    if not x_periodic:
        bocos.append(("RightBoundary", boundary, np.arange(r_start, r_start + yr, dtype=np.int64)))
        bocos.append(("LeftBoundary", boundary, np.arange(l_start, l_start + yr, dtype=np.int64)))
    conns = []
    if y_periodic:
        eb = np.array([b_start + i for i in range(xr)], dtype=np.int64)
        et = np.array([t_end - i for i in range(xr)], dtype=np.int64)
        conns.append(("YPeriodicBottom", eb, et))
        conns.append(("YPeriodicTop", et, eb))
    if x_periodic:
        er = np.array([r_start + j for j in range(yr)], dtype=np.int64)
        el = np.array([l_end - j for j in range(yr)], dtype=np.int64)
        conns.append(("XPeriodicRight", er, el))
        conns.append(("XPeriodicLeft", el, er))
    return {"x": x, "y": y, "sections": sections, "bocos": bocos, "conns": conns, "res": res}


def flatten(zone: dict) -> dict:
    """Concatenated arrays of a zone, the layout of the C entry points."""
    secs = zone["sections"]
    out = {
        "n_nodes": len(zone["x"]),
        "x": np.ascontiguousarray(zone["x"], dtype=np.float64),
        "y": np.ascontiguousarray(zone["y"], dtype=np.float64),
        "sec_type": np.array([s[1] for s in secs], dtype=np.int32),
        "sec_start": np.array([s[2] for s in secs], dtype=np.int64),
        "sec_end": np.array([s[3] for s in secs], dtype=np.int64),
        "sec_conn": np.concatenate([np.asarray(s[4], dtype=np.int64) for s in secs]) if secs else np.zeros(0, np.int64),
        "boco_type": np.array([b[1] for b in zone["bocos"]], dtype=np.int32),
        "boco_count": np.array([len(b[2]) for b in zone["bocos"]], dtype=np.int64),
        "boco_points": np.concatenate([b[2] for b in zone["bocos"]]) if zone["bocos"] else np.zeros(0, np.int64),
        "conn_count": np.array([len(c[1]) for c in zone["conns"]], dtype=np.int64),
        "conn_points": np.concatenate([c[1] for c in zone["conns"]]) if zone["conns"] else np.zeros(0, np.int64),
        "conn_donors": np.concatenate([c[2] for c in zone["conns"]]) if zone["conns"] else np.zeros(0, np.int64),
    }
    return out


def write_su2(path, zone: dict, markers: dict) -> None:
    """Writes the zone's quads and the given {tag: bar sections} as SU2 (0-based)."""
    quads = zone["sections"][0][4].reshape(-1, 4) - 1
    with open(path, "w") as f:
        f.write("NDIME= 2\n")
        f.write(f"NPOIN= {zone['x'].size}\n")
        for x, y in zip(zone["x"], zone["y"]):
            f.write(f"{x:.17g} {y:.17g}\n")
        f.write(f"NELEM= {len(quads)}\n")
        for q in quads:
            f.write("9 " + " ".join(str(v) for v in q) + "\n")
        f.write(f"NMARK= {len(markers)}\n")
        for tag, bars in markers.items():
            f.write(f"MARKER_TAG= {tag}\nMARKER_ELEMS= {len(bars)}\n")
            for b in bars:
                f.write(f"3 {b[0]} {b[1]}\n")


def su2_markers(zone: dict) -> dict:
    """SU2 markers of a non-periodic zone: one boundary kind per square side
    (bottom wall, right farfield, top symmetry, left inlet)."""
    bars = [s[4].reshape(-1, 2) - 1 for s in zone["sections"][1:]]  # bottom, right, top, left
    return {"wall": bars[0], "farfield": bars[1], "symmetry": bars[2], "inlet": bars[3]}
