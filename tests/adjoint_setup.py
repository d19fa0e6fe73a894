"""Inputs of the adjoint tests and benchmark leg: per-element wave speeds,
receivers, a Gaussian source and the interpolation weights of the receivers,
all computed from a zone of tests/meshgen.py (seeded, no files).

The adjoint configuration: a wave speed c = 1 + 0.2 tanh(sum of seeded
Gaussian bumps of amplitude +-1 and width 0.3) per element (at its centre),
receivers on a circle of radius 0.7, a Gaussian pressure pulse of width 0.1
at the origin with u = v = 0, and targets recorded from a run with a
perturbed speed.
"""
from __future__ import annotations

import numpy as np

from oracle import pyoracle


def element_corners(zone: dict) -> np.ndarray:
    """(K, 4, 2) corner coordinates of the zone's quads, in element order."""
    x, y = np.asarray(zone["x"]), np.asarray(zone["y"])
    quads = [s for s in zone["sections"] if s[1] == 0]
    conn = np.concatenate([np.asarray(s[4], np.int64).reshape(-1, 4) for s in quads]) - 1
    return np.stack([x[conn], y[conn]], axis=-1)


def element_centres(zone: dict) -> np.ndarray:
    return element_corners(zone).mean(axis=1)


def speed_field(zone: dict, seed: int = 0, n_bumps: int = 8, width: float = 0.3, amplitude: float = 0.2) -> np.ndarray:
    """c = 1 + amplitude tanh(sum_b a_b exp(-|x - x_b|^2 / (2 width^2))), a_b = +-1."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-1.0, 1.0, size=(n_bumps, 2))
    signs = rng.choice([-1.0, 1.0], size=n_bumps)
    xc = element_centres(zone)
    s = np.zeros(len(xc))
    for (bx, by), a in zip(centres, signs):
        s += a * np.exp(-((xc[:, 0] - bx) ** 2 + (xc[:, 1] - by) ** 2) / (2 * width ** 2))
    return 1.0 + amplitude * np.tanh(s)


def circle_receivers(n: int = 16, radius: float = 0.7) -> np.ndarray:
    a = 2 * np.pi * (np.arange(n) + 0.5) / n
    return np.stack([radius * np.cos(a), radius * np.sin(a)], axis=1)


def gauss_nodes(N: int) -> tuple[np.ndarray, np.ndarray]:
    """Legendre-Gauss nodes and barycentric weights of order N (oracle tables)."""
    from oracle.pyoracle import _load_oracle
    lib = _load_oracle()
    nodes, bary = np.empty(N + 1), np.empty(N + 1)
    lib.ndgo_table(N, 2, 0, N, nodes)
    lib.ndgo_table(N, 2, 2, N, bary)
    return nodes, bary


def node_coordinates(zone: dict, N: int) -> tuple[np.ndarray, np.ndarray]:
    """Physical coordinates (K, (N+1)^2) of every element's Gauss nodes,
    node i*(N+1)+j at (xi_i, eta_j) of the bilinear map."""
    cr = element_corners(zone)
    xn, _ = gauss_nodes(N)
    xi, eta = np.meshgrid(xn, xn, indexing="ij")
    xi, eta = xi.ravel(), eta.ravel()
    w = np.stack([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)], axis=1) / 4
    return cr[:, :, 0] @ w.T, cr[:, :, 1] @ w.T


def gaussian_pulse(zone: dict, N: int, sigma: float = 0.1, centre=(0.0, 0.0)) -> np.ndarray:
    X, Y = node_coordinates(zone, N)
    return np.exp(-((X - centre[0]) ** 2 + (Y - centre[1]) ** 2) / (2 * sigma ** 2)).ravel()


def lagrange(nodes: np.ndarray, bary: np.ndarray, t: float) -> np.ndarray:
    d = t - nodes
    hit = np.nonzero(np.abs(d) < 1e-14)[0]
    if hit.size:
        out = np.zeros_like(nodes)
        out[hit[0]] = 1.0
        return out
    v = bary / d
    return v / v.sum()


def receiver_weights(N: int, xi_eta: np.ndarray) -> np.ndarray:
    """(R, (N+1)^2) interpolation weights l_i(xi) l_j(eta)."""
    nodes, bary = gauss_nodes(N)
    if len(xi_eta) == 0:
        return np.zeros((0, (N + 1) ** 2))
    return np.stack([np.outer(lagrange(nodes, bary, a), lagrange(nodes, bary, b)).ravel() for a, b in xi_eta])


def locate_receivers(zone: dict, xy: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """First element containing each point and its reference coordinates
    (Newton on the bilinear map)."""
    cr = element_corners(zone)
    elems, coords = [], []
    if len(xy) == 0:
        return np.zeros(0, np.int64), np.zeros((0, 2))
    lo_all, hi_all = cr.min(axis=1), cr.max(axis=1)
    for px, py in xy:
        inside = (lo_all[:, 0] - 1e-12 <= px) & (px <= hi_all[:, 0] + 1e-12) & (lo_all[:, 1] - 1e-12 <= py) & (py <= hi_all[:, 1] + 1e-12)
        for e in np.nonzero(inside)[0]:
            c = cr[e]
            xi = eta = 0.0
            for _ in range(50):
                w = np.array([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)]) / 4
                fx, fy = w @ c[:, 0] - px, w @ c[:, 1] - py
                dxi = np.array([-(1 - eta), 1 - eta, 1 + eta, -(1 + eta)]) / 4
                deta = np.array([-(1 - xi), -(1 + xi), 1 + xi, 1 - xi]) / 4
                J = np.array([[dxi @ c[:, 0], deta @ c[:, 0]], [dxi @ c[:, 1], deta @ c[:, 1]]])
                d = np.linalg.solve(J, [fx, fy])
                xi, eta = xi - d[0], eta - d[1]
                if abs(d).sum() < 1e-15:
                    break
            if abs(xi) <= 1 + 1e-12 and abs(eta) <= 1 + 1e-12:
                elems.append(int(e))
                coords.append((xi, eta))
                break
        else:
            raise ValueError("receiver outside the mesh")
    return np.array(elems, np.int64), np.array(coords)


def oracle_problem(zone: dict, N: int, speed: np.ndarray, receivers_xy: np.ndarray):
    """An OracleSolver with the speed set, and its receivers (element, weights)."""
    o = pyoracle.OracleSolver(zone, N)
    o.set_speed(speed)
    el, xe = locate_receivers(zone, receivers_xy)
    return o, el, receiver_weights(N, xe)


def cfl_dt(zone: dict, N: int, speed: np.ndarray, cfl: float = 0.5) -> float:
    """min over elements of cfl * delta_xy_min / (N^2 c) on straight-sided quads."""
    cr = element_corners(zone)
    pairs = [(0, 1), (2, 3), (1, 2), (0, 3), (1, 3), (2, 0)]
    dmin = np.min(np.stack([np.hypot(*(cr[:, a] - cr[:, b]).T) for a, b in pairs]), axis=0)
    return float(np.min(cfl * dmin / (N * N * speed)))
