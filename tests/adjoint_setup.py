"""Inputs of the adjoint tests: the workload generators of
ndg_cuda_b200.workloads (per-element wave speeds, receivers, Gaussian
sources) and the oracle side (receiver location and interpolation weights,
the oracle's adjoint problem).

The adjoint configuration: a wave speed c = 1 + 0.2 tanh(sum of seeded
Gaussian bumps of amplitude +-1 and width 0.3) per element (at its centre),
receivers on a circle of radius 0.7, a Gaussian pressure pulse of width 0.1
at the origin with u = v = 0, and targets recorded from a run with a
perturbed speed.
"""
from __future__ import annotations

import numpy as np

from ndg_cuda_b200.workloads import (circle_receivers, element_centres, element_corners, gaussian_pulse,  # noqa: F401
                                     node_coordinates, speed_field)
from oracle import pyoracle


def gauss_nodes(N: int) -> tuple[np.ndarray, np.ndarray]:
    """Legendre-Gauss nodes and barycentric weights of order N (oracle tables)."""
    from oracle.pyoracle import _load_oracle
    lib = _load_oracle()
    nodes, bary = np.empty(N + 1), np.empty(N + 1)
    lib.ndgo_table(N, 2, 0, N, nodes)
    lib.ndgo_table(N, 2, 2, N, bary)
    return nodes, bary


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
