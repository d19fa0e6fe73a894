"""Seeded synthetic inputs of the benchmark workloads (no files, no network):
per-element wave speeds, receivers on a circle, Gaussian pressure pulses at
the elements' Gauss nodes, computed from a zone of ndg_cuda_b200.meshgen.
"""
from __future__ import annotations

import numpy as np


def element_corners(zone: dict) -> np.ndarray:
    """(K, 4, 2) corner coordinates of the zone's quads, in element order."""
    x, y = np.asarray(zone["x"]), np.asarray(zone["y"])
    quads = [s for s in zone["sections"] if s[1] == 0]
    conn = np.concatenate([np.asarray(s[4], np.int64).reshape(-1, 4) for s in quads]) - 1
    return np.stack([x[conn], y[conn]], axis=-1)


def element_centres(zone: dict) -> np.ndarray:
    return element_corners(zone).mean(axis=1)


def speed_field(zone: dict, seed: int = 0, n_bumps: int = 8, width: float = 0.3, amplitude: float = 0.2) -> np.ndarray:
    """c = 1 + amplitude tanh(sum_b a_b exp(-|x - x_b|^2 / (2 width^2))) at
    the element centres, a_b = +-1 and x_b uniform in [-1, 1]^2 (seeded)."""
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


def node_coordinates(zone: dict, N: int) -> tuple[np.ndarray, np.ndarray]:
    """Physical coordinates (K, (N+1)^2) of every element's Legendre-Gauss
    nodes, node i*(N+1)+j at (xi_i, eta_j) of the bilinear map."""
    from . import tables_compute
    cr = element_corners(zone)
    xn = tables_compute(N, 2, "nodes", N)
    xi, eta = np.meshgrid(xn, xn, indexing="ij")
    xi, eta = xi.ravel(), eta.ravel()
    w = np.stack([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)], axis=1) / 4
    return cr[:, :, 0] @ w.T, cr[:, :, 1] @ w.T


def gaussian_pulse(zone: dict, N: int, sigma: float = 0.1, centre=(0.0, 0.0)) -> np.ndarray:
    """exp(-|x - centre|^2 / (2 sigma^2)) at every node, element by element."""
    X, Y = node_coordinates(zone, N)
    return np.exp(-((X - centre[0]) ** 2 + (Y - centre[1]) ** 2) / (2 * sigma ** 2)).ravel()
