"""Immersed boundary method: direct forcing with multi-direct iterations.

Body description and stencil geometry (reference ``src/lbm/ibm.py:53-120``).
Every time step, before the collision, the CUDA solver

1. gathers density and momentum of the streamed populations at every
   stencil node (moments ``rho``, ``u* = (j + F_uniform/2)/rho``),
2. runs ``iterations`` multi-direct passes, one kernel each:
   ``u = u* + F/(2 rho)``, ``U_l = sum w u``, ``F_l = 2 rho_l (0 - U_l) dA_l``,
   ``F += sum_l w F_l`` (spread),
3. adds the node force F at the stencil nodes in the collision.

The force on the body is ``-sum_iterations sum_l F_l``. The kernels live in
``csrc/ibm.cu``; this module builds their tables (``IbmTables``).

Roma, Peskin & Berger (1999) 3-point kernel, |r| <= 3/2::

    phi(r) = (1 + sqrt(1 - 3 r^2)) / 3                  |r| <= 1/2
    phi(r) = (5 - 3|r| - sqrt(1 - 3 (1 - |r|)^2)) / 6   1/2 <= |r| <= 3/2
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .geometry import Ball, neighbour_index

STENCIL = 3


def roma(r) -> np.ndarray:
    a = np.abs(np.asarray(r, dtype=np.float64))
    near = (1.0 + np.sqrt(np.clip(1.0 - 3.0 * a * a, 0.0, None))) / 3.0
    far = (5.0 - 3.0 * a - np.sqrt(np.clip(1.0 - 3.0 * (1.0 - a) ** 2, 0.0, None))) / 6.0
    return np.where(a <= 0.5, near, np.where(a <= 1.5, far, 0.0))


@dataclass(frozen=True, eq=False)
class ImmersedBoundary:
    """Surface markers (n, d) in node units, their surface elements and the pass count."""

    markers: np.ndarray
    areas: np.ndarray
    iterations: int = 3

    def __post_init__(self) -> None:
        if self.markers.ndim != 2 or self.markers.shape[1] not in (2, 3):
            raise ValueError("markers must have shape (n, 2) or (n, 3)")
        if self.areas.shape != (len(self.markers),):
            raise ValueError("areas must have one entry per marker")
        if self.iterations < 1:
            raise ValueError("iterations must be >= 1")

    @property
    def d(self) -> int:
        return self.markers.shape[1]

    @staticmethod
    def from_ball(ball: Ball, spacing: float = 0.8, iterations: int = 3) -> ImmersedBoundary:
        """Evenly spaced circle markers, or a Fibonacci lattice on a sphere (``ibm.py:88-105``)."""
        r = ball.radius
        centre = np.asarray(ball.center, dtype=np.float64)
        if ball.d == 2:
            n = max(8, math.ceil(2.0 * math.pi * r / spacing))
            theta = 2.0 * math.pi * (np.arange(n) + 0.5) / n
            unit = np.column_stack([np.cos(theta), np.sin(theta)])
            area = 2.0 * math.pi * r / n
        else:
            n = max(32, math.ceil(4.0 * math.pi * r * r / spacing**2))
            k = np.arange(n) + 0.5
            z = 1.0 - 2.0 * k / n
            phi = math.pi * (1.0 + math.sqrt(5.0)) * k
            ring = np.sqrt(1.0 - z * z)
            unit = np.column_stack([ring * np.cos(phi), ring * np.sin(phi), z])
            area = 4.0 * math.pi * r * r / n
        return ImmersedBoundary(centre + r * unit, np.full(n, area), iterations)

    def stencil(self, shape: tuple[int, ...]) -> tuple[np.ndarray, np.ndarray]:
        """Flat node indices and Roma weights, each (n_markers, 3^d)."""
        d = self.d
        base = np.floor(self.markers - 0.5).astype(np.int64)
        grid = np.indices((STENCIL,) * d).reshape(d, -1).T  # (3^d, d) offsets, x slowest
        pts = base[:, None, :] + grid[None, :, :]
        weights = np.prod(roma(pts - self.markers[:, None, :]), axis=-1)
        extent = np.asarray(shape[::-1])
        if np.any(pts < 0) or np.any(pts >= extent):
            raise ValueError("every marker must sit at least 2 nodes inside the domain")
        flat = np.ravel_multi_index(tuple(pts[..., a] for a in range(d - 1, -1, -1)), shape)
        return flat, weights


@dataclass(frozen=True)
class IbmTables:
    """Host tables for the IBM kernels of one body on one grid.

    ``nodes`` unique stencil nodes (ascending flat index); ``stencil`` (n_markers,
    S) positions into ``nodes``; ``weights`` (n_markers, S); inverse map in CSR
    form (``inv_start``, ``inv_marker``, ``inv_weight``) listing, for every
    node, the (marker, weight) pairs that touch it, in ascending
    (marker, stencil position) order.
    """

    nodes: np.ndarray
    stencil: np.ndarray
    weights: np.ndarray
    areas: np.ndarray
    inv_start: np.ndarray
    inv_marker: np.ndarray
    inv_weight: np.ndarray
    iterations: int

    @property
    def n_nodes(self) -> int:
        return self.nodes.size

    @property
    def n_markers(self) -> int:
        return self.stencil.shape[0]


def check_clear_of_walls(lattice, solid: np.ndarray, nodes: np.ndarray) -> None:
    """Stencil nodes and all their neighbours must be fluid (``ibm.py:153-158``)."""
    flat = np.asarray(solid, dtype=bool).ravel()
    for cvec in lattice.c:
        if np.any(flat[neighbour_index(nodes, cvec, solid.shape)]):
            raise ValueError("immersed-boundary stencils must not touch solid nodes")


def build_tables(body, lattice, solid: np.ndarray) -> IbmTables:
    shape = solid.shape
    flat_stencil, weights = body.stencil(shape)
    nodes, inverse = np.unique(flat_stencil, return_inverse=True)
    inverse = inverse.reshape(flat_stencil.shape)
    check_clear_of_walls(lattice, solid, nodes)
    m, s = inverse.shape
    pair_marker = np.repeat(np.arange(m), s)
    pair_node = inverse.reshape(-1)
    order = np.argsort(pair_node, kind="stable")  # stable keeps (marker, position) order per node
    counts = np.bincount(pair_node, minlength=nodes.size)
    start = np.zeros(nodes.size + 1, dtype=np.int64)
    np.cumsum(counts, out=start[1:])
    return IbmTables(
        nodes=nodes.astype(np.int64),
        stencil=inverse.astype(np.int64),
        weights=np.asarray(weights, dtype=np.float64),
        areas=np.asarray(body.areas, dtype=np.float64),
        inv_start=start,
        inv_marker=pair_marker[order].astype(np.int64),
        inv_weight=weights.reshape(-1)[order],
        iterations=int(body.iterations),
    )
