"""Body geometry on the lattice: balls, voxelisation, wall-link fractions.

Input builders for link rules and immersed bodies. They follow the reference's
conventions (``src/lbm/geometry.py``): node ``[z, y, x]`` sits at position
(x, y, z); a wall link runs from a fluid node x to a body node x - c_j and
``q`` is the fraction of that link from x to the surface (0 < q <= 1).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .lattice import VelocitySet


@dataclass(frozen=True)
class Ball:
    """Circle (2D) or sphere (3D) (reference ``geometry.py:63-101``)."""

    center: tuple[float, ...]
    radius: float

    def __post_init__(self) -> None:
        if len(self.center) not in (2, 3):
            raise ValueError(f"a ball needs a 2D or 3D centre; got {self.center}")
        if not self.radius > 0:
            raise ValueError(f"radius must be positive; got {self.radius}")
        object.__setattr__(self, "center", tuple(float(v) for v in self.center))

    @property
    def d(self) -> int:
        return len(self.center)

    @property
    def measure(self) -> float:
        return math.pi * self.radius**2 if self.d == 2 else 4.0 / 3.0 * math.pi * self.radius**3

    def contains(self, points: np.ndarray) -> np.ndarray:
        rel = np.asarray(points, dtype=np.float64) - np.asarray(self.center)
        return np.sum(rel * rel, axis=-1) <= self.radius**2

    def ray_fraction(self, origin: np.ndarray, direction: np.ndarray) -> np.ndarray:
        """Smallest root t of |o + t d - c| = R, clipped to (0, 1]."""
        o = np.asarray(origin, dtype=np.float64) - np.asarray(self.center)
        dvec = np.asarray(direction, dtype=np.float64)
        a = np.sum(dvec * dvec, axis=-1)
        b = 2.0 * np.sum(o * dvec, axis=-1)
        k = np.sum(o * o, axis=-1) - self.radius**2
        t = (-b - np.sqrt(np.maximum(b * b - 4.0 * a * k, 0.0))) / (2.0 * a)
        return np.clip(t, np.finfo(np.float64).tiny, 1.0)


def circle(x: float, y: float, radius: float) -> Ball:
    return Ball((x, y), radius)


def sphere(x: float, y: float, z: float, radius: float) -> Ball:
    return Ball((x, y, z), radius)


def node_positions(shape: tuple[int, ...]) -> np.ndarray:
    """(*shape, d) positions, components ordered x, y[, z]."""
    axes = np.meshgrid(*(np.arange(n, dtype=np.float64) for n in shape), indexing="ij")
    return np.stack(axes[::-1], axis=-1)


def voxelize(body, shape: tuple[int, ...]) -> np.ndarray:
    if len(shape) != body.d:
        raise ValueError(f"grid shape {shape} does not match a {body.d}D body")
    return body.contains(node_positions(shape))


def neighbour_index(nodes, c, shape: tuple[int, ...]) -> np.ndarray:
    """Flat index of node + c with periodic wrap (c ordered x, y[, z])."""
    coords = np.unravel_index(np.asarray(nodes, dtype=np.int64), shape)
    moved = tuple((coords[a] + int(s)) % shape[a] for a, s in enumerate(tuple(c)[::-1]))
    return np.ravel_multi_index(moved, shape)


@dataclass(frozen=True)
class WallLinks:
    """Links from fluid nodes into one body: node x, incoming direction j, fraction q."""

    node: np.ndarray
    direction: np.ndarray
    q: np.ndarray

    def __len__(self) -> int:
        return len(self.node)


def wall_links(lattice: VelocitySet, body, solid: np.ndarray) -> WallLinks:
    """Every link from a fluid node into ``body`` (reference ``geometry.py:174-206``).

    Links are grouped by direction j = 1..q-1, nodes ascending within a group.
    """
    solid = np.asarray(solid, dtype=bool)
    shape = solid.shape
    if lattice.d != body.d or len(shape) != body.d:
        raise ValueError(f"{lattice.name}, a {body.d}D body and grid {shape} must agree")
    inside = voxelize(body, shape)
    if np.any(inside & ~solid):
        raise ValueError("every node inside the body must be marked solid")
    fluid_nodes = np.flatnonzero(~solid)
    positions = node_positions(shape).reshape(-1, body.d)
    inside_flat = inside.ravel()
    nodes, dirs, qs = [], [], []
    for j, cj in enumerate(lattice.c):
        if not any(cj):
            continue
        back = neighbour_index(fluid_nodes, [-v for v in cj], shape)
        hit = fluid_nodes[inside_flat[back]]
        if hit.size == 0:
            continue
        step = np.broadcast_to(-np.asarray(cj, dtype=np.float64), (hit.size, body.d))
        nodes.append(hit)
        dirs.append(np.full(hit.size, j, dtype=np.int64))
        qs.append(body.ray_fraction(positions[hit], step))
    if not nodes:
        empty = np.zeros(0, dtype=np.int64)
        return WallLinks(empty, empty.copy(), np.zeros(0))
    return WallLinks(np.concatenate(nodes), np.concatenate(dirs), np.concatenate(qs))


def channel_walls(nx: int, ny: int, nz: int | None = None) -> np.ndarray:
    """Solid first and last y rows (reference ``boundaries.py:81-94``)."""
    if nx <= 0 or ny < 3 or (nz is not None and nz <= 0):
        raise ValueError(f"channel needs nx > 0, ny >= 3, nz > 0; got nx={nx}, ny={ny}, nz={nz}")
    solid = np.zeros((ny, nx) if nz is None else (nz, ny, nx), dtype=bool)
    solid[..., [0, -1], :] = True
    return solid


def cavity_walls(n: int, lid_velocity: float, dimensions: int = 2):
    """Cavity of side n in a one-node solid frame, lid y = n+1 moving in +x (``boundaries.py:97-116``)."""
    if dimensions not in (2, 3):
        raise ValueError(f"cavity dimensions must be 2 or 3; got {dimensions}")
    if n <= 0:
        raise ValueError(f"cavity size must be positive; got n={n}")
    solid = np.ones((n + 2,) * dimensions, dtype=bool)
    solid[(slice(1, -1),) * dimensions] = False
    wall = np.zeros((dimensions, *solid.shape))
    wall[0, ..., -1, :] = lid_velocity
    return solid, wall


def duct_walls(nx: int, ny: int, nz: int) -> np.ndarray:
    """Square duct: solid layers at y = 0, ny-1 and z = 0, nz-1, periodic in x."""
    solid = np.zeros((nz, ny, nx), dtype=bool)
    solid[:, [0, -1], :] = True
    solid[[0, -1], :, :] = True
    return solid
