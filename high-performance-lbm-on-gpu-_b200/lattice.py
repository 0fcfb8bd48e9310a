"""Velocity sets D2Q9 and D3Q19.

The direction numbering and weights are fixed by the reference solver
(``src/lbm/lattice.py:114-146``): slot ``k`` of a population buffer means the
same direction in both code bases, so link rules, force probes and population
snapshots can be exchanged between them. D3Q19 lists every direction next to
its opposite (rest, six axis links, twelve edge links).

The CUDA kernels carry their own copy of these tables in
``csrc/lattice.cuh``; ``tests/test_lattice_tables.py`` checks that both agree.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import cached_property

import numpy as np

CS2 = 1.0 / 3.0
"""Squared lattice speed of sound of both velocity sets."""


@dataclass(frozen=True)
class VelocitySet:
    """A DdQq lattice (mirrors ``VelocitySet`` in ``src/lbm/lattice.py:52-111``).

    ``c`` holds the q integer velocities (x, y[, z]); ``w`` the weights.
    """

    name: str
    d: int
    c: tuple[tuple[int, ...], ...]
    w: tuple[float, ...]
    cs2: float = CS2

    def __post_init__(self) -> None:
        if len(self.c) != len(self.w):
            raise ValueError(f"{self.name}: {len(self.c)} velocities but {len(self.w)} weights")
        if any(len(v) != self.d for v in self.c):
            raise ValueError(f"{self.name}: every velocity must have length d={self.d}")
        if abs(sum(self.w) - 1.0) > 1e-12:
            raise ValueError(f"{self.name}: weights must sum to 1, got {sum(self.w)}")
        reverse = {tuple(-a for a in v) for v in self.c}
        if reverse != set(self.c):
            raise ValueError(f"{self.name}: every velocity needs an opposite")

    @property
    def q(self) -> int:
        return len(self.c)

    @cached_property
    def opposite(self) -> tuple[int, ...]:
        index = {v: i for i, v in enumerate(self.c)}
        return tuple(index[tuple(-a for a in v)] for v in self.c)

    def component(self, axis: int) -> tuple[int, ...]:
        """Components along ``axis`` (0 = x, 1 = y, 2 = z); zeros beyond ``d``."""
        if axis >= self.d:
            return (0,) * self.q
        return tuple(v[axis] for v in self.c)

    @cached_property
    def c_array(self) -> np.ndarray:
        a = np.array(self.c, dtype=np.int64)
        a.setflags(write=False)
        return a

    @cached_property
    def w_array(self) -> np.ndarray:
        a = np.array(self.w, dtype=np.float64)
        a.setflags(write=False)
        return a

    @cached_property
    def c3(self) -> np.ndarray:
        """(q, 3) integer velocities, z column zero in 2D."""
        out = np.zeros((self.q, 3), dtype=np.int64)
        out[:, : self.d] = self.c_array
        return out


def _axis_and_edges_3d() -> tuple[tuple[int, int, int], ...]:
    axis = []
    for a in range(3):
        for s in (1, -1):
            v = [0, 0, 0]
            v[a] = s
            axis.append(tuple(v))
    edges = []
    for a, b in ((0, 1), (0, 2), (1, 2)):
        for sa, sb in ((1, 1), (1, -1)):
            v = [0, 0, 0]
            v[a], v[b] = sa, sb
            edges.append(tuple(v))
            edges.append(tuple(-t for t in v))
    return ((0, 0, 0), *axis, *edges)


D2Q9 = VelocitySet(
    name="D2Q9",
    d=2,
    c=((0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)),
    w=(4.0 / 9.0,) + (1.0 / 9.0,) * 4 + (1.0 / 36.0,) * 4,
)

D3Q19 = VelocitySet(
    name="D3Q19",
    d=3,
    c=_axis_and_edges_3d(),
    w=(1.0 / 3.0,) + (1.0 / 18.0,) * 6 + (1.0 / 36.0,) * 12,
)

LATTICES: dict[str, VelocitySet] = {v.name: v for v in (D2Q9, D3Q19)}


def default_lattice(d: int) -> VelocitySet:
    if d == 2:
        return D2Q9
    if d == 3:
        return D3Q19
    raise ValueError(f"no default lattice for dimension {d}; supported: 2, 3")


def as_lattice(spec) -> VelocitySet:
    """This package's ``VelocitySet`` for a name or any object with ``name``, ``c`` and ``w``.

    Accepting foreign velocity-set objects lets a solver take parameter objects
    built with the reference package unchanged, as long as their tables match.
    """
    if isinstance(spec, VelocitySet):
        return spec
    name = spec if isinstance(spec, str) else getattr(spec, "name", None)
    if name not in LATTICES:
        raise ValueError(f"unknown lattice {name!r}; choose from {tuple(LATTICES)}")
    ours = LATTICES[name]
    if not isinstance(spec, str):
        if tuple(map(tuple, spec.c)) != ours.c or not np.allclose(spec.w, ours.w, rtol=0, atol=1e-15):
            raise ValueError(f"lattice {name} has a different direction order or weights")
    return ours
