"""Affine link rules: boundaries that set a streamed population from post-collision ones.

A rule sets the population arriving at fluid node x from a resting solid
neighbour x - c_j to an affine combination of post-collision populations of
the previous step (reference ``src/lbm/link_rules.py:1-40``)::

    f_j(x, t+1) = b + sum_m a_m f*_{k_m}(y_m, t)

The data classes (``AffineSet``, ``LinkRules``, ``CompiledAffine``) and the
slot layouts keep the reference's meaning, because force probes and
user-built rules cross the boundary between the two code bases:

=============  ==========================================  ==================
layout         slot of f*_k(y)                             used for
=============  ==========================================  ==================
``reference``  (k, y)                                      NumPy oracle
``pull``       (k, y)                                      two-lattice state
``aa_odd``     (opp k, y)                                  AA, before odd step
``aa_even``    (k, y + c_k); (opp k, y) if y + c_k solid   AA, before even step
=============  ==========================================  ==================

Slot index = k * n_nodes + node (unpadded). The CUDA solver applies rules
inside its boundary warps (``csrc/step_kernels.cuh``) instead of a pre-pass;
``CudaSolver._build_special`` turns them into its per-node device tables.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geometry import WallLinks, neighbour_index
from .lattice import VelocitySet

LAYOUTS = ("reference", "pull", "aa_odd", "aa_even")


@dataclass(frozen=True)
class AffineSet:
    """n affine expressions padded to m terms (reference ``link_rules.py:54-103``).

    value_r = constant[r] + sum_t coeff[r, t] * f*_{direction[r, t]}(node[r, t]);
    padding terms have coefficient 0.
    """

    direction: np.ndarray
    node: np.ndarray
    coeff: np.ndarray
    constant: np.ndarray

    def __len__(self) -> int:
        return len(self.constant)

    @property
    def terms(self) -> int:
        return self.coeff.shape[1]

    @staticmethod
    def from_lists(rows, constant=None) -> AffineSet:
        n = len(rows)
        m = max((len(r) for r in rows), default=1)
        direction = np.zeros((n, m), dtype=np.int64)
        node = np.zeros((n, m), dtype=np.int64)
        coeff = np.zeros((n, m))
        for r, row in enumerate(rows):
            if row:
                k, y, a = zip(*row, strict=True)
                direction[r, : len(row)] = k
                node[r, : len(row)] = y
                coeff[r, : len(row)] = a
        const = np.zeros(n) if constant is None else np.asarray(constant, dtype=np.float64)
        return AffineSet(direction, node, coeff, const)

    @staticmethod
    def from_dense(direction, node, coeff, constant) -> AffineSet:
        return AffineSet(
            np.asarray(direction, dtype=np.int64),
            np.asarray(node, dtype=np.int64),
            np.asarray(coeff, dtype=np.float64),
            np.asarray(constant, dtype=np.float64),
        )

    @staticmethod
    def concat(*sets: AffineSet) -> AffineSet:
        sets = tuple(s for s in sets if len(s))
        if not sets:
            return AffineSet.from_lists([])
        m = max(s.terms for s in sets)

        def widen(a):
            return np.pad(a, ((0, 0), (0, m - a.shape[1])))

        return AffineSet(
            np.concatenate([widen(s.direction) for s in sets]),
            np.concatenate([widen(s.node) for s in sets]),
            np.concatenate([widen(s.coeff) for s in sets]),
            np.concatenate([s.constant for s in sets]),
        )


@dataclass(frozen=True)
class LinkRules:
    """Rules f_j(x, t+1) = values[r] for links (node[r], direction[r])."""

    node: np.ndarray
    direction: np.ndarray
    values: AffineSet

    def __post_init__(self) -> None:
        if not (len(self.node) == len(self.direction) == len(self.values)):
            raise ValueError("node, direction and values must have the same length")
        if len(self.node):
            keys = np.asarray(self.node, dtype=np.int64) * 64 + np.asarray(self.direction)
            if np.unique(keys).size != keys.size:
                raise ValueError("a link has more than one rule")

    def __len__(self) -> int:
        return len(self.node)

    @staticmethod
    def concat(*rules: LinkRules) -> LinkRules:
        rules = tuple(r for r in rules if r is not None)
        return LinkRules(
            np.concatenate([r.node for r in rules]).astype(np.int64),
            np.concatenate([r.direction for r in rules]).astype(np.int64),
            AffineSet.concat(*(r.values for r in rules)),
        )

    def validate(self, lattice: VelocitySet, solid: np.ndarray, wall_velocity: np.ndarray) -> None:
        """Every rule must sit on a fluid-to-resting-solid link (``link_rules.py:133-148``)."""
        shape = solid.shape
        flat = np.asarray(solid, dtype=bool).ravel()
        direction = np.asarray(self.direction)
        if np.any(direction >= lattice.q) or np.any(direction < 0):
            raise ValueError(f"rule directions must be in [0, {lattice.q})")
        if np.any(flat[self.node]):
            raise ValueError("link rules must target fluid nodes")
        walls = np.asarray(wall_velocity).reshape(lattice.d, -1)
        for j in np.unique(direction):
            nodes = np.asarray(self.node)[direction == j]
            src = neighbour_index(nodes, [-v for v in lattice.c[j]], shape)
            if not np.all(flat[src]):
                raise ValueError(f"a rule for direction {j} does not start at a solid node")
            if np.abs(walls[:, src]).max(initial=0.0) > 0:
                raise ValueError("link rules are only allowed next to solid nodes at rest")


def bouzidi_rules(lattice: VelocitySet, links: WallLinks, solid: np.ndarray) -> LinkRules:
    """Linear interpolated bounce-back (Bouzidi, Firdaouss & Lallemand 2001).

    Same rule set as the reference builder (``link_rules.py:154-188``); with
    i = opp(j)::

        q <  1/2:  f_j(x) = 2q f*_i(x) + (1 - 2q) f*_i(x + c_j)
        q >= 1/2:  f_j(x) = f*_i(x) / (2q) + (1 - 1/(2q)) f*_j(x)

    A q < 1/2 link whose x + c_j is solid keeps plain bounce-back (no rule).
    """
    shape = solid.shape
    flat = np.asarray(solid, dtype=bool).ravel()
    x = np.asarray(links.node, dtype=np.int64)
    j = np.asarray(links.direction, dtype=np.int64)
    q = np.asarray(links.q, dtype=np.float64)
    i = np.asarray(lattice.opposite)[j]
    behind = np.empty_like(x)
    for jj in np.unique(j):
        sel = j == jj
        behind[sel] = neighbour_index(x[sel], lattice.c[jj], shape)
    near = q < 0.5
    keep = ~(near & flat[behind])
    n = int(keep.sum())
    direction = np.zeros((n, 2), dtype=np.int64)
    node = np.zeros((n, 2), dtype=np.int64)
    coeff = np.zeros((n, 2))
    xk, jk, ik, qk, bk, nk = x[keep], j[keep], i[keep], q[keep], behind[keep], near[keep]
    direction[:, 0] = ik
    node[:, 0] = xk
    direction[:, 1] = np.where(nk, ik, jk)
    node[:, 1] = np.where(nk, bk, xk)
    coeff[:, 0] = np.where(nk, 2.0 * qk, 0.5 / qk)
    coeff[:, 1] = np.where(nk, 1.0 - 2.0 * qk, 1.0 - 0.5 / qk)
    return LinkRules(xk.copy(), jk.copy(), AffineSet.from_dense(direction, node, coeff, np.zeros(n)))


@dataclass(frozen=True)
class CompiledAffine:
    """An ``AffineSet`` resolved to flat slots of one memory layout (host arrays)."""

    slots: np.ndarray
    coeff: np.ndarray
    constant: np.ndarray


@dataclass(frozen=True)
class CompiledRules:
    target: np.ndarray
    values: CompiledAffine


def _term_destinations(lattice, k, y, shape):
    """Flat index of y + c_k (periodic) for every term at once; k, y of any common shape."""
    c = np.asarray(lattice.c, dtype=np.int64)[k]  # (..., d), components x, y[, z]
    coords = np.unravel_index(y, shape)           # (z,) y, x
    d = len(shape)
    moved = tuple((coords[a] + c[..., d - 1 - a]) % shape[a] for a in range(d))
    return np.ravel_multi_index(moved, shape)


def compile_affine(lattice, values: AffineSet, layout: str, solid, wall_velocity) -> CompiledAffine:
    """Resolve every term f*_k(y) of ``values`` to a flat slot of the stored state in ``layout``.

    Same slot semantics as the reference's compiler (``link_rules.py:203-240``; see the layout
    table above), computed for all terms in one pass: ``reference``/``pull`` (k, y); ``aa_odd``
    (opp k, y); ``aa_even`` (k, y + c_k), or, where y + c_k is solid, (opp k, y) -- the odd step
    reflected f*_k(y) there with the moving-wall term 6 w_opp(k) (c_opp(k) . u_w) added, so each
    such term contributes coeff 6 w_k (c_k . u_w(y + c_k)) to its row's constant (summed over the
    row's terms in order). ``CudaSolver`` resolves the same slots on the device for its own
    buffers (``lbm_compile_terms``).
    """
    if layout not in LAYOUTS:
        raise ValueError(f"unknown layout {layout!r}; choose from {LAYOUTS}")
    solid = np.asarray(solid, dtype=bool)
    shape = solid.shape
    n = solid.size
    k = np.asarray(values.direction, dtype=np.int64)
    y = np.asarray(values.node, dtype=np.int64)
    coeff = np.asarray(values.coeff, dtype=np.float64)
    constant = np.array(values.constant, dtype=np.float64, copy=True)
    opp = np.asarray(lattice.opposite, dtype=np.int64)
    if layout in ("reference", "pull"):
        return CompiledAffine(slots=k * n + y, coeff=coeff, constant=constant)
    if layout == "aa_odd":
        return CompiledAffine(slots=opp[k] * n + y, coeff=coeff, constant=constant)
    dest = _term_destinations(lattice, k, y, shape)
    blocked = solid.ravel()[dest]
    slots = np.where(blocked, opp[k] * n + y, k * n + dest)
    walls = np.asarray(wall_velocity, dtype=np.float64).reshape(lattice.d, n)
    c = np.asarray(lattice.c, dtype=np.float64)[k]
    cu = c[..., 0] * walls[0][dest]
    for a in range(1, lattice.d):
        cu = cu + c[..., a] * walls[a][dest]
    w = np.asarray(lattice.w, dtype=np.float64)[k]
    extra = np.where(blocked, coeff * ((6.0 * w) * cu), 0.0)
    for t in range(extra.shape[-1]):
        constant = constant + extra[..., t]
    return CompiledAffine(slots=slots, coeff=coeff, constant=constant)


def compile_targets(lattice, rules: LinkRules, layout: str, n_nodes: int) -> np.ndarray:
    """Slot each rule's value replaces in a separate pre-pass design (the reference's GPU
    kernels, ``link_rules.py:243-250``): the streamed population f_j(x) of the rule's link, which
    a pull state keeps at (opp j, x) before the step and the AA states at (j, x)."""
    if layout not in LAYOUTS:
        raise ValueError(f"unknown layout {layout!r}; choose from {LAYOUTS}")
    j = np.asarray(rules.direction, dtype=np.int64)
    plane = np.asarray(lattice.opposite, dtype=np.int64)[j] if layout == "pull" else j
    return plane * n_nodes + np.asarray(rules.node, dtype=np.int64)


def compile_rules(lattice, rules: LinkRules, layout: str, solid, wall_velocity) -> CompiledRules:
    n_nodes = int(np.prod(np.asarray(solid).shape))
    return CompiledRules(
        target=compile_targets(lattice, rules, layout, n_nodes),
        values=compile_affine(lattice, rules.values, layout, solid, wall_velocity),
    )
