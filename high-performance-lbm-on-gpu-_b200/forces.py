"""Momentum-exchange force on a body as a linear functional of the stored state.

For a link from fluid node x into the body (i into the body, j = opp(i))::

    F_body = sum_links c_i [ f*_i(x, t) + f_j(x, t + 1) ]

with full populations; f_j(t+1) is the plain bounce-back value or the link's
rule (reference ``src/lbm/forces.py:47-103``). Shifted storage adds 2 w_i per
link. ``ForceProbe.evaluate`` hands the functional to the solver, whose CUDA
path gathers and reduces it in float64 on the device (``affine_reduce_kernel`` in
``csrc/aux.cu``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .geometry import WallLinks
from .link_rules import AffineSet, _term_destinations, compile_affine


@dataclass(frozen=True, eq=False)
class ForceProbe:
    params: object
    weight: np.ndarray
    """(n_links, d): c_i of each link, pointing into the body."""
    values: AffineSet
    _compiled: dict = field(default_factory=dict, repr=False)

    @staticmethod
    def build(params, links: WallLinks) -> ForceProbe:
        """The momentum-exchange functional of ``links``, one row per link, in the reference's row
        layout (``forces.py:47-88``): term 0 is f*_i(x) (i = opp j, coefficient 1); then, for a link
        with a rule, the rule's nonzero terms in order and its constant, else plain bounce-back's
        second f*_i(x) and the moving-wall term 6 w_j (c_j . u_w(x - c_j)); every row's constant
        starts with 2 w_i (shifted storage). Rows are padded with zero terms to the widest.

        Built for all links at once: links are matched to rules by the key node * q + direction.
        """
        lattice = params.lattice
        q = lattice.q
        opp = np.asarray(lattice.opposite, dtype=np.int64)
        w = np.asarray(lattice.w, dtype=np.float64)
        cvec = np.asarray(lattice.c, dtype=np.float64)
        x = np.asarray(links.node, dtype=np.int64)
        j = np.asarray(links.direction, dtype=np.int64)
        n = x.size
        i = opp[j]
        # the rule (if any) of each link
        rule = np.full(n, -1, dtype=np.int64)
        rules = params.link_rules
        width = 1
        if rules is not None and len(rules):
            v = rules.values
            rkey = np.asarray(rules.node, dtype=np.int64) * q + np.asarray(rules.direction, dtype=np.int64)
            order = np.argsort(rkey, kind="stable")
            pos = np.searchsorted(rkey[order], x * q + j)
            pos = np.minimum(pos, rkey.size - 1)
            found = rkey[order][pos] == x * q + j
            rule = np.where(found, order[pos], -1)
            # each rule's nonzero terms packed to the front, in order
            coeff = np.asarray(v.coeff, dtype=np.float64)
            live = coeff != 0.0
            pack = np.argsort(~live, axis=1, kind="stable")
            r_dir = np.take_along_axis(np.asarray(v.direction, dtype=np.int64), pack, axis=1)
            r_node = np.take_along_axis(np.asarray(v.node, dtype=np.int64), pack, axis=1)
            r_coeff = np.take_along_axis(coeff, pack, axis=1)
            r_live = np.take_along_axis(live, pack, axis=1)
            r_count = live.sum(axis=1)
            has = rule >= 0
            if np.any(has):
                width = max(width, int(r_count[rule[has]].max()))
        m = 1 + width if n else 1  # (no links: one padding column, as an empty row list gives)
        direction = np.zeros((n, m), dtype=np.int64)
        node = np.zeros((n, m), dtype=np.int64)
        coeffs = np.zeros((n, m))
        direction[:, 0], node[:, 0], coeffs[:, 0] = i, x, 1.0
        const = 2.0 * w[i]
        plain = rule < 0
        direction[plain, 1], node[plain, 1], coeffs[plain, 1] = i[plain], x[plain], 1.0
        if np.any(plain):
            walls = np.asarray(params.wall_velocity, dtype=np.float64).reshape(lattice.d, -1)
            src = _term_destinations(lattice, opp[j[plain]], x[plain], params.shape)  # x - c_j = x + c_opp(j)
            cu = cvec[j[plain], 0] * walls[0][src]
            for a in range(1, lattice.d):
                cu = cu + cvec[j[plain], a] * walls[a][src]
            const[plain] = const[plain] + 6.0 * w[j[plain]] * cu
        if np.any(~plain):
            r = rule[~plain]
            cols = min(width, r_dir.shape[1])
            keep = r_live[r, :cols]
            direction[~plain, 1:1 + cols] = np.where(keep, r_dir[r, :cols], 0)
            node[~plain, 1:1 + cols] = np.where(keep, r_node[r, :cols], 0)
            coeffs[~plain, 1:1 + cols] = np.where(keep, r_coeff[r, :cols], 0.0)
            const[~plain] = const[~plain] + np.asarray(rules.values.constant, dtype=np.float64)[r]
        weight = -cvec[j].reshape(-1, lattice.d)
        return ForceProbe(params=params, weight=weight, values=AffineSet(direction, node, coeffs, const))

    def compiled(self, layout: str):
        if layout not in self._compiled:
            p = self.params
            self._compiled[layout] = compile_affine(p.lattice, self.values, layout, p.solid, p.wall_velocity)
        return self._compiled[layout]

    def evaluate(self, solver) -> np.ndarray:
        """Force on the body (d,), host float64. On this package's CUDA solver the terms are
        resolved to its buffers and reduced on the device (``reduce_affine_values``); on any other
        solver of the reference's contract, ``weight.T @ evaluate_affine(compiled(layout))``."""
        if solver.params is not self.params:
            raise ValueError("this probe was built for a different SimulationParams")
        reduce = getattr(solver, "reduce_affine_values", None)
        if reduce is not None:
            return reduce(self.values, self.weight)
        return self.weight.T @ solver.evaluate_affine(self.compiled(solver.state_layout))
