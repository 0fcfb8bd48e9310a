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

from .geometry import WallLinks, neighbour_index
from .link_rules import AffineSet, compile_affine


@dataclass(frozen=True, eq=False)
class ForceProbe:
    params: object
    weight: np.ndarray
    """(n_links, d): c_i of each link, pointing into the body."""
    values: AffineSet
    _compiled: dict = field(default_factory=dict, repr=False)

    @staticmethod
    def build(params, links: WallLinks) -> ForceProbe:
        lattice = params.lattice
        shape = params.shape
        opp = np.asarray(lattice.opposite)
        w = np.asarray(lattice.w)
        c = np.asarray(lattice.c, dtype=np.float64)
        rules = params.link_rules
        rule_of = {}
        if rules is not None:
            rule_of = {
                (int(x), int(j)): r
                for r, (x, j) in enumerate(zip(np.asarray(rules.node), np.asarray(rules.direction), strict=True))
            }
        walls = np.asarray(params.wall_velocity).reshape(lattice.d, -1)
        rows, constants = [], []
        for x, j in zip(np.asarray(links.node).tolist(), np.asarray(links.direction).tolist(), strict=True):
            i = int(opp[j])
            row = [(i, x, 1.0)]
            const = 2.0 * w[i]
            r = rule_of.get((x, j))
            if r is None:
                src = int(neighbour_index([x], [-v for v in lattice.c[j]], shape)[0])
                row.append((i, x, 1.0))
                const += 6.0 * w[j] * float(c[j] @ walls[:, src])
            else:
                v = rules.values
                for k, y, a in zip(v.direction[r], v.node[r], v.coeff[r], strict=True):
                    if a != 0.0:
                        row.append((int(k), int(y), float(a)))
                const += float(v.constant[r])
            rows.append(row)
            constants.append(const)
        weight = -np.asarray([lattice.c[j] for j in np.asarray(links.direction)], dtype=np.float64)
        return ForceProbe(params=params, weight=weight.reshape(-1, lattice.d), values=AffineSet.from_lists(rows, constants))

    def compiled(self, layout: str):
        if layout not in self._compiled:
            p = self.params
            self._compiled[layout] = compile_affine(p.lattice, self.values, layout, p.solid, p.wall_velocity)
        return self._compiled[layout]

    def evaluate(self, solver) -> np.ndarray:
        """Force on the body (d,), host float64."""
        if solver.params is not self.params:
            raise ValueError("this probe was built for a different SimulationParams")
        reduce = getattr(solver, "reduce_affine", None)
        if reduce is not None:
            return reduce(self.compiled(solver.state_layout), self.weight)
        return self.weight.T @ solver.evaluate_affine(self.compiled(solver.state_layout))
