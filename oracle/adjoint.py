"""FP64 NumPy adjoint of the LBM step -- TEST INFRASTRUCTURE ONLY.

Discrete adjoint of the oracle's time step (``lbm_oracle.OracleSolver.step``,
itself the reference's ``ReferenceSolver._advance``, ``src/lbm/solver.py:257-274``)
for the loss

    L = (1/M) sum_{t = T-M+1..T} D(f_t),   D(f) = sum_r weight[r, axis] (const_r + sum coeff f[slot])

(a momentum-exchange force component, ``src/lbm/forces.py:98-103``), or
for an immersed body the mean of its body force component over the last M
steps (``src/lbm/ibm.py:189-214``), with respect to the per-node Guo force
field G and the inlet-speed scale U of Zou-He rules whose derivative is given.
The immersed-boundary force enters the collision of its stencil nodes and
depends on the streamed populations there; its vector-Jacobian product is
taken by complex steps through the oracle's own multi-direct passes
(``lbm_oracle._Ibm.force_from_moments``), one step per moment input.

Independent of the CUDA adjoint by construction: the collision Jacobian is
taken by complex-step differentiation of the oracle's own ``collide``
(exact to round-off, no hand derivation), and the transposed streaming is an
explicit scatter-add of the forward pull, bounce-back and rule indices.
"""

from __future__ import annotations

import numpy as np

from .lbm_oracle import OracleSolver, collide, equilibrium, stream_pull

H = 1e-30  # complex step


def _pull_sources(lattice, solid):
    """For every (i, x): flat source slot of s_i(x) when no rule applies."""
    shape = solid.shape
    n = solid.size
    q = lattice.q
    nodes = np.arange(n)
    coords = np.unravel_index(nodes, shape)
    src = np.empty((q, n), dtype=np.int64)
    flat_solid = solid.ravel()
    for i, ci in enumerate(lattice.c):
        moved = tuple((coords[a] - int(s)) % shape[a] for a, s in enumerate(tuple(ci)[::-1]))
        y = np.ravel_multi_index(moved, shape)
        bb = flat_solid[y]
        src[i] = np.where(bb, lattice.opposite[i] * n + nodes, i * n + y)
    return src


class OracleAdjoint:
    """Forward + backward of a fixed number of steps on small grids (float64).

    Args:
        params: float64 parameters (rules included).
        probe: (slots, coeff, constant) of the force probe in the reference layout,
            ``weight`` (n_rows, d) and the force ``axis``; probe None: the loss is
            the immersed body's force component ``axis`` (``weight`` unused).
        window: number M of final steps averaged in the loss.
        force_field: (d, *shape) per-node force (the parameter G).
        d_rules: derivative of ``params.link_rules`` w.r.t. U, same rows and
            term layout (``open_boundaries.zou_he_inlet_derivative``), or None.
    """

    def __init__(self, params, probe, weight, axis, window, force_field, d_rules=None):
        self.params = params
        self.lattice = params.lattice
        self.shape = params.shape
        self.n = int(np.prod(self.shape))
        self.d = self.lattice.d
        self.solid = np.asarray(params.solid, dtype=bool)
        self.fluid = ~self.solid
        self.G = np.asarray(force_field, dtype=np.float64).reshape(self.d, *self.shape)
        self.window = int(window)
        self.axis = int(axis)
        self.dD = np.zeros(self.lattice.q * self.n)
        self.probe = None
        if probe is not None:
            slots, coeff, const = probe
            w = np.asarray(weight, dtype=np.float64)[:, axis]
            np.add.at(self.dD, np.asarray(slots).ravel(), (w[:, None] * np.asarray(coeff)).ravel())
            self.probe = (np.asarray(slots), np.asarray(coeff), np.asarray(const), w)
        elif params.immersed is None:
            raise ValueError("without a force probe the loss is the immersed body's force: params.immersed is None")
        self.src = _pull_sources(self.lattice, self.solid)
        rules = params.link_rules
        self.rules = None
        if rules is not None and len(rules):
            v = rules.values
            target = np.asarray(rules.direction) * self.n + np.asarray(rules.node)
            tslots = np.asarray(v.direction) * self.n + np.asarray(v.node)
            self.rules = (target, tslots, np.asarray(v.coeff, dtype=np.float64))
            if d_rules is not None:
                dv = d_rules.values
                self.d_rules = (np.asarray(dv.direction) * self.n + np.asarray(dv.node),
                                np.asarray(dv.coeff, dtype=np.float64), np.asarray(dv.constant, dtype=np.float64))
            else:
                self.d_rules = None
        self.solver = OracleSolver(params, force_field=self.G)

    def _force(self):
        return tuple(float(self.params.force[a]) + self.G[a] for a in range(self.d))

    def _streamed(self, f):
        s = self.solver
        streamed = stream_pull(self.lattice, f)
        streamed = np.where(s.mask, f[list(self.lattice.opposite)] + s.wall_term, streamed)
        if s.rules is not None:
            target, slots, coeff, const = s.rules
            streamed.reshape(-1)[target] = const + (coeff * f.reshape(-1)[slots]).sum(axis=1)
        return streamed

    def loss_of(self, f) -> float:
        slots, coeff, const, w = self.probe
        values = const + (coeff * f.reshape(-1)[slots]).sum(axis=1)
        return float(w @ values)

    def forward(self, steps: int, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        self.init_fields = (rho, (ux, uy, uz)[: self.d])
        self.solver.initialize(rho, ux, uy, uz)
        self.states = [self.solver.populations()]
        total = 0.0
        for t in range(1, steps + 1):
            self.solver.step()
            self.states.append(self.solver.populations())
            if t > steps - self.window:
                if self.probe is None:
                    total += float(self.solver.ibm.body_force[self.axis])
                else:
                    total += self.loss_of(self.states[-1])
        self.steps = steps
        return total / self.window

    def _vjp_ibm(self, rho, j, a_bar, b_bar):
        """(rho_bar, j_bar) at the stencil nodes from the adjoints of the node force (d, n) and body force (d,)."""
        ibm = self.solver.ibm
        n = rho.size
        jj = np.stack(j).astype(np.complex128)
        r0 = rho.astype(np.complex128)
        bar = np.zeros((1 + self.d, n))
        for m in range(1 + self.d):
            for i in range(n):
                r, jv = r0.copy(), jj.copy()
                if m == 0:
                    r[i] += 1j * H
                else:
                    jv[m - 1, i] += 1j * H
                force, body = ibm.force_from_moments(r, list(jv))
                bar[m, i] = (a_bar * force.imag).sum() / H + float(b_bar @ body.imag) / H
        return bar[0], bar[1:]

    def _vjp_collide(self, s, lam, force=None):
        """mu = J_s^T lam and g = J_F^T lam at every node, by complex steps."""
        q, d = self.lattice.q, self.d
        wp, wm = self.params.relaxation_rates
        force = self._force() if force is None else force
        mu = np.zeros_like(s)
        for k in range(q):
            z = s.astype(np.complex128)
            z[k] += 1j * H
            jac_col = collide(self.lattice, z, wp, wm, force).imag / H  # (q, ...) d f*_i / d s_k
            mu[k] = (lam * jac_col).sum(axis=0)
        g = np.zeros((d, *self.shape))
        for a in range(d):
            fz = tuple((force[b] + 1j * H) if b == a else force[b] for b in range(d))
            jac = collide(self.lattice, s.astype(np.complex128), wp, wm, fz).imag / H
            g[a] = (lam * jac).sum(axis=0)
        return mu, g

    def backward(self):
        """(dL/dU, dL/dG) for the last forward run."""
        q, n, T, M = self.lattice.q, self.n, self.steps, self.window
        lam = self.dD.reshape(q, *self.shape) / M  # dL/df_T
        dG = np.zeros((self.d, *self.shape))
        dU = 0.0
        fluid = self.fluid
        ibm = self.solver.ibm
        for t in range(T - 1, -1, -1):
            f_t = self.states[t]
            s = self._streamed(f_t)
            force = None
            if ibm is not None:
                rho_n, j_n = ibm.moments(f_t)
                field, _ = ibm.force_from_moments(rho_n, j_n)
                force = []
                for a, fa in enumerate(self._force()):
                    full = np.broadcast_to(np.asarray(fa, dtype=np.float64), self.shape).copy()
                    full.reshape(-1)[ibm.nodes] += field[a]
                    force.append(full)
                force = tuple(force)
            mu, g = self._vjp_collide(s, lam, force)
            mu = np.where(fluid, mu, 0.0)
            dG += np.where(fluid, g, 0.0)
            new = np.zeros(q * n)
            # solid nodes keep their values: identity
            new += np.where(self.solid, lam, 0.0).reshape(-1)
            mu_flat = mu.reshape(-1)
            if self.rules is not None:
                target, tslots, coeff = self.rules
                ruled = np.zeros(q * n, dtype=bool)
                ruled[target] = True
                plain = ~ruled
                np.add.at(new, self.src.reshape(-1)[plain], mu_flat[plain])
                np.add.at(new, tslots.ravel(), (coeff * mu_flat[target][:, None]).ravel())
                if self.d_rules is not None:
                    dslots, dcoeff, dconst = self.d_rules
                    dvals = dconst + (dcoeff * f_t.reshape(-1)[dslots]).sum(axis=1)
                    dU += float(mu_flat[target] @ dvals)
            else:
                np.add.at(new, self.src.reshape(-1), mu_flat)
            if ibm is not None:
                # the node force depends on the streamed populations at the stencil nodes
                a_bar = g.reshape(self.d, -1)[:, ibm.nodes]
                b_bar = np.zeros(self.d)
                if self.probe is None and t >= T - M:
                    b_bar[self.axis] = 1.0 / M
                rho_bar, j_bar = self._vjp_ibm(rho_n, j_n, a_bar, b_bar)
                for k in range(q):
                    s_bar = rho_bar + sum(int(ibm.c[k, a]) * j_bar[a] for a in range(self.d) if ibm.c[k, a])
                    np.add.at(new, k * n + ibm.sources[k], s_bar)
            lam = new.reshape(q, *self.shape)
            if t > T - M:
                lam = lam + self.dD.reshape(q, *self.shape) / M
        # initialize() shifts the velocity by F/(2 rho), F including G: f_0 depends on G
        rho0, u0 = self.init_fields
        rho = np.broadcast_to(np.asarray(rho0, dtype=np.float64), self.shape)
        force = self._force()
        for a in range(self.d):
            u = [np.broadcast_to(np.asarray(u0[b], dtype=np.float64), self.shape) + 0.5 * force[b] / rho
                 + (0.5j * H / rho if b == a else 0.0) for b in range(self.d)]
            feq = equilibrium(self.lattice, (rho - 1.0).astype(np.complex128), tuple(u))
            dG[a] += (lam * feq.imag / H).sum(axis=0)
        return dU, dG
