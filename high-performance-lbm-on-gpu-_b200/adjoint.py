"""Reverse-mode differentiation of a whole LBM run, behind ``torch.autograd``.

Loss: a force-probe component averaged over the last ``window`` steps of a run
of ``steps`` steps (the momentum-exchange drag, ``forces.ForceProbe``)::

    L(U, G) = (1/M) sum_{t = T-M+1..T} D(f_t),   D = probe force . e_axis

Parameters: a per-node Guo force field G (d, *shape) and, optionally, the
scale U of the Zou-He inlet velocity (rules and their exact derivative from
``open_boundaries.zou_he_inlet_derivative``).

Forward: the two-lattice step (``lbm_step_pull``) from rest; the state is
checkpointed every ``checkpoint`` steps in device memory; the probe value of
every step of the window is reduced on the device in float64.
Backward: segment by segment from the end, the forward states of the segment
are recomputed from its checkpoint into a device ring, then one fused
adjoint kernel per step (``lbm_adjoint_step``: transposed streaming +
transposed TRT/Guo collision + transposed link rules + loss source) runs
backwards through them; a closing kernel adds the initial-state term. The
gradient w.r.t. U accumulates per rule in float64 and is summed at the end.

``LbmDragLoss`` wraps forward/backward as a ``torch.autograd.Function``.
"""

from __future__ import annotations

import numpy as np

from . import _native as N
from .forces import ForceProbe
from .link_rules import AffineSet, LinkRules
from .solver import CudaSolver


def aligned_rules(open_rules: LinkRules, d_open: LinkRules, other: LinkRules | None):
    """Concatenate inlet/outlet rules with other rules, and their derivatives with zeros."""
    if other is None or not len(other):
        return open_rules, d_open
    zero = LinkRules(other.node, other.direction,
                     AffineSet(other.values.direction, other.values.node, np.zeros_like(other.values.coeff),
                               np.zeros_like(other.values.constant)))
    return LinkRules.concat(open_rules, other), LinkRules.concat(d_open, zero)


class AdjointRun:
    """Forward run + adjoint for one parameter set.

    Args:
        make_params: callable (scale U) -> (params, d_rules); ``params.link_rules``
            and ``d_rules`` row/term aligned (``aligned_rules``). ``d_rules`` may be None.
        links: wall links of the body whose force is the loss.
        steps, window: run length T and averaging window M.
        axis: force component (0 = drag along x).
        checkpoint: steps between checkpoints K.
        block: bulk tile of the kernels.
    """

    def __init__(self, make_params, links, steps: int, window: int, axis: int = 0, checkpoint: int = 100,
                 block=(32, 4)):
        if window < 1 or window > steps:
            raise ValueError("need 1 <= window <= steps")
        self.make_params = make_params
        self.links = links
        self.steps, self.window, self.axis, self.K = int(steps), int(window), int(axis), int(checkpoint)
        self.block = block
        self._scale = None
        self.solver = None

    # ------------------------------------------------------------------ set-up
    def _setup(self, scale: float, G):
        params, d_rules = self.make_params(scale)
        if params.immersed is not None:
            raise ValueError("the adjoint supports walls, forces and link rules (no immersed bodies)")
        if params.dtype not in ("float32", "float64"):
            raise ValueError("the adjoint needs float32 or float64 storage (its recomputed forward must be exact)")
        s = CudaSolver(params, variant="pull", block=self.block, force_field=G, graph=False, keep_zero_terms=True)
        self.solver, self.params, self.d_rules = s, params, d_rules
        torch = s.torch
        probe = ForceProbe.build(params, self.links)
        comp = probe.compiled("pull")
        self.probe = probe
        slots, coeff, const, (rows, terms) = s._affine_tensors(comp)
        self._probe_t = (slots, coeff, const, rows, terms)
        self._probe_w = torch.from_numpy(np.ascontiguousarray(probe.weight)).to(s.device)
        self._partial = torch.empty(((rows + 255) // 256) * s.lattice.d, dtype=torch.float64, device=s.device)
        self._counter = torch.zeros(1, dtype=torch.int32, device=s.device)
        self._build_adjoint_tables(comp, probe.weight[:, self.axis])

    def _build_adjoint_tables(self, comp, w_axis):
        """Adjoint special list: forward special nodes + rule-term nodes + probe nodes, with gather tables.

        Nodes only next to a wall or on a periodic face stay with the bulk
        adjoint kernel (solid-neighbour masks from the forward classification).
        """
        s = self.solver
        torch = s.torch
        lat = s.lattice
        n, qs = s.n_nodes, s.qstride
        entries = {}  # pitched node -> list of (k, slot, coeff)
        # transposed rule terms: lambda_k(y) += coeff * mu_j(x)
        rules = self.params.link_rules
        if rules is not None and len(rules):
            v = rules.values
            x = s._pitched(np.asarray(rules.node))
            j = np.asarray(rules.direction)
            for r in range(len(rules)):
                mu_slot = int(j[r]) * qs + int(x[r])
                for k, y, a in zip(v.direction[r], v.node[r], v.coeff[r], strict=True):
                    if a != 0.0:
                        entries.setdefault(int(s._pitched(np.array([y]))[0]), []).append((int(k), mu_slot, float(a)))
        # loss gradient dD/df at probe slots (layout pull = natural)
        slots = np.asarray(comp.slots)
        coeff = np.asarray(comp.coeff)
        for r in range(slots.shape[0]):
            for t in range(slots.shape[1]):
                if coeff[r, t] != 0.0 and w_axis[r] != 0.0:
                    k, y = divmod(int(slots[r, t]), n)
                    entries.setdefault(int(s._pitched(np.array([y]))[0]), []).append((k, -1, float(w_axis[r] * coeff[r, t])))
        base = s._special.tensors.get("node")
        base_nodes = base.cpu().numpy() if base is not None else np.zeros(0, dtype=np.int64)
        extra = np.array(sorted(entries), dtype=np.int64)
        nodes = np.union1d(base_nodes, extra)
        ns = nodes.size
        # per-node forward tables re-indexed onto the adjoint list
        pos = np.searchsorted(nodes, base_nodes)
        t = s._special.tensors
        rule_mask = np.zeros(ns, dtype=np.uint32)
        rule_first = np.zeros(ns, dtype=np.int32)
        if base_nodes.size:
            rule_mask[pos] = t["rule_mask"].cpu().numpy().view(np.uint32)
            rule_first[pos] = t["rule_first"].cpu().numpy()
        starts = np.zeros(ns + 1, dtype=np.int64)
        dirs, gslots, gcoef = [], [], []
        for i, node in enumerate(nodes.tolist()):
            for k, slot, a in entries.get(node, ()):
                dirs.append(k)
                gslots.append(slot)
                gcoef.append(a)
            starts[i + 1] = len(dirs)
        dev = s.device
        self._adj_t = {
            "node": torch.from_numpy(nodes).to(dev),
            "rule_mask": torch.from_numpy(rule_mask.view(np.int32)).to(dev),
            "rule_first": torch.from_numpy(rule_first).to(dev),
            "force_slot": torch.full((ns,), -1, dtype=torch.int32, device=dev),
            "zero": torch.zeros(max(ns, 1), dtype=torch.int32, device=dev),
            "gather_start": torch.from_numpy(starts.astype(np.int32)).to(dev),
            "gather_dir": torch.from_numpy(np.asarray(dirs, dtype=np.int32)).to(dev),
            "gather_slot": torch.from_numpy(np.asarray(gslots, dtype=np.int64)).to(dev),
            "gather_coeff": torch.from_numpy(np.asarray(gcoef, dtype=np.float64)).to(dev, s.t_real),
        }
        # kind: adjoint-list nodes are SPECIAL so the bulk skips them
        self._adj_kind = s._kind.clone()
        self._adj_kind[self._adj_t["node"]] |= N.KIND_SPECIAL

        # rule derivative tables (aligned with the device rule terms)
        self._rule_du = None
        if self.d_rules is not None and s._special.n_rules:
            dv = self.d_rules.values
            order = s._rule_order
            live = s._rule_live
            dconst = np.asarray(dv.constant, dtype=np.float64)[order]
            dcoeff = np.asarray(dv.coeff, dtype=np.float64)[order][live]
            self._adj_t["rule_dconst"] = torch.from_numpy(dconst).to(dev, s.t_real)
            self._adj_t["term_dcoeff"] = torch.from_numpy(dcoeff).to(dev, s.t_real)
            self._rule_du = torch.zeros(s._special.n_rules, dtype=torch.float64, device=dev)
        self._force_grad = torch.zeros((lat.d, qs), dtype=s.t_real, device=dev)

    def _special_struct(self):
        s = self.solver
        t, f = self._adj_t, s._special
        g = t.get
        return N.Special(
            int(t["node"].numel()), N.ptr(g("node")), N.ptr(g("rule_mask")), N.ptr(g("rule_first")),
            N.ptr(g("force_slot")), N.ptr(g("zero")), N.ptr(g("zero")), f.n_rules, f.n_terms,
            N.ptr(f.tensors.get("term_start")), N.ptr(f.tensors.get("rule_const")), N.ptr(f.tensors.get("term_dir")),
            N.ptr(f.tensors.get("term_node")), None, N.ptr(f.tensors.get("term_coeff")), None, 0, 0, None, None,
        )

    def _adj_struct(self):
        t = self._adj_t
        return N.Adjoint(N.ptr(t["gather_start"]), N.ptr(t["gather_dir"]), N.ptr(t["gather_slot"]),
                         N.ptr(t["gather_coeff"]), N.ptr(t.get("rule_dconst")), N.ptr(t.get("term_dcoeff")),
                         N.ptr(self._rule_du), N.ptr(self._force_grad))

    # ------------------------------------------------------------------ forward
    def _probe_value(self, out_slot):
        s = self.solver
        slots, coeff, const, rows, terms = self._probe_t
        N.call("lbm_affine_reduce", s.grid.storage, N.ptr(s._f), N.ptr(slots), N.ptr(coeff), N.ptr(const),
               N.ptr(self._probe_w), rows, terms, s.lattice.d, N.ptr(self._partial), N.ptr(self._counter),
               N.ptr(out_slot), s._stream())

    def forward(self, scale: float = 1.0, G=None) -> float:
        """Run T steps from rest; returns the loss (host float)."""
        import torch

        self._setup(float(scale), G)
        s = self.solver
        T, M, K = self.steps, self.window, self.K
        s.initialize()
        self._rho0 = torch.ones(s.qstride, dtype=torch.float64, device=s.device)
        self._u0 = torch.zeros((s.lattice.d, s.qstride), dtype=torch.float64, device=s.device)
        self._checkpoints = {}
        values = torch.zeros((M, s.lattice.d), dtype=torch.float64, device=s.device)
        for t in range(T):
            if t % K == 0:
                self._checkpoints[t] = s._f.clone()
            s._launch_pull()
            if t + 1 > T - M:
                self._probe_value(values[t + 1 - (T - M + 1)])
        self.loss = float(values[:, self.axis].sum().item()) / M
        return self.loss

    # ------------------------------------------------------------------ backward
    def backward(self):
        """(dL/dU, dL/dG (d, *shape) host float64) for the last forward()."""
        s = self.solver
        torch = s.torch
        T, M, K = self.steps, self.window, self.K
        q = s.lattice.q
        ring = [torch.empty((q, s.qstride), dtype=s.t_store, device=s.device) for _ in range(K)]
        mu = [torch.empty((q, s.qstride), dtype=s.t_real, device=s.device) for _ in range(2)]
        self._force_grad.zero_()
        if self._rule_du is not None:
            self._rule_du.zero_()
        sp, adj = self._special_struct(), self._adj_struct()
        g, ph = N.C.byref(s.grid), N.C.byref(s.physics)
        launches = [N.Launch(self.block[0], self.block[1], m) for m in (N.LAUNCH_BULK, N.LAUNCH_BOUNDARY)]
        stream = s._stream()
        mu_next = None
        cur = 0
        for start in sorted(self._checkpoints, reverse=True):
            stop = min(start + K, T)
            # recompute f_start .. f_{stop-1} into the ring
            ring[0].copy_(self._checkpoints[start])
            for t in range(start, stop - 1):
                s._f, s._f_next = ring[t - start], ring[t - start + 1]
                s._launch_pull()
            for t in range(stop - 1, start - 1, -1):
                scale = 1.0 / M if t + 1 > T - M else 0.0
                out = mu[cur]
                for lc in launches:
                    N.call("lbm_adjoint_step", g, ph, N.C.byref(sp), N.C.byref(adj), N.C.byref(lc),
                           N.ptr(self._adj_kind), N.ptr(ring[t - start]), N.ptr(mu_next), N.ptr(out), scale, stream)
                mu_next = out
                cur ^= 1
        N.call("lbm_adjoint_initial", g, ph, N.C.byref(sp), N.C.byref(adj), N.ptr(self._adj_kind), N.ptr(mu_next),
               N.ptr(self._rho0), N.ptr(self._u0), 0.0, stream)
        dU = float(self._rule_du.sum().item()) if self._rule_du is not None else 0.0
        dG = s._from_pitched(self._force_grad).astype(np.float64)
        return dU, dG


def _torch_function():
    import torch

    class LbmDragLoss(torch.autograd.Function):
        """L = AdjointRun.forward(U, G); backward returns (dL/dU, dL/dG) from the adjoint."""

        @staticmethod
        def forward(ctx, scale, G, run):
            loss = run.forward(float(scale.detach().cpu().item()), G.detach().cpu().numpy())
            ctx.run = run
            ctx.G_like = G
            return torch.tensor(loss, dtype=torch.float64, device=G.device)

        @staticmethod
        def backward(ctx, grad):
            dU, dG = ctx.run.backward()
            g = grad.detach().to(torch.float64)
            gU = (g * dU).to(ctx.G_like.device).reshape(())
            gG = torch.from_numpy(dG).to(ctx.G_like.device, ctx.G_like.dtype) * g.to(ctx.G_like.dtype)
            return gU, gG, None

    return LbmDragLoss


def drag_loss(scale, G, run: AdjointRun):
    """Differentiable drag loss: ``drag_loss(U_tensor, G_tensor, run).backward()``."""
    return _torch_function().apply(scale, G, run)
