"""Reverse-mode differentiation of a whole LBM run, behind ``torch.autograd``.

Loss: a force-probe component averaged over the last ``window`` steps of a run
of ``steps`` steps (the momentum-exchange drag, ``forces.ForceProbe``)::

    L(U, G) = (1/M) sum_{t = T-M+1..T} D(f_t),   D = probe force . e_axis

or, for an immersed body and no probe, its body-force component averaged over
the last ``window`` steps (``lbm_ibm_body_force``).

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
With an immersed body, every backward step first recomputes the step's
multi-direct passes from its state (the node force enters the collision of the
stencil nodes), and after the adjoint kernel runs the passes in reverse
(``lbm_ibm_adjoint_iteration``) and adds the resulting dL/d(streamed
populations) at the stencil nodes to mu (``lbm_ibm_adjoint_moments``).

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
        links: wall links of the body whose force is the loss, or None: the loss is
            the force on the immersed body (``params.immersed``).
        steps, window: run length T and averaging window M.
        axis: force component (0 = drag along x).
        checkpoint: steps between checkpoints K.
        block: bulk tile of the kernels.
        dense_rules: link rules in the dense per-node form (``CudaSolver``); False: term by term.
    """

    def __init__(self, make_params, links, steps: int, window: int, axis: int = 0, checkpoint: int = 100,
                 block=(32, 4), dense_rules: bool = True):
        if window < 1 or window > steps:
            raise ValueError("need 1 <= window <= steps")
        self.make_params = make_params
        self.links = links
        self.steps, self.window, self.axis, self.K = int(steps), int(window), int(axis), int(checkpoint)
        self.block = block
        self.dense_rules = bool(dense_rules)
        self._scale = None
        self.solver = None

    # ------------------------------------------------------------------ set-up
    def _setup(self, scale: float, G):
        if self.solver is not None and self._scale == scale:
            # same inlet scale, same rules and tables: only the force field changes
            s = self.solver
            field = np.zeros((s.lattice.d, *s.shape)) if G is None else np.asarray(G, dtype=np.float64)
            s._force_field.copy_(s._upload_field(field.reshape(s.lattice.d, *s.shape)))
            return
        params, d_rules = self.make_params(scale)
        if self.links is None and params.immersed is None:
            raise ValueError("without wall links the loss is the immersed body's force: params.immersed is None")
        if params.dtype not in ("float32", "float64"):
            raise ValueError("the adjoint needs float32 or float64 storage (its recomputed forward must be exact)")
        if G is None:
            G = np.zeros((params.d, *params.shape))
        # rule terms: those with a nonzero coefficient or a nonzero U-derivative
        keep = None if d_rules is None else np.asarray(d_rules.values.coeff) != 0.0
        s = CudaSolver(params, variant="pull", block=self.block, force_field=G, graph=True, keep_terms=keep,
                       dense_rules=self.dense_rules)
        self.solver, self.params, self.d_rules = s, params, d_rules
        self._scale = scale
        torch = s.torch
        self.probe = comp = None
        if self.links is not None:
            probe = ForceProbe.build(params, self.links)
            comp = probe.compiled("pull")
            self.probe = probe
            slots, coeff, const, (rows, terms) = s._affine_tensors(comp)
            self._probe_t = (slots, coeff, const, rows, terms)
            self._probe_w = torch.from_numpy(np.ascontiguousarray(probe.weight)).to(s.device)
            self._partial = torch.empty(((rows + 255) // 256) * s.lattice.d, dtype=torch.float64, device=s.device)
            self._counter = torch.zeros(1, dtype=torch.int32, device=s.device)
        self._ibm_adj = self._build_ibm_adjoint() if s._ibm is not None else None
        self._build_adjoint_tables(comp, None if self.probe is None else self.probe.weight[:, self.axis])

    def _build_ibm_adjoint(self):
        """Scratch of the immersed-boundary adjoint: a private copy of the pass buffers (the recomputed
        forward of one step), every pass's node force, the ping-pong node-force adjoints and the
        float64 moment adjoints."""
        s = self.solver
        torch = s.torch
        ibm = s._ibm
        tab = ibm.tables
        rules = self.params.link_rules
        if rules is not None and len(rules):
            if np.intersect1d(np.asarray(rules.node), tab.nodes).size:
                raise ValueError("the adjoint needs the immersed-boundary stencil nodes free of link rules")
        d, n, dev, real = s.lattice.d, tab.n_nodes, s.device, s.t_real
        st = {
            "rho": torch.zeros(n, dtype=real, device=dev),
            "u_star": torch.zeros((d, n), dtype=real, device=dev),
            "marker_force": torch.zeros((tab.iterations, d, tab.n_markers), dtype=real, device=dev),
            "force": torch.zeros((tab.iterations, d, n), dtype=real, device=dev),
            "adj": [torch.zeros((d, n), dtype=real, device=dev) for _ in range(2)],
            "moments": torch.zeros((1 + d, n), dtype=torch.float64, device=dev),
            # each marker's forward and adjoint terms of a reverse pass, formed once
            "marker_scratch": torch.zeros((1 + 2 * d, tab.n_markers), dtype=torch.float64, device=dev),
        }
        base = ibm.struct
        st["struct"] = N.Ibm(base.n_nodes, base.n_markers, base.stencil_size, base.node, base.stencil, base.weight,
                             base.area, base.inv_start, base.inv_marker, base.inv_weight, N.ptr(st["rho"]),
                             N.ptr(st["u_star"]), N.ptr(st["marker_force"]), N.ptr(st["marker_scratch"]))
        return st

    def _ibm_recompute(self, f, stream):
        """The multi-direct passes of the step from state f (as the forward step), every pass's node force kept."""
        s, st = self.solver, self._ibm_adj
        N.call("lbm_ibm_force", N.C.byref(s.grid), N.C.byref(s.physics), N.C.byref(st["struct"]), N.ptr(f),
               N.LAYOUT_PULL, st["force"].shape[0], N.ptr(st["force"]), stream)

    def _ibm_reverse(self, mu, body_scale, stream):
        """Passes in reverse from dL/d(node force) (written by the adjoint step), then add the moment
        adjoints into mu at the stencil nodes."""
        s, st = self.solver, self._ibm_adj
        g, ib = N.C.byref(s.grid), N.C.byref(st["struct"])
        axis = self.axis if self.probe is None else -1
        cur = 0
        K = len(st["force"])
        for j in range(K - 1, -1, -1):
            prev = st["force"][j - 1] if j else None
            out = st["adj"][cur ^ 1] if j else None
            N.call("lbm_ibm_adjoint_iteration", g, ib, N.ptr(prev), N.ptr(st["adj"][cur]), axis, body_scale,
                   N.ptr(out), N.ptr(st["moments"]), stream)
            cur ^= 1
        N.call("lbm_ibm_adjoint_moments", g, ib, N.ptr(st["moments"]), N.ptr(mu), stream)

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
        if comp is not None:
            slots = np.asarray(comp.slots)
            coeff = np.asarray(comp.coeff)
            for r in range(slots.shape[0]):
                for t in range(slots.shape[1]):
                    if coeff[r, t] != 0.0 and w_axis[r] != 0.0:
                        k, y = divmod(int(slots[r, t]), n)
                        entries.setdefault(int(s._pitched(np.array([y]))[0]), []).append(
                            (k, -1, float(w_axis[r] * coeff[r, t])))
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
        force_slot = np.full(ns, -1, dtype=np.int32)
        if base_nodes.size:
            rule_mask[pos] = t["rule_mask"].cpu().numpy().view(np.uint32)
            rule_first[pos] = t["rule_first"].cpu().numpy()
            force_slot[pos] = t["force_slot"].cpu().numpy()
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
            "force_slot": torch.from_numpy(force_slot).to(dev),
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
            if getattr(s, "_dense_pos", None) is not None:
                ddense = np.zeros(t["rule_dense"].numel())
                np.add.at(ddense, s._dense_pos, dcoeff)
                self._adj_t["rule_ddense"] = torch.from_numpy(ddense).to(dev, s.t_real)
        # dense rule form on the adjoint list: the forward nodes keep their distinct-term ranges (the
        # lists are both sorted by node, so the ranges stay in order); the added nodes have none
        if "ut_start" in t and base_nodes.size:
            fwd_start = t["ut_start"].cpu().numpy().astype(np.int64)
            before = np.searchsorted(base_nodes, nodes, side="left")  # forward nodes before each adjoint node
            adj_start = np.zeros(ns + 1, dtype=np.int64)
            adj_start[:-1] = fwd_start[before]
            adj_start[-1] = fwd_start[-1]
            self._adj_t["ut_start"] = torch.from_numpy(adj_start.astype(np.int32)).to(dev)
        self._force_grad = torch.zeros((lat.d, qs), dtype=s.t_real, device=dev)

    def _special_struct(self):
        s = self.solver
        t, f = self._adj_t, s._special
        g = t.get
        st = self._ibm_adj
        local = st["force"][-1] if st is not None else None  # the node force of the recomputed last pass
        return N.Special(
            int(t["node"].numel()), N.ptr(g("node")), N.ptr(g("rule_mask")), N.ptr(g("rule_first")),
            N.ptr(g("force_slot")), N.ptr(g("zero")), N.ptr(g("zero")), f.n_rules, f.n_terms,
            N.ptr(f.tensors.get("term_start")), N.ptr(f.tensors.get("rule_const")), N.ptr(f.tensors.get("term_dir")),
            N.ptr(f.tensors.get("term_node")), None, N.ptr(f.tensors.get("term_coeff")), N.ptr(local),
            f.n_local if st is not None else 0, 0, None, None,
            N.ptr(g("ut_start")), N.ptr(f.tensors.get("ut_slot") if "ut_start" in t else None), None,
            N.ptr(f.tensors.get("rule_row") if "ut_start" in t else None),
            N.ptr(f.tensors.get("rule_dense") if "ut_start" in t else None),
        )

    def _adj_struct(self):
        t = self._adj_t
        st = self._ibm_adj
        return N.Adjoint(N.ptr(t["gather_start"]), N.ptr(t["gather_dir"]), N.ptr(t["gather_slot"]),
                         N.ptr(t["gather_coeff"]), N.ptr(t.get("rule_dconst")), N.ptr(t.get("term_dcoeff")),
                         N.ptr(self._rule_du), N.ptr(self._force_grad), N.ptr(st["adj"][0] if st is not None else None),
                         N.ptr(t.get("rule_ddense")))

    # ------------------------------------------------------------------ forward
    def _probe_value(self, out_slot):
        s = self.solver
        if self.probe is None:
            ibm = s._ibm
            N.call("lbm_ibm_body_force", N.C.byref(s.grid), N.C.byref(ibm.struct), ibm.tables.iterations,
                   N.ptr(out_slot), s._stream())
            return
        slots, coeff, const, rows, terms = self._probe_t
        N.call("lbm_affine_reduce", s.grid.storage, N.ptr(s._f), N.ptr(slots), N.ptr(coeff), N.ptr(const),
               N.ptr(self._probe_w), rows, terms, s.lattice.d, N.ptr(self._partial), N.ptr(self._counter),
               N.ptr(out_slot), s._stream())

    def forward(self, scale: float = 1.0, G=None) -> float:
        """Run T steps from rest; returns the loss (host float).

        Steps between checkpoints that are outside the loss window replay the
        solver's CUDA graphs; steps in the window run one by one, each followed
        by the probe reduction of its value (or the immersed body's force of
        that step).
        """
        import torch

        self._setup(float(scale), G)
        s = self.solver
        T, M, K = self.steps, self.window, self.K
        s.initialize()
        self._rho0 = torch.ones(s.qstride, dtype=torch.float64, device=s.device)
        self._u0 = torch.zeros((s.lattice.d, s.qstride), dtype=torch.float64, device=s.device)
        self._checkpoints = {}
        values = torch.zeros((M, s.lattice.d), dtype=torch.float64, device=s.device)
        t = 0
        while t < T:
            if t % K == 0:
                self._checkpoints[t] = s._f.clone()
            stop = min((t // K + 1) * K, T)
            if t + 1 > T - M:
                for u in range(t, stop):
                    s._launch_pull()
                    self._probe_value(values[u + 1 - (T - M + 1)])
                t = stop
            else:
                run = min(stop, T - M) - t
                s._advance(run)
                t += run
        self.loss = float(values[:, self.axis].sum().item()) / M
        return self.loss

    # ------------------------------------------------------------------ backward
    def _capture(self, fn):
        """A CUDA graph of the launches fn makes (fn computes its stream inside)."""
        s = self.solver
        torch = s.torch
        stream = torch.cuda.Stream(s.device)
        stream.wait_stream(torch.cuda.current_stream(s.device))
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(stream):
            graph.capture_begin()
            try:
                fn()
            finally:
                graph.capture_end()
        torch.cuda.current_stream(s.device).wait_stream(stream)
        return graph

    def backward(self):
        """(dL/dU, dL/dG (d, *shape) host float64) for the last forward().

        Segments of K steps, from the last: the forward states of a segment
        are recomputed from its checkpoint into a ring of K buffers, then the
        adjoint steps run backwards through them. Two rings alternate, so the
        recomputation of the next (earlier) segment runs on its own stream
        while the adjoint kernels sweep the current one. Full segments replay
        CUDA graphs (the recomputation, and the adjoint steps per loss-source
        scale); the first adjoint step and partial segments launch one by one.
        """
        s = self.solver
        torch = s.torch
        T, M, K = self.steps, self.window, self.K
        q = s.lattice.q
        rings = [[torch.empty((q, s.qstride), dtype=s.t_store, device=s.device) for _ in range(K)] for _ in range(2)]
        mu = [torch.empty((q, s.qstride), dtype=s.t_real, device=s.device) for _ in range(2)]
        self._force_grad.zero_()
        if self._rule_du is not None:
            self._rule_du.zero_()
        sp, adj = self._special_struct(), self._adj_struct()
        g, ph = N.C.byref(s.grid), N.C.byref(s.physics)
        launches = [N.Launch(self.block[0], self.block[1], m) for m in (N.LAUNCH_BULK, N.LAUNCH_BOUNDARY)]
        f_saved = (s._f, s._f_next)
        main = torch.cuda.current_stream(s.device)
        rec_stream = torch.cuda.Stream(s.device)
        adj_side = torch.cuda.Stream(s.device)

        def recompute(ring, n):
            for j in range(n - 1):
                s._f, s._f_next = ring[j], ring[j + 1]
                s._launch_pull()

        def scale_of(t):
            return 1.0 / M if t + 1 > T - M else 0.0

        def adjoint_steps(ring, start, stop, cur, mu_next):
            # bulk and boundary adjoint kernels touch disjoint nodes: the
            # boundary one runs on a side stream, concurrently
            here = torch.cuda.current_stream(s.device)
            ibm_loss = self.probe is None
            for t in range(stop - 1, start - 1, -1):
                out = mu[cur]
                fork, join = torch.cuda.Event(), torch.cuda.Event()
                fork.record(here)
                adj_side.wait_event(fork)
                if self._ibm_adj is not None:  # the boundary kernel reads the step's node force
                    self._ibm_recompute(ring[t - start], adj_side.cuda_stream)
                for lc, stream in ((launches[1], adj_side), (launches[0], here)):
                    N.call("lbm_adjoint_step", g, ph, N.C.byref(sp), N.C.byref(adj), N.C.byref(lc),
                           N.ptr(self._adj_kind), N.ptr(ring[t - start]), N.ptr(mu_next), N.ptr(out),
                           0.0 if ibm_loss else scale_of(t), stream.cuda_stream)
                join.record(adj_side)
                here.wait_event(join)
                if self._ibm_adj is not None:
                    self._ibm_reverse(out, scale_of(t) if ibm_loss else 0.0, here.cuda_stream)
                mu_next = out
                cur ^= 1
            return cur, mu_next

        graphs = {}
        starts = sorted(self._checkpoints, reverse=True)
        ready = [None, None]  # recomputation of the ring finished
        free = [None, None]   # adjoint steps done reading the ring

        def launch_recompute(idx):
            start = starts[idx]
            n = min(start + K, T) - start
            rid = idx & 1
            with torch.cuda.stream(rec_stream):
                if free[rid] is not None:
                    rec_stream.wait_event(free[rid])
                rings[rid][0].copy_(self._checkpoints[start])
                if n == K and K > 1:  # (K = 1: the checkpoint alone, nothing to recompute or capture)
                    key = ("recompute", rid)
                    if key not in graphs:
                        graphs[key] = self._capture(lambda: recompute(rings[rid], K))
                    graphs[key].replay()
                else:
                    recompute(rings[rid], n)
                ready[rid] = torch.cuda.Event()
                ready[rid].record(rec_stream)

        launch_recompute(0)
        mu_next = None
        cur = 0
        for idx, start in enumerate(starts):
            if idx + 1 < len(starts):
                launch_recompute(idx + 1)
            rid = idx & 1
            stop = min(start + K, T)
            n = stop - start
            main.wait_event(ready[rid])
            scales = {scale_of(t) for t in range(start, stop)}
            if n == K and mu_next is not None and len(scales) == 1:
                key = ("adjoint", scales.pop(), cur, rid)
                if key not in graphs:
                    c0 = cur
                    graphs[key] = self._capture(lambda: adjoint_steps(rings[rid], start, stop, c0, mu[c0 ^ 1]))
                graphs[key].replay()
                cur ^= K & 1
                mu_next = mu[cur ^ 1]
            else:
                cur, mu_next = adjoint_steps(rings[rid], start, stop, cur, mu_next)
            free[rid] = torch.cuda.Event()
            free[rid].record(main)
        s._f, s._f_next = f_saved
        N.call("lbm_adjoint_initial", g, ph, N.C.byref(sp), N.C.byref(adj), N.ptr(self._adj_kind), N.ptr(mu_next),
               N.ptr(self._rho0), N.ptr(self._u0), 0.0, s._stream())
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
