"""Solver contract and the CUDA solver (the drop-in ``cuda`` backend).

``Solver`` keeps the reference's driver semantics (``src/lbm/solver.py:61-221``):
``run`` advances in chunks of ``check_every``/``every`` steps, checks for
divergence after every chunk and fires the callback. ``CudaSolver`` holds the
populations in PyTorch CUDA tensors and advances them with the fused sm_100a
kernels of ``liblbm_b200.so``; nothing here computes on the CPU except input
preparation (rule tables, geometry) and unit conversion of readouts.

Backends (reference ``src/lbm/backends/__init__.py:23``):

==============  ===========================================================
``cuda``        two-lattice fused pull kernel (same as ``cuda-naive``)
``cuda-naive``  two-lattice fused pull kernel
``cuda-aa``     in-place AA pair (one lattice, steps in pairs)
==============  ===========================================================
"""

from __future__ import annotations

import functools
import math
from abc import ABC, abstractmethod
from collections.abc import Callable
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .diagnostics import MacroscopicFields
from .lattice import as_lattice
from .params import COMPUTE_DTYPE

DEFAULT_CHECK_EVERY = 500
DEFAULT_BLOCK = (32, 4)
BACKENDS = ("cuda", "cuda-naive", "cuda-tiled", "cuda-aa")
"""``cuda-tiled`` keeps the reference's 2D-only backend name working: this build's pull
step (its shared-memory staging is the TMA kernel for 16-bit storage)."""
VARIANTS = ("pull", "aa")


class BackendUnavailable(RuntimeError):
    """The CUDA backend needs a CUDA device and the built library; one is missing."""


class SimulationDiverged(RuntimeError):
    """Non-finite populations or rho <= 0 at a fluid node (reference ``solver.py:39-51``)."""

    def __init__(self, step: int, location: tuple[int, ...], reason: str):
        self.step = step
        self.location = location
        names = "(y, x)" if len(location) == 2 else "(z, y, x)"
        super().__init__(f"simulation diverged by step {step}: {reason} at node {names}={location}")


@functools.cache
def gpu_available() -> bool:
    try:
        import torch

        if not torch.cuda.is_available() or torch.cuda.device_count() == 0:
            return False
        N.load()
    except (ImportError, N.NativeUnavailable):
        return False
    return True


def available_backends() -> tuple[str, ...]:
    return BACKENDS if gpu_available() else ()


def make_solver(params, backend: str = "cuda", **options) -> CudaSolver:
    """Create a solver for ``params`` (reference ``backends/__init__.py:62-83``).

    ``options`` go to ``CudaSolver`` (``block=``, ``force_field=``, ``graph=``...).
    """
    if backend not in BACKENDS:
        raise ValueError(f"unknown backend {backend!r}; choose from {BACKENDS}")
    if backend == "cuda-tiled" and params.d != 2:  # reference cuda_solver.py:56-62
        raise ValueError(f"CUDA variant 'tiled' is 2D only; use 'naive' or 'aa' for a {params.d}D grid")
    return CudaSolver(params, variant="aa" if backend == "cuda-aa" else "pull", **options)


class Solver(ABC):
    """Driver shared by the CUDA variants: chunked run loop, watchdog, callbacks."""

    step_multiple = 1
    state_layout = "pull"

    def __init__(self, params):
        self.params = params
        self.time_step = 0

    @abstractmethod
    def initialize(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0) -> None: ...

    @abstractmethod
    def _advance(self, steps: int) -> None: ...

    @abstractmethod
    def _check_health(self) -> None: ...

    def _advance_checked(self, steps: int) -> None:
        """``_advance`` for the run loop: a solver that checks its state inside the last step of
        the chunk (for ``_check_health`` to read) overrides it."""
        self._advance(steps)

    def run(self, steps: int, *, every: int = 0, callback: Callable | None = None,
            check_every: int = DEFAULT_CHECK_EVERY) -> None:
        """Advance ``steps`` steps (reference ``solver.py:119-160``, same chunking and errors)."""
        if steps < 0 or every < 0 or check_every <= 0:
            raise ValueError(f"need steps >= 0, every >= 0, check_every > 0; got {steps}, {every}, {check_every}")
        m = self.step_multiple
        if steps % m or every % m or check_every % m:
            raise ValueError(
                f"{type(self).__name__} advances in multiples of {m} steps; "
                f"steps, every and check_every must be multiples of {m}"
            )
        done = 0
        while done < steps:
            stop = min(steps, (done // check_every + 1) * check_every)
            if every:
                stop = min(stop, (done // every + 1) * every)
            self._advance_checked(stop - done)
            self.time_step += stop - done
            done = stop
            self._check_health()
            if callback is not None and ((every and done % every == 0) or done == steps):
                callback(self)


# ---------------------------------------------------------------------------- device tables


def dense_rule_tables(nodes, rule_nodes, start, term_key, term_coeff, max_terms: int):
    """Dense per-node form of link rules (``lbm_special_t.ut_start``).

    ``nodes``: the sorted special-node list; rule r belongs to node ``rule_nodes[r]`` and owns the
    terms ``start[r]:start[r+1]``, each reading population ``term_key`` (a slot, or an export index)
    with ``term_coeff``. Returns ``(ut_start, ut_key, rule_row, dense, pos)``: per node the range of
    its rules' distinct populations, their keys, per rule the start of its coefficient row (rows
    zero-padded to multiples of 4, so rule r of node s is
    ``const + dense[rule_row[r] : rule_row[r] + n_s] @ values[ut_start[s] : ut_start[s+1]]``), and the
    dense position of every term; None when a node reads more than ``max_terms`` distinct populations.
    """
    nodes = np.asarray(nodes)
    counts = np.diff(np.asarray(start))
    n_rules = counts.size
    rule_of_term = np.repeat(np.arange(n_rules), counts)
    s_of_rule = np.searchsorted(nodes, np.asarray(rule_nodes))
    s_of_term = s_of_rule[rule_of_term]
    pairs, inverse = np.unique(np.stack([s_of_term, np.asarray(term_key)], axis=1), axis=0, return_inverse=True)
    inverse = inverse.reshape(-1)
    ut_start = np.searchsorted(pairs[:, 0], np.arange(nodes.size + 1))
    n_distinct = np.diff(ut_start)
    if n_distinct.max(initial=0) > max_terms:
        return None
    local = inverse - ut_start[s_of_term]
    row_len = (n_distinct[s_of_rule] + 3) // 4 * 4
    rule_row = np.zeros(n_rules, dtype=np.int64)
    np.cumsum(row_len[:-1], out=rule_row[1:])
    dense = np.zeros(max(int(row_len.sum()), 4))
    pos = rule_row[rule_of_term] + local
    np.add.at(dense, pos, np.asarray(term_coeff, dtype=np.float64))
    return ut_start, pairs[:, 1], rule_row, dense, pos


PINNED_READOUT_BYTES = 1 << 30
"""Largest host readout (macroscopic fields, populations) copied through page-locked memory."""


@dataclass
class _SpecialTables:
    """Device form of the boundary-warp work list (see ``lbm_special_t``)."""

    tensors: dict
    n_special: int
    n_rules: int
    n_terms: int
    n_export: int
    n_local: int


def row_pitch(nx: int, storage: str) -> int:
    """Default row stride (in nodes) of a lattice of width nx.

    16-bit storage: nx rounded up to 16 nodes (the pair and TMA kernels need
    16-byte row strides). 4- and 8-byte storage: nx rounded up to 32 bytes
    (a DRAM sector) when that adds at most a quarter to the row, else nx.
    Rows that start only 8-byte aligned cost 7-8 % (float32 pull, one B200:
    D2Q9 2050 x 2048 70.9 GLUPS at pitch 2050, 76.5 at 2056, 75.9 at 2064,
    74.8 at 2080; D3Q19 250 x 256^2 476 -> 446 us per step at pitch 256);
    wider alignment gains nothing more (D3Q19 244 x 256^2: 37.3, 37.0, 36.0
    GLUPS at pitch 244, 248, 256). Padding columns are never read or written.
    """
    if storage in ("float16", "bfloat16"):
        return -(-nx // 16) * 16
    align = 32 // (8 if storage == "float64" else 4)
    padded = -(-nx // align) * align
    return padded if 4 * padded <= 5 * nx else nx


def _pitched_index(flat: np.ndarray, shape: tuple[int, ...], pitch: int) -> np.ndarray:
    """Natural flat node index -> pitched index (x row padded to ``pitch``)."""
    flat = np.asarray(flat, dtype=np.int64)
    nx = shape[-1]
    return (flat // nx) * pitch + flat % nx


def _natural_index(pitched: int, shape: tuple[int, ...], pitch: int) -> tuple[int, ...]:
    row, x = divmod(int(pitched), pitch)
    if len(shape) == 2:
        return (row, x)
    z, y = divmod(row, shape[1])
    return (z, y, x)


class CudaSolver(Solver):
    """Fused stream-bounce-collide on a B200 (reference ``backends/cuda_solver.py:179-326``).

    Args:
        params: a ``SimulationParams`` (this package's or the reference's).
        variant: ``"pull"`` (two lattices) or ``"aa"`` (in place, steps in pairs).
        block: bulk tile (x, y) in threads; x a multiple of 32, at most 256 threads.
        force_field: optional per-node Guo force (d, *shape) added to the uniform force (and,
            at immersed-boundary stencil nodes, to the node force; the immersed-boundary
            moments u* use the uniform force only, as the reference's).
        graph: capture chunks of steps in CUDA graphs (saves launch latency on small grids).
        dense_rules: evaluate link rules in the dense per-node form (each node's distinct term
            populations loaded once for all its rules); False: term by term.
        device: CUDA device (default: current).
        pitch: row stride in nodes (>= nx); default ``row_pitch(nx, dtype)``.
    """

    def __init__(self, params, variant: str = "pull", block=DEFAULT_BLOCK, force_field=None,
                 graph: bool = True, device=None, pitch: int | None = None, launch: str = "split",
                 keep_zero_terms: bool = False, keep_terms=None, dense_rules: bool = True):
        if variant not in VARIANTS:
            raise ValueError(f"unknown CUDA variant {variant!r}; choose from {VARIANTS}")
        if launch not in ("fused", "split"):
            raise ValueError(f"launch must be 'fused' or 'split'; got {launch!r}")
        bx, by = (int(b) for b in block)
        if bx <= 0 or by <= 0 or bx * by > 1024:
            raise ValueError(f"block must be positive with at most 1024 threads; got {block}")
        if bx % 32 or bx * by > 256:
            raise ValueError(f"block x must be a multiple of 32 and block at most 256 threads; got {block}")
        try:
            import torch
        except ImportError as exc:  # pragma: no cover
            raise BackendUnavailable("PyTorch is required for the CUDA backend") from exc
        if not torch.cuda.is_available():
            raise BackendUnavailable("no CUDA device found")
        try:
            N.load()
        except N.NativeUnavailable as exc:
            raise BackendUnavailable(str(exc)) from exc
        super().__init__(params)
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.variant = variant
        self.step_multiple = 2 if variant == "aa" else 1
        self.use_graph = bool(graph)
        self._graphs: dict = {}

        lattice = as_lattice(params.lattice)
        self.lattice = lattice
        d, q = lattice.d, lattice.q
        shape = tuple(params.shape)
        self.shape = shape
        self.n_nodes = math.prod(shape)
        nx = shape[-1]
        ny = shape[-2]
        nz = shape[0] if d == 3 else 1
        self.pitch = int(pitch) if pitch is not None else row_pitch(nx, params.dtype)
        if self.pitch < nx:
            raise ValueError(f"pitch must be >= nx={nx}; got {self.pitch}")
        self.qstride = self.pitch * ny * nz
        self.storage = params.dtype
        self.compute = COMPUTE_DTYPE[params.dtype]
        tdt = {"float32": torch.float32, "float64": torch.float64, "float16": torch.float16, "bfloat16": torch.bfloat16}
        self.t_store = tdt[self.storage]
        self.t_real = tdt[self.compute]
        self.grid = N.Grid(N.LATTICE_CODE[lattice.name], N.STORAGE_CODE[self.storage], nx, ny, nz, self.pitch, self.qstride)
        self.launch_mode = launch
        self.keep_zero_terms = bool(keep_zero_terms)
        # optional mask (rules x terms, in the rules' order) of zero-coefficient
        # terms to keep: the adjoint keeps those whose U-derivative is nonzero
        self._keep_terms = None if keep_terms is None else np.asarray(keep_terms, dtype=bool)
        self.dense_rules = bool(dense_rules)
        self._launches = {m: N.Launch(bx, by, m) for m in N.LAUNCH_MODES}
        self.block = (bx, by)

        # ---- physics
        wp, wm = params.relaxation_rates
        force = tuple(float(v) for v in params.force) + (0.0,) * (3 - d)
        wall = np.asarray(params.wall_velocity, dtype=np.float64)
        self._wall = self._upload_field(wall) if np.any(wall != 0.0) else None
        self._force_field = None
        if force_field is not None:
            self._force_field = self._upload_field(np.asarray(force_field, dtype=np.float64).reshape(d, *shape))
        self.physics = N.Physics(wp, wm, (N.C.c_double * 3)(*force), N.ptr(self._wall), N.ptr(self._force_field), None,
                                 N.COLLISION_CODE[params.collision])
        # Small device words, read back in one copy by _check_health:
        #   int32 view of int64 [0:2] -- slots 0, 1: step counter of the stochastic rounding of
        #     16-bit storage (reset whenever the populations are set); slot 2: kernel status word;
        #   int64 [2:4] -- health words (first bad node, non-finite flag);
        #   int64 [4] -- the float64 bits of the last checked step's sum of f~* over fluid nodes.
        self._words = torch.zeros(5, dtype=torch.int64, device=self.device)
        self._seed = self._words[:2].view(torch.int32)
        self._health = self._words[2:4]
        self.physics.round_seed = N.ptr(self._seed)
        self.mass = None
        """Total mass (sum of rho over fluid nodes, float64, summed on the device) of the state
        after the last check of the run loop; None before the first."""
        self._health_fresh = False
        # rho and u written by the checked step of the run loop once macroscopic() has been asked
        # for (allocated then); fresh while no other step or state change followed that step
        self._readout = None
        self._readout_fresh = False

        # ---- immersed boundary and link rules -> special nodes
        self._ibm = None
        if params.immersed is not None:
            from .ibm import build_tables

            self._ibm = _IbmState(self, build_tables(params.immersed, lattice, np.asarray(params.solid)))
        self._solid_host = np.asarray(params.solid, dtype=bool)
        self._special = self._build_special(params)
        self._ibm_split = self._split_special()

        # ---- populations
        self._f = torch.empty((q, self.qstride), dtype=self.t_store, device=self.device)
        self._f_next = torch.empty_like(self._f) if variant == "pull" else None
        self._n_fluid = int((~self._solid_host).sum())
        self._setup_checked_launches()
        self.initialize()

    # ------------------------------------------------------------------ helpers
    def _stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def _native(self, name, *args):
        N.call(name, *args)

    def _to_pitched(self, host: np.ndarray, dtype):
        """(..., *shape) host array -> device tensor (..., qstride), zero padding columns."""
        torch = self.torch
        host = np.ascontiguousarray(host)
        if not host.flags.writeable:  # the parameters' arrays are read-only; torch wants a writable buffer
            host = host.copy()
        lead = host.shape[: host.ndim - len(self.shape)]
        t = torch.from_numpy(host).to(self.device, dtype)
        if self.pitch == self.shape[-1]:
            return t.reshape(*lead, self.qstride).contiguous()
        out = torch.zeros((*lead, *self.shape[:-1], self.pitch), dtype=dtype, device=self.device)
        out[..., : self.shape[-1]] = t
        return out.reshape(*lead, self.qstride)

    def _from_pitched(self, t):
        """Device tensor (..., qstride) -> host array (..., *shape).

        Readouts up to PINNED_READOUT_BYTES land in page-locked host memory
        (torch's caching host allocator reuses the block once the returned
        array is dropped), which the copy engine fills at full link speed; a
        pageable destination goes through a staging buffer at a fraction of it.
        """
        torch = self.torch
        lead = t.shape[:-1]
        view = t.reshape(*lead, *self.shape[:-1], self.pitch)[..., : self.shape[-1]]
        if self.pitch != self.shape[-1]:
            view = view.contiguous()
        if view.numel() * view.element_size() > PINNED_READOUT_BYTES:
            return view.cpu().numpy()
        host = torch.empty(view.shape, dtype=view.dtype, pin_memory=True)
        host.copy_(view, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return host.numpy()

    def _upload_field(self, host):
        return self._to_pitched(np.asarray(host, dtype=np.float64), self.t_real)

    def _upload_scalar(self, host, dtype):
        return self._to_pitched(host, dtype)

    def _pitched(self, flat):
        return _pitched_index(flat, self.shape, self.pitch)

    # ------------------------------------------------------------------ special nodes
    def _build_special(self, params) -> _SpecialTables:
        """Classify the nodes on the device and build the boundary-warp list.

        The list holds the SPECIAL nodes: those carrying link rules, an
        immersed-boundary force or (AA) rule-term exports. Nodes that are only
        next to a wall or on a periodic face stay with the bulk kernel, which
        reads their solid-neighbour mask. Rules are sorted by (node, direction).
        """
        torch = self.torch
        lat = self.lattice
        n = self.n_nodes
        rules = params.link_rules
        t = {}
        n_rules = n_terms = n_export = 0
        rule_nodes = np.zeros(0, dtype=np.int64)
        rule_dir = np.zeros(0, dtype=np.int64)
        if rules is not None and len(rules):
            node = np.asarray(rules.node, dtype=np.int64)
            direction = np.asarray(rules.direction, dtype=np.int64)
            v = rules.values
            coeff = np.asarray(v.coeff, dtype=np.float64)
            tdir = np.asarray(v.direction, dtype=np.int64)
            tnode = np.asarray(v.node, dtype=np.int64)
            const = np.asarray(v.constant, dtype=np.float64)
            order = np.lexsort((direction, node))
            node, direction = node[order], direction[order]
            coeff, tdir, tnode, const = coeff[order], tdir[order], tnode[order], const[order]
            # keep_zero_terms: a fixed term structure; keep_terms: zero terms that
            # another table (the adjoint's derivatives) aligns with
            live = np.ones_like(coeff, dtype=bool) if self.keep_zero_terms else coeff != 0.0
            if self._keep_terms is not None:
                live |= self._keep_terms[order]
            self._rule_order, self._rule_live = order, live
            start = np.zeros(len(node) + 1, dtype=np.int64)
            np.cumsum(live.sum(axis=1), out=start[1:])
            term_dir, term_node, term_coeff = tdir[live], tnode[live], coeff[live]
            n_rules, n_terms = len(node), int(start[-1])
            if n_terms >= 2**31:
                raise ValueError("too many rule terms")
            if np.any(term_node < 0) or np.any(term_node >= n) or np.any(term_dir < 0) or np.any(term_dir >= lat.q):
                raise ValueError("a rule term points outside the lattice")
            rule_nodes, rule_dir = self._pitched(node), direction
            t["term_start"] = torch.from_numpy(start.astype(np.int32)).to(self.device)
            t["rule_const"] = torch.from_numpy(const).to(self.device, self.t_real)
            t["term_dir"] = torch.from_numpy(term_dir.astype(np.int32)).to(self.device)
            t["term_node"] = torch.from_numpy(self._pitched(term_node)).to(self.device)
            t["term_coeff"] = torch.from_numpy(term_coeff).to(self.device, self.t_real)
            term_slot = term_dir * self.qstride + self._pitched(term_node)
        ibm_nodes = self._pitched(self._ibm.tables.nodes) if self._ibm is not None else np.zeros(0, dtype=np.int64)
        export_nodes = export_dirs = np.zeros(0, dtype=np.int64)
        if self.variant == "aa" and n_rules:
            if np.any(self._solid_host.ravel()[term_node]):
                raise ValueError("the AA variant needs every rule term on a fluid node")
            keys = self._pitched(term_node) * 32 + term_dir
            ukeys, term_export = np.unique(keys, return_inverse=True)
            n_export = ukeys.size
            export_nodes, export_dirs = ukeys // 32, ukeys % 32
            t["term_export"] = torch.from_numpy(term_export.astype(np.int32)).to(self.device)
            term_slot = term_export.astype(np.int64)  # the AA rules read the export buffer
            t["export_a"] = torch.zeros(n_export, dtype=self.t_real, device=self.device)
            t["export_b"] = torch.zeros(n_export, dtype=self.t_real, device=self.device)

        # ---- node kinds and solid-neighbour masks on the device; marked nodes get the SPECIAL bit
        nodes = np.unique(np.concatenate([rule_nodes, ibm_nodes, export_nodes])).astype(np.int64)
        marked_t = torch.from_numpy(nodes).to(self.device) if nodes.size else None
        solid = self._upload_scalar(self._solid_host.astype(np.uint8), torch.uint8)
        self._kind = torch.empty(self.qstride, dtype=torch.uint8, device=self.device)
        self._nbr = torch.empty(self.qstride, dtype=torch.int32, device=self.device)
        self._native("lbm_classify", N.C.byref(self.grid), N.ptr(solid), N.ptr(marked_t), int(nodes.size),
                     N.ptr(self._kind), N.ptr(self._nbr), self._stream())
        self.physics.solid_nbr = N.ptr(self._nbr)
        ns = nodes.size
        if ns == 0:
            return _SpecialTables({}, 0, 0, 0, 0, 0)
        if ns >= 2**31:
            raise ValueError("too many special nodes")
        rule_mask = np.zeros(ns, dtype=np.uint32)
        rule_first = np.zeros(ns, dtype=np.int32)
        if n_rules:
            pos = np.searchsorted(nodes, rule_nodes)
            np.bitwise_or.at(rule_mask, pos, (np.uint32(1) << rule_dir.astype(np.uint32)))
            rule_first = np.searchsorted(rule_nodes, nodes, side="left").astype(np.int32)
        force_slot = np.full(ns, -1, dtype=np.int32)
        if ibm_nodes.size:
            force_slot[np.searchsorted(nodes, ibm_nodes)] = np.arange(ibm_nodes.size, dtype=np.int32)
        export_mask = np.zeros(ns, dtype=np.uint32)
        export_first = np.zeros(ns, dtype=np.int32)
        if n_export:
            pos = np.searchsorted(nodes, export_nodes)
            np.bitwise_or.at(export_mask, pos, (np.uint32(1) << export_dirs.astype(np.uint32)))
            export_first = np.searchsorted(export_nodes, nodes, side="left").astype(np.int32)
        self._dense_pos = None
        if n_rules and self.dense_rules:
            self._dense_rules(t, nodes, rule_nodes, start, term_slot, term_coeff)
        t["node"] = marked_t
        t["rule_mask"] = torch.from_numpy(rule_mask.view(np.int32)).to(self.device)
        t["rule_first"] = torch.from_numpy(rule_first).to(self.device)
        t["force_slot"] = torch.from_numpy(force_slot).to(self.device)
        t["export_mask"] = torch.from_numpy(export_mask.view(np.int32)).to(self.device)
        t["export_first"] = torch.from_numpy(export_first).to(self.device)
        return _SpecialTables(t, ns, n_rules, n_terms, n_export, int(ibm_nodes.size))

    def _split_special(self):
        """The boundary-warp list of a pull step with an immersed body, cut in two: the body's
        stencil nodes, which ``lbm_step_pull_ibm`` updates in the launch that forms their force, and
        the rest, for a boundary launch beside it. None (one list, force then boundary launch) for
        the AA variant, a body beyond the one-block kernel, or a stencil node that also has rules."""
        sp, ibm = self._special, self._ibm
        if ibm is None or self.variant != "pull" or sp.n_special == 0:
            return None
        if ibm.tables.n_nodes > N.IBM_FUSED_MAX or ibm.tables.n_markers > N.IBM_FUSED_MAX:
            return None
        t = sp.tensors
        on_body = (t["force_slot"] >= 0).cpu().numpy()
        if np.any(t["rule_mask"].cpu().numpy()[on_body] != 0):
            return None
        torch, dev = self.torch, self.device
        rest = torch.from_numpy(np.flatnonzero(~on_body)).to(dev)
        body = torch.from_numpy(np.flatnonzero(on_body)).to(dev)
        per_node = ("node", "rule_mask", "rule_first", "force_slot", "export_mask", "export_first")
        shared = {k: v for k, v in t.items() if k not in per_node and k != "ut_start"}
        t_rest = {k: t[k][rest] for k in per_node} | shared
        if "ut_start" in t:
            # stencil nodes have no rules, so their distinct-term ranges are empty: the other
            # nodes' ranges stay contiguous
            t_rest["ut_start"] = torch.cat([t["ut_start"][rest], t["ut_start"][-1:]])
        t_body = {k: t[k][body] for k in ("node", "force_slot")}
        t_body["rule_mask"] = torch.zeros_like(t_body["force_slot"])
        t_body["rule_first"] = torch.zeros_like(t_body["force_slot"])
        return (_SpecialTables(t_rest, int(rest.numel()), sp.n_rules, sp.n_terms, sp.n_export, 0),
                _SpecialTables(t_body, int(body.numel()), 0, 0, 0, sp.n_local))

    def _dense_rules(self, t, nodes, rule_nodes, start, term_slot, term_coeff) -> None:
        """Dense form of the rules on the device (``dense_rule_tables``); left out (term-by-term
        evaluation) when a node's rules read more than ``DENSE_TERMS`` distinct populations."""
        torch = self.torch
        tables = dense_rule_tables(nodes, rule_nodes, start, term_slot, term_coeff, N.DENSE_TERMS)
        self._dense_pos = None
        if tables is None:
            return
        ut_start, ut_key, rule_row, dense, self._dense_pos = tables
        dev = self.device
        t["ut_start"] = torch.from_numpy(ut_start.astype(np.int32)).to(dev)
        key = "ut_export" if self.variant == "aa" else "ut_slot"
        t[key] = torch.from_numpy(ut_key.astype(np.int32 if self.variant == "aa" else np.int64)).to(dev)
        t["rule_row"] = torch.from_numpy(rule_row.astype(np.int32)).to(dev)
        t["rule_dense"] = torch.from_numpy(dense).to(dev, self.t_real)

    def _setup_checked_launches(self) -> None:
        """Launch descriptors of the checked step (health epilogue) and its partial-sum buffer."""
        torch = self.torch
        fused = self.launch_mode == "fused" and self._special.n_special > 0
        probe = self._launches[N.LAUNCH_FUSED if fused else N.LAUNCH_BULK]
        sp = self._special_struct()
        n = N.load().lbm_health_partials(N.C.byref(self.grid), N.C.byref(sp), N.C.byref(probe))
        if n <= 0:
            raise N.NativeError(f"lbm_health_partials: invalid arguments (status {n})")
        self._health_partial = torch.empty(int(n), dtype=torch.float64, device=self.device)
        self._health_struct = N.Health(N.ptr(self._health), N.ptr(self._health_partial), int(n))
        if getattr(self, "_readout", None) is not None:
            self._health_struct.rho, self._health_struct.u = N.ptr(self._readout[0]), N.ptr(self._readout[1:])
        bx, by = self.block
        self._checked_launches = {m: N.Launch(bx, by, m, 0, N.C.pointer(self._health_struct))
                                  for m in N.LAUNCH_MODES}

    def _special_struct(self, export_in=None, export_out=None, tables=None) -> N.Special:
        s = self._special if tables is None else tables
        t = s.tensors
        g = t.get
        local = self._ibm.final_force if self._ibm is not None else None
        return N.Special(
            s.n_special, N.ptr(g("node")), N.ptr(g("rule_mask")), N.ptr(g("rule_first")), N.ptr(g("force_slot")),
            N.ptr(g("export_mask")), N.ptr(g("export_first")), s.n_rules, s.n_terms, N.ptr(g("term_start")),
            N.ptr(g("rule_const")), N.ptr(g("term_dir")), N.ptr(g("term_node")), N.ptr(g("term_export")),
            N.ptr(g("term_coeff")), N.ptr(local), s.n_local, s.n_export, N.ptr(export_in), N.ptr(export_out),
            N.ptr(g("ut_start")), N.ptr(g("ut_slot")), N.ptr(g("ut_export")), N.ptr(g("rule_row")),
            N.ptr(g("rule_dense")),
        )

    # ------------------------------------------------------------------ state
    @property
    def xp(self):
        return self.torch

    @property
    def lattice_bytes(self) -> int:
        """Device memory held by the population buffers (reference ``cuda_solver.py:251-256``)."""
        buffers = 1 if self.variant == "aa" else 2
        return buffers * self.lattice.q * self.n_nodes * self.t_store.itemsize

    @property
    def state_layout(self) -> str:
        return "aa_odd" if self.variant == "aa" else "pull"

    @property
    def _layout_code(self) -> int:
        return N.LAYOUT_AA_ODD if self.variant == "aa" else N.LAYOUT_PULL

    def _field_f64(self, value, lead: tuple[int, ...] = ()):
        """Scalar, host array or tensor broadcast to (*lead, *shape) -> float64 device (*lead, qstride)."""
        torch = self.torch
        shape = (*lead, *self.shape)
        if isinstance(value, torch.Tensor):
            t = value.to(self.device, torch.float64, non_blocking=True)
        else:
            arr = np.asarray(value, dtype=np.float64)
            if arr.ndim == 0:
                return torch.full((*lead, self.qstride), float(arr), dtype=torch.float64, device=self.device)
            t = torch.from_numpy(np.ascontiguousarray(arr)).to(self.device, non_blocking=True)
        t = t.expand(shape)
        if self.pitch == self.shape[-1]:
            return t.reshape(*lead, self.qstride).contiguous()
        out = torch.zeros((*shape[:-1], self.pitch), dtype=torch.float64, device=self.device)
        out[..., : self.shape[-1]] = t
        return out.reshape(*lead, self.qstride)

    def initialize(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0) -> None:
        """Equilibrium with u + F/(2 rho), combined in float64 on the device (reference ``solver.py:101-117``).

        Fields may be scalars, NumPy arrays or torch tensors (pinned host
        tensors are copied asynchronously).
        """
        torch = self.torch
        d = self.lattice.d
        if d == 2 and bool(np.any(np.asarray(uz.cpu() if hasattr(uz, "cpu") else uz) != 0)):
            raise ValueError("a 2D simulation has no z velocity; leave uz at 0")
        rho_t = self._field_f64(rho)
        comps = (ux, uy, uz)[:d]
        u_t = torch.stack([self._field_f64(c) for c in comps])
        self._native("lbm_init_equilibrium", N.C.byref(self.grid), N.C.byref(self.physics), N.ptr(rho_t), N.ptr(u_t),
                     self._layout_code, N.ptr(self._f), self._stream())
        if self._f_next is not None:
            self._f_next.copy_(self._f)
        self._after_state_change()
        self.time_step = 0

    def set_populations(self, f) -> None:
        """Population-exact restore from natural order (q, *shape) (host array or tensor)."""
        torch = self.torch
        q = self.lattice.q
        if isinstance(f, torch.Tensor):
            f = f.detach().cpu().numpy()
        f = np.asarray(f, dtype=np.float64)
        if f.shape != (q, *self.shape):
            raise ValueError(f"populations must have shape {(q, *self.shape)}; got {f.shape}")
        nat = self._to_pitched(f.astype(self.compute), self.t_real)
        self._native("lbm_pack", N.C.byref(self.grid), N.ptr(nat), self._layout_code, N.ptr(self._f), self._stream())
        if self._f_next is not None:
            self._f_next.copy_(self._f)
        self._after_state_change()

    def save_checkpoint(self, path) -> None:
        """Population-exact snapshot on disk.

        ``.npy``: the populations alone, natural direction order, shape (q, *shape), in the compute
        type (exact for every storage format) -- the array ``populations()`` returns, which the
        reference's solvers and the NumPy oracle hold as their state (reference ``solver.py:190-192``).
        Any other suffix (``.npz``): the same populations plus the time step and the step counter of
        the stochastic rounding of 16-bit storage, so that a restored run continues bit for bit.
        """
        if str(path).endswith(".npy"):
            np.save(path, self.populations())
            return
        counter = int(self._seed[:2].cpu().numpy().view(np.uint32).max())
        np.savez(path, populations=self.populations(), time_step=np.int64(self.time_step),
                 round_step=np.uint32(counter), dtype=np.str_(self.params.dtype), shape=np.asarray(self.shape),
                 lattice=np.str_(self.lattice.name))

    def load_checkpoint(self, path) -> None:
        """Restore a ``save_checkpoint`` snapshot of a run with the same lattice, shape and storage
        (a ``.npy`` of natural-order populations from any solver: the time step is left as it is
        and the 16-bit rounding counter restarts at 0)."""
        if str(path).endswith(".npy"):
            self.set_populations(np.load(path))
            return
        with np.load(path) as z:
            if (tuple(int(v) for v in z["shape"]) != tuple(self.shape) or str(z["dtype"]) != self.params.dtype
                    or str(z["lattice"]) != self.lattice.name):
                raise ValueError(f"checkpoint of a {z['lattice']} {tuple(z['shape'])} {z['dtype']} run; this solver "
                                 f"is {self.lattice.name} {tuple(self.shape)} {self.params.dtype}")
            self.set_populations(z["populations"])
            counter = np.array([int(z["round_step"])], dtype=np.uint32).view(np.int32)[0]
            self._seed[:2].fill_(int(counter))
            self.time_step = int(z["time_step"])

    def _after_state_change(self):
        # step counter of the rounding, and the kernel status word: a fresh state
        # starts with no report of an earlier step
        self._seed[:3].zero_()
        self._health_fresh = False
        self._readout_fresh = False
        s = self._special
        if self.variant == "aa" and s.n_export:
            self._export_cur = s.tensors["export_a"]
            self._export_nxt = s.tensors["export_b"]
            sp = self._special_struct()
            self._native("lbm_export_prime", N.C.byref(self.grid), N.C.byref(sp), N.ptr(self._f), N.LAYOUT_AA_ODD,
                         N.ptr(self._export_cur), self._stream())
            # captured graphs baked the export buffers' order in
            self._graphs.clear()

    def _natural_populations(self):
        """Device tensor (q, qstride) of f*_i in natural order, compute dtype."""
        out = self.torch.empty((self.lattice.q, self.qstride), dtype=self.t_real, device=self.device)
        self._native("lbm_unpack", N.C.byref(self.grid), N.ptr(self._f), self._layout_code, N.ptr(out), self._stream())
        return out

    def _device_populations(self):
        """Post-collision populations in natural order, (q, *shape) torch tensor (compute dtype)."""
        t = self._natural_populations()
        view = t.reshape(self.lattice.q, *self.shape[:-1], self.pitch)[..., : self.shape[-1]]
        return view

    def populations(self) -> np.ndarray:
        """Host copy of f~* in natural order, shape (q, *shape) (reference ``solver.py:190-192``)."""
        return self._from_pitched(self._natural_populations())

    def _state_buffer(self):
        return self._f

    # ------------------------------------------------------------------ stepping
    def _step_launch(self, name, sp, *tail, before_boundary=None, checked=False):
        """One time step: a fused launch, or bulk + boundary kernels forked onto two streams.

        ``before_boundary(stream)`` (the immersed-boundary force of a pull step) runs first: on the side
        stream ahead of the boundary kernel when the launch is split, so that it overlaps the bulk
        kernel, which neither reads nor writes what it touches; else ahead of the step on this stream.
        """
        g, ph = N.C.byref(self.grid), N.C.byref(self.physics)
        launches = self._checked_launches if checked else self._launches
        if self.launch_mode == "fused" or self._special.n_special == 0:
            if before_boundary is not None:
                before_boundary(self._stream())
            mode = N.LAUNCH_FUSED if (self._special.n_special and self.launch_mode == "fused") else N.LAUNCH_BULK
            self._native(name, g, ph, N.C.byref(sp), N.C.byref(launches[mode]), N.ptr(self._kind), *tail,
                         self._stream())
            return
        torch = self.torch
        main = torch.cuda.current_stream(self.device)
        side = self._side_stream
        fork, join = torch.cuda.Event(), torch.cuda.Event()
        fork.record(main)
        side.wait_event(fork)
        if before_boundary is not None:
            before_boundary(side.cuda_stream)
        self._native(name, g, ph, N.C.byref(sp), N.C.byref(launches[N.LAUNCH_BOUNDARY]), N.ptr(self._kind), *tail,
                     side.cuda_stream)
        join.record(side)
        self._native(name, g, ph, N.C.byref(sp), N.C.byref(launches[N.LAUNCH_BULK]), N.ptr(self._kind), *tail,
                     main.cuda_stream)
        main.wait_event(join)

    @property
    def _side_stream(self):
        s = getattr(self, "_side", None)
        if s is None:
            s = self._side = self.torch.cuda.Stream(self.device)
        return s

    def _step_pull_ibm(self) -> None:
        """A pull step with an immersed body, three launches on three streams, none waiting on
        another: the body force and its stencil nodes' update (``lbm_step_pull_ibm``), the other
        special nodes (boundary launch), the bulk."""
        torch = self.torch
        g, ph = N.C.byref(self.grid), N.C.byref(self.physics)
        rest, body = self._ibm_split
        ibm = self._ibm
        main = torch.cuda.current_stream(self.device)
        sides = self._side_streams(2)
        fork = torch.cuda.Event()
        fork.record(main)
        joins = []
        for side in sides:
            side.wait_event(fork)
        self._native("lbm_step_pull_ibm", g, ph, N.C.byref(self._special_struct(tables=body)), N.C.byref(ibm.struct),
                     ibm.tables.iterations, N.ptr(self._kind), N.ptr(self._f), N.ptr(self._f_next), N.ptr(ibm.force),
                     sides[0].cuda_stream)
        if rest.n_special:
            self._native("lbm_step_pull", g, ph, N.C.byref(self._special_struct(tables=rest)),
                         N.C.byref(self._launches[N.LAUNCH_BOUNDARY]), N.ptr(self._kind), N.ptr(self._f),
                         N.ptr(self._f_next), sides[1].cuda_stream)
        for side in sides:
            joins.append(torch.cuda.Event())
            joins[-1].record(side)
        self._native("lbm_step_pull", g, ph, N.C.byref(self._special_struct(tables=rest)),
                     N.C.byref(self._launches[N.LAUNCH_BULK]), N.ptr(self._kind), N.ptr(self._f), N.ptr(self._f_next),
                     main.cuda_stream)
        for join in joins:
            main.wait_event(join)
        self._f, self._f_next = self._f_next, self._f

    def _side_streams(self, n: int):
        streams = getattr(self, "_sides", None)
        if streams is None or len(streams) < n:
            streams = self._sides = [self._side_stream] + [self.torch.cuda.Stream(self.device) for _ in range(n - 1)]
        return streams[:n]

    def _launch_pull(self, checked=False):
        if self._ibm_split is not None and not checked and self.launch_mode != "fused":
            self._step_pull_ibm()
            return
        # the immersed-boundary force reads f_src only and feeds only the boundary kernel
        f = self._f
        ibm = None if self._ibm is None else (lambda stream: self._ibm.run(f, N.LAYOUT_PULL, stream))
        sp = self._special_struct()
        self._step_launch("lbm_step_pull", sp, N.ptr(self._f), N.ptr(self._f_next), before_boundary=ibm,
                          checked=checked)
        self._f, self._f_next = self._f_next, self._f

    def _launch_aa(self, parity, layout, checked=False):
        if self._ibm is not None:
            self._ibm.run(self._f, layout)
        ex_in = ex_out = None
        if self._special.n_export:
            ex_in, ex_out = self._export_cur, self._export_nxt
        sp = self._special_struct(ex_in, ex_out)
        self._step_launch("lbm_step_aa", sp, N.ptr(self._f), parity, checked=checked)
        if self._special.n_export:
            self._export_cur, self._export_nxt = self._export_nxt, self._export_cur

    def _launch_steps(self, steps: int):
        if self.variant == "aa":
            for _ in range(steps // 2):
                self._launch_aa(N.LBM_AA_ODD, N.LAYOUT_AA_ODD)
                self._launch_aa(N.LBM_AA_EVEN, N.LAYOUT_AA_EVEN)
        else:
            for _ in range(steps):
                self._launch_pull()

    GRAPH_CHUNK = 32

    def _advance_checked(self, steps: int) -> None:
        """``_advance``, with the state check fused into the last step (the even half of the
        last AA pair): its kernels also flag bad nodes and sum f~* in float64, and
        ``_check_health`` reads the three words instead of scanning the lattice again. Once
        ``macroscopic()`` has been called, the same step also writes rho and u of the state it
        leaves, which the next ``macroscopic()`` returns without reading the lattice again."""
        if steps <= 0:
            return
        m = self.step_multiple
        self._advance(steps - m)
        stream = self._stream()
        self._native("lbm_health_reset", N.ptr(self._health), stream)
        if self.variant == "aa":
            self._launch_aa(N.LBM_AA_ODD, N.LAYOUT_AA_ODD)
            self._launch_aa(N.LBM_AA_EVEN, N.LAYOUT_AA_EVEN, checked=True)
        else:
            self._launch_pull(checked=True)
        mass_bits = self._words[4:5]  # float64 written through its int64 storage
        self._native("lbm_health_finish", N.C.byref(self._health_struct), N.ptr(mass_bits), stream)
        self._health_fresh = True
        self._readout_fresh = self._readout is not None

    def _advance(self, steps: int) -> None:
        if steps <= 0:
            return
        self._health_fresh = False
        self._readout_fresh = False
        if not self.use_graph or steps < self.GRAPH_CHUNK:
            self._launch_steps(steps)
            return
        chunk = self.GRAPH_CHUNK
        graph = self._graph(chunk)
        for _ in range(steps // chunk):
            graph.replay()
        self._launch_steps(steps % chunk)

    def _graph(self, chunk: int):
        """A CUDA graph of ``chunk`` steps; it leaves every buffer pointer where it found it."""
        key = (chunk, self._f.data_ptr())
        graph = self._graphs.get(key)
        if graph is not None:
            return graph
        torch = self.torch
        f0, f1 = self._f, self._f_next
        ex = (getattr(self, "_export_cur", None), getattr(self, "_export_nxt", None))
        stream = torch.cuda.Stream(self.device)
        stream.wait_stream(torch.cuda.current_stream(self.device))
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(stream):
            graph.capture_begin()
            try:
                self._launch_steps(chunk)
            finally:
                graph.capture_end()
        torch.cuda.current_stream(self.device).wait_stream(stream)
        # Capture only recorded the launches; restore the pointer rotation.
        self._f, self._f_next = f0, f1
        self._export_cur, self._export_nxt = ex
        self._graphs[key] = graph
        return graph

    def synchronize(self) -> None:
        self.torch.cuda.synchronize(self.device)

    # ------------------------------------------------------------------ readouts
    def _check_health(self) -> None:
        """Device watchdog (reference ``solver.py:162-172``); raises ``SimulationDiverged``.

        After ``_advance_checked`` (the run loop) the last step has already checked the state
        and summed its mass: one read of five words. Otherwise a separate scan of the lattice.
        """
        fused = self._health_fresh
        if not fused:
            self._native("lbm_health_reset", N.ptr(self._health), self._stream())
            self._native("lbm_health", N.C.byref(self.grid), N.ptr(self._kind), N.ptr(self._f), N.ptr(self._health),
                         self._stream())
        words = self._words.cpu().numpy()
        first, nonfinite = int(words[2]), int(words[3])
        if fused:
            self.mass = self._n_fluid + float(words[4:5].view(np.float64)[0])
        if int(words[:2].view(np.int32)[2]) != 0:
            self._seed[2].zero_()  # reported once; the state itself stays suspect until it is set again
            raise N.NativeError("a step kernel gave up waiting for its staged tiles (TMA loads did not arrive)")
        if first == 2**63 - 1:
            return
        location = _natural_index(first, self.shape, self.pitch)
        reason = "non-finite populations" if nonfinite else "non-positive density"
        raise SimulationDiverged(self.time_step, location, reason)

    def macroscopic(self) -> MacroscopicFields:
        """rho and u on the host (reference ``solver.py:209-221``).

        Straight after the run loop's checked step (``run``), the fields that step wrote (the
        readout fused into it, the same bits as the readout kernel); otherwise one pass of the
        readout kernel over the lattice. The first call also asks the checked steps that follow
        to write the fields."""
        torch = self.torch
        d = self.lattice.d
        if self._readout_fresh:
            fields = self._readout
        else:
            fields = torch.empty((d + 1, self.qstride), dtype=self.t_real, device=self.device)
            rho, u = fields[0], fields[1:]
            local_nodes = local = None
            n_local = 0
            if self._ibm is not None:
                local_nodes = self._ibm.node
                local = self._ibm.final_force
                n_local = self._ibm.tables.n_nodes
            self._native("lbm_macroscopic", N.C.byref(self.grid), N.C.byref(self.physics), N.ptr(self._kind),
                         N.ptr(self._f), self._layout_code, N.ptr(local_nodes), N.ptr(local), n_local, N.ptr(rho),
                         N.ptr(u), self._stream())
        if self._readout is None:
            # solid nodes keep rho = 1, u = 0: the steps write fluid nodes only
            self._readout = torch.zeros((d + 1, self.qstride), dtype=self.t_real, device=self.device)
            self._readout[0].fill_(1.0)
            self._health_struct.rho, self._health_struct.u = N.ptr(self._readout[0]), N.ptr(self._readout[1:])
        host = self._from_pitched(fields)  # one copy for rho and u
        return MacroscopicFields(rho=host[0], u=tuple(host[1 + a] for a in range(d)), solid=np.array(self._solid_host))

    def _device_slots(self, compiled):
        slots = np.asarray(compiled.slots, dtype=np.int64)
        k, node = np.divmod(slots, self.n_nodes)
        return k * self.qstride + self._pitched(node)

    def _affine_tensors(self, compiled):
        """Device slots, coefficients and constants of compiled expressions, uploaded once per
        ``CompiledAffine`` object (a probe read every few steps keeps its tables on the device)."""
        cache = self.__dict__.setdefault("_affine_cache", {})
        hit = cache.get(id(compiled))
        if hit is not None and hit[0] is compiled:
            return hit[1]
        if len(cache) >= 64:
            cache.clear()
        tensors = self._upload_affine(compiled)
        cache[id(compiled)] = (compiled, tensors)
        return tensors

    def _upload_affine(self, compiled):
        torch = self.torch
        coeff = np.asarray(compiled.coeff, dtype=np.float64)
        if coeff.ndim == 1:
            coeff = coeff[:, None]
        slots = self._device_slots(compiled).reshape(coeff.shape)
        const = np.asarray(compiled.constant, dtype=np.float64)
        return (torch.from_numpy(np.ascontiguousarray(slots)).to(self.device),
                torch.from_numpy(np.ascontiguousarray(coeff)).to(self.device),
                torch.from_numpy(np.ascontiguousarray(const)).to(self.device), coeff.shape)

    def evaluate_affine(self, compiled) -> np.ndarray:
        """Host float64 values of compiled affine expressions (reference ``solver.py:178-188``)."""
        slots, coeff, const, (rows, terms) = self._affine_tensors(compiled)
        values = self.torch.empty(rows, dtype=self.torch.float64, device=self.device)
        self._native("lbm_affine_gather", self.grid.storage, N.ptr(self._f), N.ptr(slots), N.ptr(coeff), N.ptr(const),
                     rows, terms, N.ptr(values), self._stream())
        return values.cpu().numpy()

    def reduce_affine(self, compiled, weight) -> np.ndarray:
        """sum_r weight[r] * value_r in float64 on the device (momentum-exchange force)."""
        torch = self.torch
        slots, coeff, const, (rows, terms) = self._affine_tensors(compiled)
        weight = np.asarray(weight, dtype=np.float64).reshape(rows, -1)
        d = weight.shape[1]
        if rows == 0:
            return np.zeros(d)
        key = ("reduce", id(compiled))
        cache = self.__dict__.setdefault("_affine_cache", {})
        hit = cache.get(key)
        if hit is not None and hit[0] is compiled and np.array_equal(hit[2], weight):
            w, partial, counter, out = hit[1]
        else:
            blocks = (rows + 255) // 256
            w = torch.from_numpy(np.ascontiguousarray(weight)).to(self.device)
            partial = torch.empty(blocks * d, dtype=torch.float64, device=self.device)
            counter = torch.zeros(1, dtype=torch.int32, device=self.device)  # re-armed by every reduction
            out = torch.empty(d, dtype=torch.float64, device=self.device)
            cache[key] = (compiled, (w, partial, counter, out), np.array(weight))
        self._native("lbm_affine_reduce", self.grid.storage, N.ptr(self._f), N.ptr(slots), N.ptr(coeff), N.ptr(const),
                     N.ptr(w), rows, terms, d, N.ptr(partial), N.ptr(counter), N.ptr(out), self._stream())
        return out.cpu().numpy()

    def _values_on_device(self, values):
        """Slots, coefficients and constants of an ``AffineSet`` resolved for this solver's stored
        layout on the device (``lbm_compile_terms``: pitched slots of ``state_layout``), once per
        set object."""
        torch = self.torch
        cache = self.__dict__.setdefault("_affine_cache", {})
        key = ("values", id(values))
        hit = cache.get(key)
        if hit is not None and hit[0] is values:
            return hit[1]
        if len(cache) >= 64:
            cache.clear()
        to = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(self.device, dt)  # noqa: E731
        k = to(np.asarray(values.direction, dtype=np.int64), torch.int64)
        y = to(np.asarray(values.node, dtype=np.int64), torch.int64)
        coeff = to(np.asarray(values.coeff, dtype=np.float64), torch.float64)
        const = to(np.asarray(values.constant, dtype=np.float64), torch.float64)
        rows, terms = coeff.shape if coeff.dim() == 2 else (coeff.shape[0], 1)
        slots = torch.empty(rows * terms, dtype=torch.int64, device=self.device)
        self._native("lbm_compile_terms", N.C.byref(self.grid), self._layout_code, None, None, rows * terms, N.ptr(k),
                     N.ptr(y), None, N.ptr(slots), None, self._stream())
        tensors = (slots, coeff.reshape(-1), const, (rows, terms))
        cache[key] = (values, tensors)
        return tensors

    def reduce_affine_values(self, values, weight) -> np.ndarray:
        """sum_r weight[r] * value_r of an uncompiled ``AffineSet`` (terms f*_k(y), natural node
        indices), its slots resolved on the device for this solver's layout; float64 on the device."""
        torch = self.torch
        slots, coeff, const, (rows, terms) = self._values_on_device(values)
        weight = np.asarray(weight, dtype=np.float64).reshape(rows, -1)
        d = weight.shape[1]
        if rows == 0:
            return np.zeros(d)
        w = torch.from_numpy(np.ascontiguousarray(weight)).to(self.device)
        partial = torch.empty((rows + 255) // 256 * d, dtype=torch.float64, device=self.device)
        counter = torch.zeros(1, dtype=torch.int32, device=self.device)
        out = torch.empty(d, dtype=torch.float64, device=self.device)
        self._native("lbm_affine_reduce", self.grid.storage, N.ptr(self._f), N.ptr(slots), N.ptr(coeff), N.ptr(const),
                     N.ptr(w), rows, terms, d, N.ptr(partial), N.ptr(counter), N.ptr(out), self._stream())
        return out.cpu().numpy()

    @property
    def immersed_force(self) -> np.ndarray:
        """Force on the immersed body during the last step, host float64 (reference ``solver.py:201-207``)."""
        if self._ibm is None:
            raise AttributeError("this simulation has no immersed body")
        return self._ibm.body_force()

    def kernel_resources(self) -> dict[str, dict[str, int]]:
        """Registers, spill bytes and shared memory of the step kernels (``cuda_solver.py:311-326``)."""
        lib = N.load()
        variants = {"aa_odd": N.LBM_AA_ODD, "aa_even": N.LBM_AA_EVEN} if self.variant == "aa" else {"pull": N.LBM_PULL}
        modes = {"fused": N.LAUNCH_FUSED} if self.launch_mode == "fused" else {"bulk": N.LAUNCH_BULK,
                                                                               "boundary": N.LAUNCH_BOUNDARY}
        out = {}
        for vname, code in variants.items():
            for mname, mode in modes.items():
                buf = (N.i32 * 4)()
                N.check(lib.lbm_kernel_resources(self.grid.lattice, self.grid.storage, code + 3 * mode, buf),
                        "lbm_kernel_resources")
                out[f"{vname}_{mname}"] = {"registers": buf[0], "local_bytes": buf[1], "shared_bytes": buf[2],
                                           "max_threads": buf[3]}
        return out


class _IbmState:
    """Device tables and scratch of the immersed-boundary kernels for one solver."""

    def __init__(self, solver: CudaSolver, tables):
        torch = solver.torch
        dev, real = solver.device, solver.t_real
        d = solver.lattice.d
        self.solver = solver
        self.tables = tables
        self.d = d
        to = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
        self.node = to(solver._pitched(tables.nodes), torch.int64)
        self._t = {
            "stencil": to(tables.stencil.astype(np.int32), torch.int32),
            "weight": to(tables.weights, real),
            "area": to(tables.areas, real),
            "inv_start": to(tables.inv_start.astype(np.int32), torch.int32),
            "inv_marker": to(tables.inv_marker.astype(np.int32), torch.int32),
            "inv_weight": to(tables.inv_weight, real),
            "rho": torch.zeros(tables.n_nodes, dtype=real, device=dev),
            "u_star": torch.zeros((d, tables.n_nodes), dtype=real, device=dev),
            "marker_force": torch.zeros((tables.iterations, d, tables.n_markers), dtype=real, device=dev),
        }
        # node force after every pass; the last pass's is the one the step adds
        self.force = torch.zeros((tables.iterations, d, tables.n_nodes), dtype=real, device=dev)
        self.final_force = self.force[tables.iterations - 1]
        self._body = torch.zeros(d, dtype=torch.float64, device=dev)
        g = self._t.get
        self.struct = N.Ibm(
            tables.n_nodes, tables.n_markers, tables.stencil.shape[1], N.ptr(self.node), N.ptr(g("stencil")),
            N.ptr(g("weight")), N.ptr(g("area")), N.ptr(g("inv_start")), N.ptr(g("inv_marker")),
            N.ptr(g("inv_weight")), N.ptr(g("rho")), N.ptr(g("u_star")), N.ptr(g("marker_force")),
        )

    def run(self, f, layout: int, stream=None) -> None:
        """Node force of the step from state f (moments + every multi-direct pass, one call)."""
        s = self.solver
        N.call("lbm_ibm_force", N.C.byref(s.grid), N.C.byref(s.physics), N.C.byref(self.struct), N.ptr(f), layout,
               self.tables.iterations, N.ptr(self.force), s._stream() if stream is None else stream)

    def body_force(self) -> np.ndarray:
        s = self.solver
        N.call("lbm_ibm_body_force", N.C.byref(s.grid), N.C.byref(self.struct), self.tables.iterations, N.ptr(self._body), s._stream())
        return self._body.cpu().numpy().astype(np.float64)
