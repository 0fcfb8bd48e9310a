"""Many independent domains of uneven size, one persistent launch per step.

``BatchedSolver`` packs every domain's populations, node kinds,
solid-neighbour masks and wall velocities into pooled device buffers, builds
one work list of tiles over all domains and advances all of them with
``lbm_batch_step`` -- a persistent kernel whose blocks walk the list
round-robin without waiting for each other (``csrc/batch.cu``). Steps are
replayed from CUDA graphs. Tile shape and grid size come from
``autotune.tune_batch`` unless given.

The reference has no batched mode; each domain evolves exactly as the same
domain in a ``CudaSolver`` (same per-node code), which the tests check bit for
bit, and as the oracle within the usual tolerances.
"""

from __future__ import annotations

import math

import numpy as np

from . import _native as N
from .diagnostics import MacroscopicFields
from .lattice import as_lattice
from .params import COMPUTE_DTYPE
from .solver import BackendUnavailable, SimulationDiverged, _natural_index

PLANE_ALIGN = 32
"""Direction planes start on 128-byte boundaries (float32): qstride rounded up to 32 elements."""


class BatchedSolver:
    """Advance a list of ``SimulationParams`` (same lattice and dtype) together.

    Args:
        params_list: the domains; no link rules or immersed bodies.
        block: bulk tile (x, y); ``None`` = autotune.
        blocks: persistent grid size; ``None`` = SMs x resident blocks per SM.
        graph: replay steps from CUDA graphs.
    """

    GRAPH_CHUNK = 50

    def __init__(self, params_list, block=None, blocks=None, graph: bool = True, device=None):
        import torch

        if not torch.cuda.is_available():
            raise BackendUnavailable("no CUDA device found")
        try:
            N.load()
        except N.NativeUnavailable as exc:
            raise BackendUnavailable(str(exc)) from exc
        if not params_list:
            raise ValueError("a batch needs at least one domain")
        if any(getattr(p, "collision", "bgk") in ("regularized", "cumulant") for p in params_list):
            raise ValueError("the batched step runs TRT/BGK collision only; use CudaSolver for 'regularized' "
                             "and 'cumulant'")
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.params = list(params_list)
        lat = as_lattice(self.params[0].lattice)
        dtype = self.params[0].dtype
        for p in self.params:
            if as_lattice(p.lattice) is not lat or p.dtype != dtype:
                raise ValueError("every domain of a batch needs the same lattice and dtype")
            if (p.link_rules is not None and len(p.link_rules)) or p.immersed is not None:
                raise ValueError("batched domains support walls and forces only (no link rules or immersed bodies)")
        self.lattice, self.storage = lat, dtype
        self.compute = COMPUTE_DTYPE[dtype]
        tdt = {"float32": torch.float32, "float64": torch.float64, "float16": torch.float16, "bfloat16": torch.bfloat16}
        self.t_store, self.t_real = tdt[dtype], tdt[self.compute]
        self.use_graph = graph
        self._graphs: dict = {}
        self.time_step = 0
        q, d = lat.q, lat.d

        # ---- layout of the pools
        self.grids, self.offsets, self.kind_offsets, self.wall_offsets = [], [], [], []
        off = koff = woff = 0
        walls = 0
        for p in self.params:
            shape = tuple(p.shape)
            nx, ny = shape[-1], shape[-2]
            nz = shape[0] if d == 3 else 1
            # unpadded rows: padded ones made the batched step slower on the 256-cavity
            # batch (32-byte rows 59.8, 128-byte rows 54.7, against 60.4-60.9 GLUPS),
            # unlike a lone lattice (row_pitch)
            pitch = nx
            qstride = -(-pitch * ny * nz // PLANE_ALIGN) * PLANE_ALIGN
            self.grids.append(N.Grid(N.LATTICE_CODE[lat.name], N.STORAGE_CODE[dtype], nx, ny, nz, pitch, qstride))
            self.offsets.append(off)
            self.kind_offsets.append(koff)
            wall = np.asarray(p.wall_velocity, dtype=np.float64)
            if np.any(wall != 0):
                self.wall_offsets.append(woff)
                walls += 1
                woff += d * qstride
            else:
                self.wall_offsets.append(-1)
            off += q * qstride
            koff += qstride
        self.total = off
        self._f = torch.zeros(off, dtype=self.t_store, device=self.device)
        self._g = torch.zeros(off, dtype=self.t_store, device=self.device)
        # step counter (two slots) of the stochastic rounding of 16-bit storage,
        # shared by all domains (they advance together); reset by initialize
        self._seed = torch.zeros(4, dtype=torch.int32, device=self.device)
        self._kind = torch.full((koff,), N.KIND_SOLID, dtype=torch.uint8, device=self.device)
        self._wall = None
        if walls:
            self._wall = torch.zeros(woff, dtype=self.t_real, device=self.device)
            for i, g in enumerate(self.grids):
                w0 = self.wall_offsets[i]
                if w0 < 0:
                    continue
                n = g.nx * g.ny * g.nz
                wall = np.asarray(self.params[i].wall_velocity, dtype=np.float64).reshape(d, n)
                # a writable copy: the parameters' arrays are read-only
                self._wall[w0 : w0 + d * g.qstride].view(d, g.qstride).copy_(
                    self._pitched(i, torch.from_numpy(np.array(wall, copy=True)).to(self.device, self.t_real)))

        # ---- node kinds and solid-neighbour masks, domain by domain
        self._nbr = torch.zeros(koff, dtype=torch.int32, device=self.device)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        for i, (p, g) in enumerate(zip(self.params, self.grids, strict=True)):
            solid = self._pitched(i, torch.from_numpy(np.asarray(p.solid, dtype=np.uint8).reshape(-1)).to(self.device))
            k0 = self.kind_offsets[i]
            N.call("lbm_classify", N.C.byref(g), N.ptr(solid), None, 0, N.ptr(self._kind[k0:]), N.ptr(self._nbr[k0:]),
                   stream)

        # ---- descriptors
        dom = (N.Domain * len(self.params))()
        for i, (p, g) in enumerate(zip(self.params, self.grids, strict=True)):
            wp, wm = p.relaxation_rates
            force = tuple(float(v) for v in p.force) + (0.0,) * (3 - d)
            dom[i] = N.Domain(g.nx, g.ny, g.nz, g.pitch, self.offsets[i], g.qstride, self.kind_offsets[i],
                              self.wall_offsets[i], wp, wm, (N.C.c_double * 3)(*force))
        raw = np.frombuffer(bytes(dom), dtype=np.uint8)
        self._domains = torch.from_numpy(raw.copy()).to(self.device)
        self.n_sm = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.configure(block or (32, 4), blocks)
        if block is None:
            from .autotune import tune_batch

            best = tune_batch(self)
            self.configure(best["block"], blocks if blocks is not None else best["blocks"])
        self.initialize()

    # ------------------------------------------------------------------ layout
    def _pitched(self, i, t):
        """(..., n) node values of domain i in natural order -> (..., qstride), padding zero."""
        g = self.grids[i]
        lead = tuple(t.shape[:-1])
        out = self.torch.zeros((*lead, g.qstride), dtype=t.dtype, device=self.device)
        rows = out[..., : g.pitch * g.ny * g.nz].view(*lead, g.nz, g.ny, g.pitch)
        rows[..., : g.nx] = t.reshape(*lead, g.nz, g.ny, g.nx)
        return out

    def _natural(self, i, t):
        """(..., qstride) of domain i -> (..., *shape): its nodes without the padding."""
        g = self.grids[i]
        lead = tuple(t.shape[:-1])
        rows = t[..., : g.pitch * g.ny * g.nz].reshape(*lead, g.nz, g.ny, g.pitch)[..., : g.nx]
        return rows.reshape(*lead, *self.params[i].shape)

    # ------------------------------------------------------------------ configuration
    def configure(self, block, blocks=None):
        """Set the bulk tile and persistent grid size; rebuilds the tile list."""
        torch = self.torch
        bx, by = (int(v) for v in block)
        if bx <= 0 or by <= 0 or bx % 32 or bx * by > 256:
            raise ValueError(f"block x must be a multiple of 32 and block at most 256 threads; got {block}")
        tiles = []
        for i, g in enumerate(self.grids):
            tx, ty = -(-g.nx // bx), -(-g.ny // by)
            zz, yy, xx = np.meshgrid(np.arange(g.nz), np.arange(ty), np.arange(tx), indexing="ij")
            t = np.stack([np.full(xx.size, i), xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
            tiles.append(t)
        tiles = np.concatenate(tiles).astype(np.int32)
        self._tiles = torch.from_numpy(np.ascontiguousarray(tiles)).to(self.device)
        if blocks is None:
            occ = N.i32(0)
            N.check(N.load().lbm_batch_occupancy(self.grids[0].lattice, self.grids[0].storage, bx, by, N.C.byref(occ)),
                    "lbm_batch_occupancy")
            blocks = self.n_sm * max(1, occ.value)
        self.block, self.blocks = (bx, by), int(blocks)
        self.batch = N.Batch(
            self.grids[0].lattice, self.grids[0].storage, len(self.params), N.ptr(self._domains), len(tiles),
            N.ptr(self._tiles), bx, by, self.blocks, N.ptr(self._kind), N.ptr(self._nbr), N.ptr(self._wall),
            N.ptr(self._seed),
        )
        self._graphs.clear()

    @property
    def nodes(self) -> int:
        return sum(int(np.prod(p.shape)) for p in self.params)

    def _slice(self, buf, i):
        g = self.grids[i]
        return buf[self.offsets[i] : self.offsets[i] + self.lattice.q * g.qstride]

    def _physics(self, i):
        p = self.params[i]
        wp, wm = p.relaxation_rates
        d = self.lattice.d
        force = tuple(float(v) for v in p.force) + (0.0,) * (3 - d)
        wall = None
        if self.wall_offsets[i] >= 0:
            wall = self._wall[self.wall_offsets[i] :]
        return N.Physics(wp, wm, (N.C.c_double * 3)(*force), N.ptr(wall), None, N.ptr(self._nbr[self.kind_offsets[i]:]),
                         N.COLLIDE_TRT, N.ptr(self._seed))

    # ------------------------------------------------------------------ state
    def initialize(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0, domain: int | None = None) -> None:
        """Equilibrium state of one domain (or all, with scalar fields)."""
        torch = self.torch
        targets = range(len(self.params)) if domain is None else [domain]
        stream = torch.cuda.current_stream(self.device).cuda_stream
        d = self.lattice.d
        for i in targets:
            g = self.grids[i]
            shape = tuple(self.params[i].shape)
            # torch.tensor copies: a broadcast (read-only) view is fine
            rho_t = self._pitched(i, torch.tensor(np.broadcast_to(np.asarray(rho, dtype=np.float64), shape).reshape(-1),
                                                  device=self.device))
            u_t = self._pitched(i, torch.stack([
                torch.tensor(np.broadcast_to(np.asarray(c, dtype=np.float64), shape).reshape(-1), device=self.device)
                for c in (ux, uy, uz)[:d]]))
            ph = self._physics(i)
            N.call("lbm_init_equilibrium", N.C.byref(g), N.C.byref(ph), N.ptr(rho_t), N.ptr(u_t), N.LAYOUT_PULL,
                   N.ptr(self._slice(self._f, i)), stream)
        self._g.copy_(self._f)
        self._seed[:2].zero_()
        self._graphs.clear()
        self.time_step = 0

    def populations(self, i: int) -> np.ndarray:
        torch = self.torch
        g = self.grids[i]
        q = self.lattice.q
        out = torch.empty((q, g.qstride), dtype=self.t_real, device=self.device)
        N.call("lbm_unpack", N.C.byref(g), N.ptr(self._slice(self._f, i)), N.LAYOUT_PULL, N.ptr(out),
               torch.cuda.current_stream(self.device).cuda_stream)
        return self._natural(i, out).cpu().numpy()

    def macroscopic(self, i: int) -> MacroscopicFields:
        torch = self.torch
        g = self.grids[i]
        d = self.lattice.d
        rho = torch.empty(g.qstride, dtype=self.t_real, device=self.device)
        u = torch.empty((d, g.qstride), dtype=self.t_real, device=self.device)
        ph = self._physics(i)
        kind = self._kind[self.kind_offsets[i] :]
        N.call("lbm_macroscopic", N.C.byref(g), N.C.byref(ph), N.ptr(kind), N.ptr(self._slice(self._f, i)),
               N.LAYOUT_PULL, None, None, 0, N.ptr(rho), N.ptr(u), torch.cuda.current_stream(self.device).cuda_stream)
        rho_h = self._natural(i, rho).cpu().numpy()
        u_h = self._natural(i, u).cpu().numpy()
        return MacroscopicFields(rho=rho_h, u=tuple(u_h), solid=np.array(self.params[i].solid))

    # ------------------------------------------------------------------ stepping
    def _launch(self):
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        N.call("lbm_batch_step", N.C.byref(self.batch), N.ptr(self._f), N.ptr(self._g), stream)
        self._f, self._g = self._g, self._f

    def _graph(self, chunk):
        key = (chunk, self._f.data_ptr())
        if key in self._graphs:
            return self._graphs[key]
        torch = self.torch
        f0, g0 = self._f, self._g
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            graph.capture_begin()
            try:
                for _ in range(chunk):
                    self._launch()
            finally:
                graph.capture_end()
        torch.cuda.current_stream(self.device).wait_stream(side)
        self._f, self._g = f0, g0
        self._graphs[key] = graph
        return graph

    def _advance(self, steps: int) -> None:
        chunk = self.GRAPH_CHUNK
        if self.use_graph and steps >= chunk:
            graph = self._graph(chunk)
            for _ in range(steps // chunk):
                graph.replay()
            steps %= chunk
        for _ in range(steps):
            self._launch()

    def run(self, steps: int, check: bool = True) -> None:
        if steps < 0:
            raise ValueError(f"need steps >= 0; got {steps}")
        self._advance(steps)
        self.time_step += steps
        if check:
            self.check_health()

    def check_health(self) -> None:
        """Watchdog over every domain; raises ``SimulationDiverged`` with the domain in the message."""
        torch = self.torch
        out = torch.empty(2, dtype=torch.int64, device=self.device)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        for i, g in enumerate(self.grids):
            N.call("lbm_health_reset", N.ptr(out), stream)
            N.call("lbm_health", N.C.byref(g), N.ptr(self._kind[self.kind_offsets[i] :]), N.ptr(self._slice(self._f, i)),
                   N.ptr(out), stream)
            first, nonfinite = (int(v) for v in out.cpu().tolist())
            if first != 2**63 - 1:
                loc = _natural_index(first, tuple(self.params[i].shape), g.pitch)
                raise SimulationDiverged(self.time_step, loc, ("non-finite populations" if nonfinite else "non-positive density")
                                         + f" in domain {i}")

    def run_separately(self, steps: int) -> None:
        """Reference point: every domain launched on its own every step (no batching, no graphs)."""
        stream = self.torch.cuda.current_stream(self.device).cuda_stream
        launch = N.Launch(self.block[0], self.block[1], N.LAUNCH_BULK)
        phys = [self._physics(i) for i in range(len(self.grids))]
        for _ in range(steps):
            for i, g in enumerate(self.grids):
                N.call("lbm_step_pull", N.C.byref(g), N.C.byref(phys[i]), None, N.C.byref(launch),
                       N.ptr(self._kind[self.kind_offsets[i] :]), N.ptr(self._slice(self._f, i)),
                       N.ptr(self._slice(self._g, i)), stream)
            self._f, self._g = self._g, self._f
        self.time_step += steps

    def synchronize(self) -> None:
        self.torch.cuda.synchronize(self.device)


def cavity_batch(lbm, count: int = 256, n_min: int = 64, n_max: int = 512, re_min: float = 100.0,
                 re_max: float = 1000.0, lid: float = 0.1, seed: int = 0, dtype: str = "float32"):
    """The batched-cavity configuration: side n ~ U{n_min..n_max}, Re ~ U(re_min, re_max), seeded.

    tau = 3 lid n / Re + 1/2 (reference ``cases/lid_driven_cavity.py:98-103``).
    """
    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, size=count)
    reynolds = rng.uniform(re_min, re_max, size=count)
    params = []
    for n, re in zip(sizes.tolist(), reynolds.tolist(), strict=True):
        solid, wall = lbm.cavity_walls(n, lid)
        params.append(lbm.SimulationParams(nx=n + 2, ny=n + 2, tau=3.0 * lid * n / re + 0.5, collision="trt",
                                           solid=solid, wall_velocity=wall, dtype=dtype))
    return params, sizes, reynolds


def _total_nodes(params) -> int:
    return sum(math.prod(p.shape) for p in params)
