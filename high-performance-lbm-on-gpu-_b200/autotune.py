"""Project-written autotuner for launch shapes.

Times a short run of each candidate configuration with CUDA events on the
solver's own workload and keeps the fastest. Results are cached per workload
signature for the life of the process, and in a JSON file when the
``LBM_B200_TUNE_CACHE`` environment variable names one.

* ``tune_step(solver)``  -- bulk tile (x, y) of a ``CudaSolver``.
* ``tune_batch(batch)``  -- bulk tile and persistent grid size of a ``BatchedSolver``.

Tuning runs real time steps; callers re-initialise the state afterwards
(``BatchedSolver`` does so in its constructor).
"""

from __future__ import annotations

import json
import os
from pathlib import Path

TILES = ((32, 4), (32, 8), (64, 2), (64, 4), (128, 1), (128, 2), (256, 1), (32, 2))
_CACHE: dict = {}


def _file():
    path = os.environ.get("LBM_B200_TUNE_CACHE")
    return Path(path) if path else None


def _load():
    f = _file()
    if f is not None and f.exists():
        try:
            _CACHE.update(json.loads(f.read_text()))
        except (OSError, ValueError):
            pass


def _store():
    f = _file()
    if f is not None:
        try:
            f.write_text(json.dumps(_CACHE, indent=1, sort_keys=True))
        except OSError:
            pass


def _time(torch, fn, steps: int, repeats: int = 2) -> float:
    fn(steps)  # warm-up (also builds graphs)
    best = float("inf")
    for _ in range(repeats):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn(steps)
        b.record()
        b.synchronize()
        best = min(best, a.elapsed_time(b) / steps)
    return best


def tune_step(solver, tiles=TILES, steps: int = 20) -> dict:
    """Fastest bulk tile for a CudaSolver's workload; the solver keeps the winner."""
    from . import _native as N

    _load()
    g = solver.grid
    key = f"step:{g.lattice}:{g.storage}:{g.nx}x{g.ny}x{g.nz}:{solver.variant}:{solver.launch_mode}"
    if key not in _CACHE:
        results = {}
        steps += steps % solver.step_multiple
        for tx, ty in tiles:
            solver._launches = {m: N.Launch(tx, ty, m) for m in N.LAUNCH_MODES}
            solver._graphs.clear()
            results[f"{tx}x{ty}"] = _time(solver.torch, solver._advance, steps)
        best = min(results, key=results.get)
        _CACHE[key] = {"block": [int(v) for v in best.split("x")], "ms_per_step": results[best], "tried": results}
        _store()
    best = _CACHE[key]
    tx, ty = best["block"]
    solver._launches = {m: N.Launch(tx, ty, m) for m in N.LAUNCH_MODES}
    solver.block = (tx, ty)
    solver._setup_checked_launches()  # the checked step's partial sums follow the tile
    solver._graphs.clear()
    return best


def tune_batch(batch, tiles=TILES, steps: int = 10, blocks_per_sm=(1, 2, 4, 8)) -> dict:
    """Fastest (tile, persistent grid) for a BatchedSolver's workload."""
    from . import _native as N

    _load()
    sizes = sorted((g.nx, g.ny, g.nz) for g in batch.grids)
    key = f"batch:{batch.grids[0].lattice}:{batch.grids[0].storage}:{len(sizes)}:{hash(tuple(sizes)) & 0xffffffff:08x}"
    if key not in _CACHE:
        results = {}
        for tx, ty in tiles:
            occ = N.i32(0)
            N.check(N.load().lbm_batch_occupancy(batch.grids[0].lattice, batch.grids[0].storage, tx, ty, N.C.byref(occ)),
                    "lbm_batch_occupancy")
            for per in blocks_per_sm:
                if per > max(1, occ.value):
                    continue
                batch.configure((tx, ty), batch.n_sm * per)
                results[f"{tx}x{ty}/{per}"] = _time(batch.torch, batch._advance, steps)
        best = min(results, key=results.get)
        tile, per = best.split("/")
        _CACHE[key] = {"block": [int(v) for v in tile.split("x")], "blocks": batch.n_sm * int(per),
                       "ms_per_step": results[best], "tried": results}
        _store()
    return _CACHE[key]
