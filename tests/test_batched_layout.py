"""Pool layout of the batched solver on the host (no GPU): natural node order <-> pitched rows."""

from __future__ import annotations

import numpy as np
import torch

from lbm_b200 import _native as N
from lbm_b200.batched import BatchedSolver


def _layout(cases):
    """A BatchedSolver shell holding only the grids and shapes its layout helpers read."""
    b = object.__new__(BatchedSolver)
    b.torch, b.device = torch, torch.device("cpu")
    b.grids, b.params = [], []
    for shape, pitch in cases:
        nz = shape[0] if len(shape) == 3 else 1
        ny, nx = shape[-2], shape[-1]
        qstride = -(-pitch * ny * nz // 32) * 32
        b.grids.append(N.Grid(0, 0, nx, ny, nz, pitch, qstride))
        b.params.append(type("P", (), {"shape": tuple(shape)})())
    return b


def test_pitched_and_natural_round_trip_with_padded_and_plain_rows():
    b = _layout([((5, 7), 8), ((3, 4, 6), 8), ((4, 9), 9), ((2, 3, 5), 5)])
    for i, p in enumerate(b.params):
        g = b.grids[i]
        n = int(np.prod(p.shape))
        t = torch.arange(1, 2 * n + 1, dtype=torch.float64).reshape(2, n)
        padded = b._pitched(i, t)
        assert padded.shape == (2, g.qstride)
        assert int((padded != 0).sum()) == 2 * n  # padding columns and the plane tail stay zero
        # node (z, y, x) of the natural order sits at (z ny + y) pitch + x
        nat = t.reshape(2, g.nz, g.ny, g.nx)
        z, y, x = g.nz - 1, g.ny - 1, g.nx - 1
        assert padded[1, (z * g.ny + y) * g.pitch + x] == nat[1, z, y, x]
        back = b._natural(i, padded)
        assert tuple(back.shape) == (2, *p.shape)
        np.testing.assert_array_equal(back.reshape(2, n).numpy(), t.numpy())
