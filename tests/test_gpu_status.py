"""The kernel status word: the TMA-staged kernels' bounded waits report, and a new state clears (GPU).

A TMA-staged block that gives up waiting for a tile's staged loads sets bit 0
of the status word (``lbm_physics_t.round_seed[2]``) and returns; the solver's
health check turns it into ``NativeError``. The time-out is made to happen by
a launch whose first wait polls zero times (``LBM_TMA_WAIT_NONE``): every block
gives up at its first tile, then waits -- with the default bound -- for the
loads it has in flight, so no load is outstanding when it exits. Nothing
faults or hangs; the test then checks that the next state runs normally.
"""

from __future__ import annotations

import numpy as np
import pytest

from lbm_b200 import _native as N
from oracle import OracleSolver
from tests import cases
from tests.helpers import NS

import lbm_b200 as lbm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("backend", ["cuda-naive", "cuda-aa"])
def test_tma_wait_time_out_is_reported_and_the_next_state_runs_normally(backend):
    p = cases.duct(NS, n=64, dtype="float16")
    state = cases.random_state(p)
    gpu = lbm.make_solver(p, backend=backend, graph=False)
    gpu.initialize(*state)
    bulk = gpu._launches[N.LAUNCH_BULK]
    bulk.tma_wait_limit = N.TMA_WAIT_NONE
    gpu._advance(2)
    with pytest.raises(N.NativeError, match="gave up waiting"):
        gpu._check_health()
    gpu._check_health()  # reported once
    # default waits again: a fresh state steps like the oracle (4 storage ulps, as the TMA parity tests)
    bulk.tma_wait_limit = 0
    gpu._seed[2].fill_(1)  # a stale report from before is cleared by setting the state
    gpu.initialize(*state)
    gpu.run(4)
    ref = OracleSolver(p)
    ref.initialize(*state)
    ref.run(4)
    a, b = ref.populations()[:, p.fluid], gpu.populations()[:, p.fluid]
    assert np.abs(a - b).max() <= 4 * 2.0**-10 * np.abs(a).max()
    assert np.mean(a == b) > 0.7


def test_a_restored_checkpoint_clears_the_status_word(tmp_path):
    p = cases.duct(NS, n=64, dtype="float16")
    gpu = lbm.make_solver(p, backend="cuda-naive")
    gpu.run(2)
    path = tmp_path / "state.npz"
    gpu.save_checkpoint(path)
    gpu._seed[2].fill_(1)
    gpu.load_checkpoint(path)
    gpu._check_health()
