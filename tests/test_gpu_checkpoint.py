"""Population-exact checkpoint and restore on disk (GPU).

A run saved after some steps and restored into a new solver continues bit
for bit like the uninterrupted run -- in 16-bit storage too, whose
stochastic rounding depends on the step counter that the checkpoint carries.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests import cases
from tests.helpers import NS

import lbm_b200 as lbm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("backend,dtype,d", [
    ("cuda-naive", "float32", 2),
    ("cuda-aa", "float64", 3),
    ("cuda-naive", "float16", 3),
    ("cuda-aa", "bfloat16", 2),
])
def test_restored_run_continues_bit_for_bit(tmp_path, backend, dtype, d):
    params, _ = cases.bouzidi(NS, d, dtype)
    state = cases.random_state(params)
    a = lbm.make_solver(params, backend=backend)
    a.initialize(*state)
    a.run(12)
    path = tmp_path / "state.npz"
    a.save_checkpoint(path)
    a.run(10)
    b = lbm.make_solver(params, backend=backend)
    b.load_checkpoint(path)
    assert b.time_step == 12
    b.run(10)
    assert b.time_step == a.time_step == 22
    np.testing.assert_array_equal(b.populations(), a.populations())


def test_checkpoint_of_another_grid_is_rejected(tmp_path):
    params, _ = cases.bouzidi(NS, 2, "float32")
    a = lbm.make_solver(params, backend="cuda-naive")
    path = tmp_path / "state.npz"
    a.save_checkpoint(path)
    other, _ = cases.bouzidi(NS, 2, "float64")
    b = lbm.make_solver(other, backend="cuda-naive")
    with pytest.raises(ValueError, match="checkpoint"):
        b.load_checkpoint(path)
