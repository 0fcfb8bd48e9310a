"""Population-exact checkpoint and restore on disk (GPU).

A run saved after some steps and restored into a new solver continues bit
for bit like the uninterrupted run -- in 16-bit storage too, whose
stochastic rounding depends on the step counter that the checkpoint carries.
A ``.npy`` snapshot holds the natural-order populations alone (the array
``populations()`` returns): loaded into the NumPy oracle, or into the
reference's own ``ReferenceSolver`` (baseline/_ref), the run continues there
like on the GPU, at the parity bounds.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import OracleSolver, reference_package
from tests import cases
from tests.helpers import NS, reference_ns

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


ABS = {"float64": 1e-15, "float32": 1e-7}


@pytest.mark.parametrize("backend", ["cuda-naive", "cuda-aa"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("d", [2, 3])
def test_npy_snapshot_continues_in_the_oracle(tmp_path, backend, dtype, d):
    params, _ = cases.bouzidi(NS, d, dtype)
    gpu = lbm.make_solver(params, backend=backend)
    gpu.initialize(*cases.random_state(params))
    gpu.run(20)
    path = tmp_path / "state.npy"
    gpu.save_checkpoint(path)
    saved = np.load(path)
    assert saved.shape == (params.lattice.q, *params.shape)
    ref = OracleSolver(params)
    ref.f = np.array(saved, dtype=ref.f.dtype)
    gpu.run(40)
    ref.run(40)
    fluid = params.fluid
    assert np.abs(ref.populations()[:, fluid] - gpu.populations()[:, fluid]).max() < ABS[dtype]
    # and back: the oracle's state restored on a new GPU solver continues like the oracle
    np.save(path, ref.populations())
    again = lbm.make_solver(params, backend=backend)
    again.load_checkpoint(path)
    again.run(10)
    ref.run(10)
    assert np.abs(ref.populations()[:, fluid] - again.populations()[:, fluid]).max() < ABS[dtype]


@pytest.mark.skipif(not reference_package.available(), reason="baseline/_ref (the reference package) is absent")
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_npy_snapshot_continues_in_the_reference_solver(tmp_path, dtype):
    """The snapshot is the reference's own state array: its ReferenceSolver (unmodified, NumPy)
    continues from it like the GPU."""
    ref_pkg = reference_package.modules()
    ns = reference_ns()
    params, _ = cases.bouzidi(ns, 3, dtype)
    gpu = lbm.make_solver(params, backend="cuda-naive")
    gpu.initialize(*cases.random_state(params))
    gpu.run(20)
    path = tmp_path / "state.npy"
    gpu.save_checkpoint(path)
    ref = ref_pkg.backends.make_solver(params, backend="numpy")
    ref._f = np.array(np.load(path), dtype=dtype)  # the reference solver's state array, (q, *shape)
    gpu.run(40)
    ref.run(40)
    fluid = np.asarray(params.fluid)
    assert np.abs(ref.populations()[:, fluid] - gpu.populations()[:, fluid]).max() < ABS[dtype]
