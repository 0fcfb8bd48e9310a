"""Batched domains: one persistent launch per step over many uneven cavities (GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import OracleSolver
from tests import cases
from tests.helpers import NS

import lbm_b200 as lbm
from lbm_b200.batched import BatchedSolver, cavity_batch

pytestmark = pytest.mark.gpu


def small_batch(dtype="float64", count=5, seed=3):
    params, sizes, _ = cavity_batch(lbm, count=count, n_min=10, n_max=40, seed=seed, dtype=dtype)
    return params, sizes


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_batched_cavities_match_the_oracle(dtype):
    """Oracle parity for a few domains over 200 steps.

    float64: |df| < 1e-15. float32: these cavities run at tau down to 0.503
    with a lid speed of 0.1, where rounding differences grow over 200 steps to
    ~6e-6 of max|f| (measured 2.9e-7 absolute); checked at 2e-5 of max|f|.
    """
    params, _ = small_batch(dtype, count=3)
    batch = BatchedSolver(params, block=(32, 4))
    batch.run(200)
    for i, p in enumerate(params):
        ref = OracleSolver(p)
        ref.run(200)
        fluid = p.fluid
        a = ref.populations()[:, fluid]
        diff = np.abs(a - batch.populations(i)[:, fluid]).max()
        if dtype == "float64":
            assert diff < 1e-15, (i, diff)
        else:
            assert diff <= 2e-5 * np.abs(a).max(), (i, diff)


@pytest.mark.parametrize("block", [(32, 4), (64, 2), (128, 1)])
def test_each_domain_evolves_exactly_as_alone(block):
    params, _ = small_batch("float32", count=6)
    batch = BatchedSolver(params, block=block, blocks=37)
    batch.run(60)
    for i, p in enumerate(params):
        alone = lbm.make_solver(p, backend="cuda-naive")
        alone.run(60)
        np.testing.assert_array_equal(batch.populations(i), alone.populations())


def test_batched_and_separate_launches_agree():
    params, _ = small_batch("float32", count=4)
    a = BatchedSolver(params, block=(32, 4))
    b = BatchedSolver(params, block=(32, 4))
    a.run(40)
    b.run_separately(40)
    for i in range(len(params)):
        np.testing.assert_array_equal(a.populations(i), b.populations(i))


def test_batched_lid_drives_flow_and_conserves_mass():
    params, _ = small_batch("float64", count=3)
    batch = BatchedSolver(params, block=(32, 4))
    m0 = [batch.macroscopic(i).total_mass for i in range(3)]
    batch.run(300)
    for i in range(3):
        f = batch.macroscopic(i)
        assert f.total_mass == pytest.approx(m0[i], rel=1e-13)
        assert np.abs(f.ux).max() > 1e-3


def test_autotuner_picks_a_valid_configuration():
    params, _ = small_batch("float32", count=4)
    batch = BatchedSolver(params)  # block=None -> autotune
    assert batch.block[0] % 32 == 0 and batch.block[0] * batch.block[1] <= 256
    assert batch.blocks >= batch.n_sm
    batch.run(20)
    alone = lbm.make_solver(params[0], backend="cuda-naive")
    alone.run(20)
    np.testing.assert_array_equal(batch.populations(0), alone.populations())


def test_step_autotuner_keeps_results_identical():
    from lbm_b200.autotune import tune_step

    p = cases.mixed(NS, "float32", "trt", 3)
    a = lbm.make_solver(p, backend="cuda-naive")
    best = tune_step(a, steps=4)
    assert tuple(best["block"]) == a.block
    a.initialize(*cases.random_state(p))
    b = lbm.make_solver(p, backend="cuda-naive")
    b.initialize(*cases.random_state(p))
    a.run(8)
    b.run(8)
    np.testing.assert_array_equal(a.populations(), b.populations())


def test_batch_rejects_mixed_dtypes_and_rules():
    p1 = lbm.SimulationParams(nx=8, ny=8, tau=0.8, dtype="float32")
    p2 = lbm.SimulationParams(nx=8, ny=8, tau=0.8, dtype="float64")
    with pytest.raises(ValueError, match="same lattice and dtype"):
        BatchedSolver([p1, p2], block=(32, 4))
    p3, _ = cases.bouzidi(NS, 2, "float32")
    with pytest.raises(ValueError, match="no link rules"):
        BatchedSolver([p3], block=(32, 4))
