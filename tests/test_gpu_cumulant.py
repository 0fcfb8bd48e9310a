"""Cumulant collision (``collision="cumulant"``, D2Q9) on the GPU against the oracle.

The reference lists advanced collision models on its roadmap (README, "High
Reynolds numbers") but has none, so the parity anchor is the oracle's FP64/FP32
NumPy restatement of the published method (``oracle.lbm_oracle.collide_cumulant``:
Geier et al. 2015, central moments by the chimera transformation, shear rate
1/tau, bulk and higher-order rates 1, forcing by the half-force velocity shift),
itself pinned by the method's defining properties in ``tests/test_oracle_cumulant.py``.
Same bars as the TRT parity tests (float64 |df| < 1e-15, float32 < 1e-7, 16-bit
storage within 4 storage ulps of the emulating oracle); on a periodic grid,
where a step is streaming plus the collision, the kernels round every
operation as the oracle does, so the states are identical bit for bit.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np
import pytest

from oracle import OracleSolver
from tests import cases
from tests.helpers import NS

import lbm_b200 as lbm

pytestmark = pytest.mark.gpu

BACKENDS = ["cuda-naive", "cuda-aa"]
ABS = {"float64": 1e-15, "float32": 1e-7}
REL = {"float64": 1e-14, "float32": 1e-6}


def cumulant(p):
    return dataclasses.replace(p, collision="cumulant")


def build(name, dtype):
    if name == "mixed":
        return cumulant(cases.mixed(NS, dtype, "trt", 2))
    if name == "bouzidi":
        return cumulant(cases.bouzidi(NS, 2, dtype)[0])
    if name == "ibm":
        return cumulant(cases.ibm(NS, 2, dtype))
    return cumulant(cases.open_channel_case(NS, 2, dtype=dtype)[0])


def run_pair(p, backend, steps=cases.EQUIVALENCE_STEPS, **options):
    state = cases.random_state(p)
    ref = OracleSolver(p)
    gpu = lbm.make_solver(p, backend=backend, **options)
    ref.initialize(*state)
    gpu.initialize(*state)
    ref.run(steps)
    gpu.run(steps)
    return ref, gpu


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("name", ["mixed", "bouzidi", "ibm", "open"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_cumulant_collision_matches_the_oracle(backend, name, dtype):
    p = build(name, dtype)
    ref, gpu = run_pair(p, backend)
    fluid = p.fluid
    a, b = ref.populations()[:, fluid], gpu.populations()[:, fluid]
    diff = np.abs(a - b).max()
    assert diff < ABS[dtype], diff
    assert diff <= REL[dtype] * np.abs(a).max(), diff


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_cumulant_step_is_bit_identical_to_the_oracle_on_a_periodic_grid(backend, dtype):
    p = cumulant(cases.tgv(NS, n=48, dtype=dtype, tau=0.56)[0])
    p = dataclasses.replace(p, force=(2e-6, -1e-6))
    gpu = lbm.make_solver(p, backend=backend)
    gpu.initialize(*cases.random_state(p, u_scale=0.05))
    ref = OracleSolver(p)
    ref.set_populations(gpu.populations())
    gpu.run(12)
    ref.run(12)
    np.testing.assert_array_equal(gpu.populations(), ref.populations())


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
def test_cumulant_collision_in_16bit_storage_matches_the_emulating_oracle(backend, storage):
    p = cumulant(cases.bouzidi(NS, 2, storage, size=(96, 40), body=NS.circle(40.3, 19.6, 7.2))[0])
    ref, gpu = run_pair(p, backend, steps=10)
    a, b = ref.populations()[:, p.fluid], gpu.populations()[:, p.fluid]
    ulp = 2.0**-10 if storage == "float16" else 2.0**-7
    assert np.abs(a - b).max() <= 4 * ulp * np.abs(a).max()
    assert np.mean(a == b) > 0.7


@pytest.mark.parametrize("launch", ["split", "fused"])
def test_cumulant_pull_and_aa_store_the_same_bits(launch):
    p = build("bouzidi", "float64")
    state = cases.random_state(p)
    a = lbm.make_solver(p, backend="cuda-naive", launch=launch)
    b = lbm.make_solver(p, backend="cuda-aa", launch=launch)
    for s in (a, b):
        s.initialize(*state)
        s.run(20)
    np.testing.assert_array_equal(a.populations(), b.populations())


def test_cumulant_taylor_green_decays_at_the_lattice_viscosity():
    """D2Q9 128^2 Taylor-Green vortex, tau = 0.8, 2000 steps: the velocity amplitude follows
    exp(-2 nu k^2 t) within 1e-3 relative."""
    n, tau = 128, 0.8
    p0, state = cases.tgv(NS, n=n, dtype="float64", tau=tau)
    p = cumulant(p0)
    gpu = lbm.make_solver(p, backend="cuda-naive")
    gpu.initialize(*state)
    steps = 2000
    gpu.run(steps)
    ux0 = state[1]
    amp = float((gpu.macroscopic().u[0] * ux0).sum() / (ux0 * ux0).sum())
    k = 2 * math.pi / n
    exact = math.exp(-2 * (tau - 0.5) / 3 * k * k * steps)
    assert abs(amp - exact) / exact < 1e-3


def test_batched_step_rejects_the_cumulant_model():
    from lbm_b200.batched import BatchedSolver

    p = cumulant(cases.cavity(NS, 32, 100.0))
    with pytest.raises(ValueError, match="TRT"):
        BatchedSolver([p])
