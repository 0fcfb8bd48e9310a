"""The state check fused into the last step of each run-loop chunk (GPU).

``Solver.run`` advances in chunks and checks the state after each
(reference ``src/lbm/solver.py:119-172``). Here the last step of a chunk is a
checked step: its kernels flag non-finite or non-positive-density nodes and sum
f~* in float64 while they store the state, so the check reads a few words
instead of scanning the lattice again. These tests hold it to three things:
the checked step stores the same bits as a plain one; it reports the same
first bad node as the reference's scan (the oracle's); and its mass is the
float64 sum of the stored state.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import OracleDiverged, OracleSolver
from tests import cases
from tests.helpers import NS

import lbm_b200 as lbm

pytestmark = pytest.mark.gpu

BACKENDS = ["cuda-naive", "cuda-aa"]


def case(name):
    if name == "duct16":
        return cases.duct(NS, n=64, dtype="float16")
    if name == "duct_bf16":
        return cases.duct(NS, n=32, nx=64, dtype="bfloat16")
    if name == "bouzidi3d":
        return cases.bouzidi(NS, 3, "float32")[0]
    if name == "mixed2d":
        return cases.mixed(NS, "float64", "trt", 2)
    if name == "ibm2d":
        return cases.ibm(NS, 2, "float32")
    raise KeyError(name)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("name", ["duct16", "duct_bf16", "bouzidi3d", "mixed2d", "ibm2d"])
@pytest.mark.parametrize("launch", ["split", "fused"])
def test_checked_steps_store_the_bits_of_plain_steps(backend, name, launch):
    p = case(name)
    state = cases.random_state(p)
    plain = lbm.make_solver(p, backend=backend, launch=launch)
    checked = lbm.make_solver(p, backend=backend, launch=launch)
    for s in (plain, checked):
        s.initialize(*state)
    plain._advance(12)
    checked.run(12, check_every=4)  # three checked steps
    np.testing.assert_array_equal(plain.populations(), checked.populations())
    assert checked.mass is not None


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("kind", ["nan", "negative"])
def test_fused_check_reports_the_oracles_first_bad_node(backend, d, kind):
    """Bad values planted in the initial state: same step, same node, same reason as the oracle's
    (the reference's) scan of the state."""
    p = cases.mixed(NS, "float64", "trt", d)
    rho, *u = cases.random_state(p)
    rho = np.array(rho)
    spot = (11, 7, 20)[-d:] if d == 3 else (20, 30)
    if kind == "nan":
        rho[spot] = np.nan
    else:
        rho[tuple(slice(s - 1, s + 2) for s in spot)] = -0.5
    ref = OracleSolver(p)
    ref.initialize(rho, *u)
    with pytest.raises(OracleDiverged) as want:
        ref.run(4, check_every=2)
    gpu = lbm.make_solver(p, backend=backend)
    gpu.initialize(rho, *u)
    with pytest.raises(lbm.SimulationDiverged) as got:
        gpu.run(4, check_every=2)
    assert got.value.step == want.value.step
    assert got.value.location == want.value.location
    assert ("non-finite" in str(got.value)) == ("non-finite" in want.value.reason)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("dtype", ["float64", "float32", "float16"])
def test_fused_mass_is_the_float64_sum_of_the_stored_state(backend, dtype):
    p = cases.mixed(NS, dtype, "trt", 3) if dtype != "float16" else cases.duct(NS, n=32, nx=64, dtype=dtype)
    gpu = lbm.make_solver(p, backend=backend)
    gpu.initialize(*cases.random_state(p))
    gpu.run(8, check_every=8)
    f = gpu.populations().astype(np.float64)[:, p.fluid]
    want = p.fluid.sum() + f.sum()
    assert abs(gpu.mass - want) <= 1e-12 * want
    if dtype == "float64":  # and the oracle's own state
        ref = OracleSolver(p)
        ref.initialize(*cases.random_state(p))
        ref.run(8)
        want = p.fluid.sum() + ref.populations()[:, p.fluid].sum()
        assert abs(gpu.mass - want) <= 1e-12 * want


@pytest.mark.parametrize("backend", BACKENDS)
def test_closed_box_mass_stays_put_through_the_run_loop(backend):
    """A closed 3D box with a moving lid conserves mass: every chunk's fused float64 sum agrees
    with the first, and with the mass of the macroscopic readout."""
    solid, wall = lbm.cavity_walls(n=14, lid_velocity=0.05, dimensions=3)
    p = lbm.SimulationParams(nx=16, ny=16, nz=16, tau=0.7, solid=solid, wall_velocity=wall, dtype="float64")
    gpu = lbm.make_solver(p, backend=backend)
    m0 = gpu.macroscopic().total_mass
    seen = []
    gpu.run(400, every=100, check_every=100, callback=lambda s: seen.append(s.mass))
    assert len(seen) == 4
    for m in seen:
        assert m == pytest.approx(m0, rel=1e-13)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("name", ["duct16", "bouzidi3d", "mixed2d", "ibm2d"])
@pytest.mark.parametrize("launch", ["split", "fused"])
def test_readout_fused_into_the_checked_step_equals_the_readout_kernel(backend, name, launch):
    """Once macroscopic() has been asked for, the run loop's checked step also writes rho and u
    (reference diagnostics.py:72-80); the next macroscopic() returns them, bit for bit what the
    separate readout pass gives for the same state, and within the parity bounds of the oracle's."""
    p = case(name)
    state = cases.random_state(p)
    gpu = lbm.make_solver(p, backend=backend, launch=launch)
    ref = OracleSolver(p)
    gpu.initialize(*state)
    ref.initialize(*state)
    gpu.run(4, check_every=4)
    ref.run(4)
    first = gpu.macroscopic()  # the readout pass; asks the following checked steps for the fields
    assert not gpu._readout_fresh
    gpu.run(8, check_every=4)
    ref.run(8)
    assert gpu._readout_fresh
    fused = gpu.macroscopic()
    gpu._readout_fresh = False  # the same state through the separate readout pass
    separate = gpu.macroscopic()
    np.testing.assert_array_equal(fused.rho, separate.rho)
    for a, b in zip(fused.u, separate.u, strict=True):
        np.testing.assert_array_equal(a, b)
    assert not np.array_equal(first.rho, fused.rho)
    want = ref.macroscopic()
    tol = {"float64": 1e-14, "float32": 1e-6}.get(p.dtype, 2e-4)  # 16-bit: a few storage ulps
    np.testing.assert_allclose(fused.rho, want[0], rtol=0, atol=tol)
    for a in range(p.d):
        np.testing.assert_allclose(fused.u[a], want[1][a], rtol=0, atol=tol)


def test_a_plain_step_or_a_new_state_retires_the_fused_readout():
    p = case("mixed2d")
    gpu = lbm.make_solver(p, backend="cuda-naive")
    gpu.initialize(*cases.random_state(p))
    gpu.macroscopic()
    gpu.run(4, check_every=4)
    assert gpu._readout_fresh
    gpu._advance(2)
    assert not gpu._readout_fresh
    gpu.run(4, check_every=4)
    assert gpu._readout_fresh
    gpu.initialize(*cases.random_state(p, seed=1))
    assert not gpu._readout_fresh
    gpu.run(4, check_every=4)
    gpu.set_populations(gpu.populations())
    assert not gpu._readout_fresh
