"""The CUDA path against the reference's own CUDA kernels on the same B200 (GPU).

``oracle/ref_kernels.py`` compiles the reference's ``stream_collide_naive``,
``aa_odd``, ``aa_even``, ``stream_collide_tiled`` (2D) and its link-rule
pre-pass (``src/lbm/backends/kernels/*.cu``) unmodified for sm_100a and drives
them as the reference's ``CudaSolver`` does. Both sides
start from the same populations (the oracle's initial state, restored
population-exactly) and advance 40 steps of the reference's mixed-geometry
case: walls, a moving wall, an obstacle and a body force. Bounds: those of the
oracle parity tests (float64 |df| < 1e-15, float32 |df| < 1e-7).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import OracleSolver
from oracle import ref_kernels
from tests import cases
from tests.helpers import NS

import lbm_b200 as lbm

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not ref_kernels.available(), reason="oracle/_ref holds no compiled reference kernels"),
]

ABS = {"float64": 1e-15, "float32": 1e-7}


@pytest.mark.parametrize("variant", ["naive", "aa"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("collision", ["bgk", "trt"])
@pytest.mark.parametrize("d", [2, 3])
def test_step_matches_the_reference_kernels(d, collision, dtype, variant):
    p = cases.mixed(NS, dtype, collision, d)
    start = OracleSolver(p)
    start.initialize(*cases.random_state(p))
    f0 = start.populations()
    ref = ref_kernels.RefSolver(p, variant)
    ref.set_populations(f0)
    ours = lbm.make_solver(p, backend="cuda-aa" if variant == "aa" else "cuda-naive")
    ours.set_populations(f0)
    ref.advance(cases.EQUIVALENCE_STEPS)
    ours.run(cases.EQUIVALENCE_STEPS)
    fluid = p.fluid
    a, b = ref.populations()[:, fluid], ours.populations()[:, fluid]
    diff = float(np.abs(a - b).max())
    assert diff < ABS[dtype], diff
    assert np.isfinite(a).all() and np.abs(a).max() > 1e-4  # the flow is not trivial


@pytest.mark.parametrize("variant", ["naive", "aa"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("case", ["bouzidi", "zou_he"])
@pytest.mark.parametrize("d", [2, 3])
def test_link_rules_match_the_reference_rule_prepass(d, case, dtype, variant):
    """Bouzidi bodies (with a moving wall and a force) and Zou-He inlet/outlet: this build
    evaluates the rules inside its step; the reference runs its rule pre-pass kernels
    (rules_evaluate, rules_write) before each launch, in the launch's layout."""
    if case == "bouzidi":
        p, _ = cases.bouzidi(NS, d, dtype)
    else:
        p, _ = cases.open_channel_case(NS, d, dtype=dtype)
    start = OracleSolver(p)
    start.initialize(*cases.random_state(p, seed=1, u_scale=0.03))
    f0 = start.populations()
    ref = ref_kernels.RefSolver(p, variant)
    assert ref.rule_passes
    ref.set_populations(f0)
    ours = lbm.make_solver(p, backend="cuda-aa" if variant == "aa" else "cuda-naive")
    ours.set_populations(f0)
    ref.advance(cases.EQUIVALENCE_STEPS)
    ours.run(cases.EQUIVALENCE_STEPS)
    fluid = p.fluid
    diff = float(np.abs(ref.populations()[:, fluid] - ours.populations()[:, fluid]).max())
    assert diff < ABS[dtype], diff


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_pull_step_matches_the_reference_tiled_kernel(dtype):
    """The reference's shared-memory tiled kernel (2D only) on the 2D mixed case."""
    p = cases.mixed(NS, dtype, "trt", 2)
    start = OracleSolver(p)
    start.initialize(*cases.random_state(p))
    f0 = start.populations()
    ref = ref_kernels.RefSolver(p, "tiled")
    ref.set_populations(f0)
    ours = lbm.make_solver(p, backend="cuda-naive")
    ours.set_populations(f0)
    ref.advance(cases.EQUIVALENCE_STEPS)
    ours.run(cases.EQUIVALENCE_STEPS)
    fluid = p.fluid
    diff = float(np.abs(ref.populations()[:, fluid] - ours.populations()[:, fluid]).max())
    assert diff < ABS[dtype], diff


@pytest.mark.parametrize("block", [(32, 8), (64, 4), (16, 16)])
def test_reference_launch_shapes_agree_with_ours_on_the_duct(block):
    """The reference's block shape changes nothing; a 64^3 duct (walls in y and z, force)
    in float32 from rest, 20 steps."""
    n = 64
    p = lbm.SimulationParams(nx=n, ny=n, nz=n, tau=0.9, collision="trt", force=(1e-5, 0.0, 0.0),
                             solid=lbm.duct_walls(n, n, n), dtype="float32")
    ours = lbm.make_solver(p, backend="cuda-naive")
    ours.initialize()
    f0 = ours.populations()
    ref = ref_kernels.RefSolver(p, "naive", block=block)
    ref.set_populations(f0)
    ref.advance(20)
    ours.run(20)
    fluid = p.fluid
    diff = float(np.abs(ref.populations()[:, fluid] - ours.populations()[:, fluid]).max())
    assert diff < 1e-7, diff
