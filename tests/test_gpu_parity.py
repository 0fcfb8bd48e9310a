"""CUDA path against the oracle: the parity contract of the hot path (GPU).

Mirrors the reference's GPU-equivalence tests (``tests/test_cuda_backend.py``,
``test_geometry_link_rules.py``, ``test_ibm.py``, ``test_open_boundaries.py``):
random initial state (rho = 1 + 0.01 N, u = 0.02 N, seed 0), 40 steps, fluid
nodes compared. Tolerances: float64 |df| < 1e-15 and max|df|/max|f| <= 1e-14;
float32 |df| < 1e-7 and relative <= 1e-6 -- the reference's absolute bounds and
the relative bounds of the build target, whichever is tighter.
"""

from __future__ import annotations

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


def run_pair(params, backend, state=None, steps=cases.EQUIVALENCE_STEPS, **options):
    ref = OracleSolver(params)
    gpu = lbm.make_solver(params, backend=backend, **options)
    if state is not None:
        ref.initialize(*state)
        gpu.initialize(*state)
    ref.run(steps)
    gpu.run(steps)
    return ref, gpu


def assert_parity(params, ref, gpu, dtype=None):
    dtype = dtype or params.dtype
    fluid = params.fluid
    a, b = ref.populations()[:, fluid], gpu.populations()[:, fluid]
    diff = np.abs(a - b).max()
    assert diff < ABS[dtype], diff
    assert diff <= REL[dtype] * np.abs(a).max(), diff


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("collision", ["bgk", "trt"])
def test_float64_matches_oracle_to_round_off(backend, d, collision):
    p = cases.mixed(NS, "float64", collision, d)
    ref, gpu = run_pair(p, backend, cases.random_state(p))
    assert_parity(p, ref, gpu)


DEGENERATE = [(1, 7), (7, 1), (3, 2), (33, 5), (64, 3), (1, 4, 3), (5, 1, 3), (6, 4, 1), (33, 3, 2), (64, 2, 2)]


@pytest.mark.parametrize("storage", ["float64", "float32", "float16", "bfloat16"])
@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("size", DEGENERATE, ids=lambda s: "x".join(map(str, s)))
def test_degenerate_and_ragged_grids_match_oracle(backend, size, storage):
    """Fully periodic grids one or two nodes thick, odd widths, rows shorter than a
    warp, and power-of-two widths that the TMA-staged 16-bit kernels take with
    fewer rows than a tile needs for staging: every node wraps onto itself or
    its one neighbour. 10 steps from a random state with a body force; float64
    and float32 to the parity bounds, 16-bit storage within 4 storage ulps of
    max|f| of the emulating oracle."""
    d = len(size)
    dims = dict(zip(("nx", "ny", "nz"), size))
    force = (1e-5, -2e-6, 3e-6)[:d]
    p = NS.SimulationParams(**dims, tau=0.7, collision="trt", force=force, dtype=storage)
    ref, gpu = run_pair(p, backend, cases.random_state(p), steps=10)
    if storage in ABS:
        assert_parity(p, ref, gpu)
    else:
        a, b = ref.populations(), gpu.populations()
        ulp = 2.0**-10 if storage == "float16" else 2.0**-7
        assert np.abs(a - b).max() <= 4 * ulp * np.abs(a).max()


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_float32_matches_oracle(backend, d):
    p = cases.mixed(NS, "float32", "trt", d)
    ref, gpu = run_pair(p, backend, cases.random_state(p))
    assert_parity(p, ref, gpu)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_macroscopic_fields_match_oracle(backend, d):
    p = cases.mixed(NS, "float64", "trt", d)
    ref, gpu = run_pair(p, backend, cases.random_state(p))
    rho, u = ref.macroscopic()
    out = gpu.macroscopic()
    np.testing.assert_allclose(out.rho, rho, rtol=0, atol=1e-14)
    for a in range(d):
        np.testing.assert_allclose(out.u[a], u[a], rtol=0, atol=1e-14)


@pytest.mark.parametrize("backend", BACKENDS)
def test_closed_3d_box_with_moving_lid_conserves_mass(backend):
    solid, wall = lbm.cavity_walls(n=14, lid_velocity=0.05, dimensions=3)
    p = lbm.SimulationParams(nx=16, ny=16, nz=16, tau=0.7, solid=solid, wall_velocity=wall, dtype="float64")
    s = lbm.make_solver(p, backend=backend)
    m0 = s.macroscopic().total_mass
    s.run(400)
    assert s.macroscopic().total_mass == pytest.approx(m0, rel=1e-13)


def test_aa_backend_advances_in_pairs_only():
    s = lbm.make_solver(lbm.SimulationParams(nx=8, ny=8, tau=0.8), backend="cuda-aa")
    with pytest.raises(ValueError, match="multiples of 2"):
        s.run(3)
    s.run(4)
    assert s.time_step == 4


def test_aa_backend_uses_half_the_lattice_memory():
    p = lbm.SimulationParams(nx=64, ny=32, tau=0.8)
    naive, aa = lbm.make_solver(p, backend="cuda-naive"), lbm.make_solver(p, backend="cuda-aa")
    assert aa.lattice_bytes * 2 == naive.lattice_bytes == 2 * 9 * 64 * 32 * 4
    p3 = lbm.SimulationParams(nx=16, ny=12, nz=8, tau=0.8)
    assert lbm.make_solver(p3, backend="cuda-aa").lattice_bytes == 19 * 16 * 12 * 8 * 4


@pytest.mark.parametrize("dtype", ["float32", "float64", "float16", "bfloat16"])
@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_kernels_keep_populations_in_registers(backend, d, dtype):
    sizes = {"nx": 8, "ny": 8} | ({"nz": 8} if d == 3 else {})
    s = lbm.make_solver(lbm.SimulationParams(**sizes, tau=0.8, dtype=dtype), backend=backend)
    for name, res in s.kernel_resources().items():
        assert res["local_bytes"] == 0, f"{name} spills to local memory"


def test_invalid_block_is_rejected():
    with pytest.raises(ValueError, match="block"):
        lbm.make_solver(lbm.SimulationParams(nx=8, ny=8, tau=0.8), backend="cuda-naive", block=(64, 32))


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_bouzidi_matches_oracle(backend, d):
    """Every rule layout of the reference (pull, AA odd, AA even) is exercised here."""
    for dtype in ("float64", "float32"):
        p, _ = cases.bouzidi(NS, d, dtype)
        ref, gpu = run_pair(p, backend, cases.random_state(p))
        assert_parity(p, ref, gpu)


@pytest.mark.parametrize("backend", BACKENDS)
def test_bouzidi_with_q_one_half_equals_plain_bounce_back(backend):
    body = lbm.circle(15.3, 10.4, 4.6)
    solid = lbm.channel_walls(33, 21) | lbm.voxelize(body, (21, 33))
    links = lbm.wall_links(lbm.D2Q9, body, solid)
    half = lbm.WallLinks(links.node, links.direction, np.full(len(links), 0.5))
    common = dict(nx=33, ny=21, tau=0.7, collision="trt", force=(1e-5, 0.0), solid=solid, dtype="float64")
    plain = lbm.make_solver(lbm.SimulationParams(**common), backend=backend)
    ruled = lbm.make_solver(lbm.SimulationParams(**common, link_rules=lbm.bouzidi_rules(lbm.D2Q9, half, solid)), backend=backend)
    for s in (plain, ruled):
        s.run(30)
    np.testing.assert_allclose(ruled.populations(), plain.populations(), rtol=0, atol=1e-16)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_force_probe_reads_every_layout_the_same(backend, d):
    p, links = cases.bouzidi(NS, d, "float64")
    probe = lbm.ForceProbe.build(p, links)
    ref, gpu = run_pair(p, backend, cases.random_state(p))
    expect = probe.weight.T @ ref.evaluate_affine(probe.compiled("reference"))
    np.testing.assert_allclose(probe.evaluate(gpu), expect, rtol=1e-12, atol=1e-16)
    values = gpu.evaluate_affine(probe.compiled(gpu.state_layout))
    np.testing.assert_allclose(probe.weight.T @ values, expect, rtol=1e-12, atol=1e-16)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_ibm_matches_oracle(backend, d):
    """Body force: rtol 1e-13 (fp64, measured 1.04e-14) and 1e-5 (fp32, measured
    1.4e-6). It is a sum of ~100-800 marker forces of both signs: the oracle
    sums them in the storage precision, the kernels in float64."""
    for dtype, rtol in (("float64", 1e-13), ("float32", 1e-5)):
        p = cases.ibm(NS, d, dtype)
        ref, gpu = run_pair(p, backend, cases.random_state(p))
        assert_parity(p, ref, gpu)
        np.testing.assert_allclose(gpu.immersed_force, ref.immersed_force, rtol=rtol)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("radius,size,path", [(1.4, (24, 20, 20), "tables"), (2.5, (24, 20, 20), "shared"),
                                              (4.5, (32, 24, 24), "global"), (9.5, (48, 36, 36), "per-pass")])
def test_every_immersed_boundary_kernel_path_matches_oracle(backend, radius, size, path):
    """lbm_ibm_force runs a body in one block with its arrays and tables in shared memory
    when both fit, with its arrays alone there when they fit, in one block on global
    memory up to 4096 stencil nodes and markers, and with a launch per pass beyond:
    spheres sized for each path (float64)."""
    from lbm_b200 import _native as N
    from lbm_b200.ibm import build_tables

    nx, ny, nz = size
    body = NS.sphere(nx / 2 - 0.3, (ny - 1) / 2 + 0.2, (nz - 1) / 2 - 0.1, radius)
    p = cases.ibm(NS, 3, "float64", size=size, body=body)
    t = build_tables(p.immersed, p.lattice, np.asarray(p.solid))
    smem = (t.n_nodes * 13 + 3 * t.n_markers) * 8
    tables = t.n_markers * 55 * 8 + (t.n_markers * 54 + t.n_nodes + 1) * 4
    taken = ("tables" if smem + tables <= N.IBM_SMEM_BYTES else "shared" if smem <= N.IBM_SMEM_BYTES else
             "global" if max(t.n_nodes, t.n_markers) <= N.IBM_FUSED_MAX else "per-pass")
    assert taken == path
    ref, gpu = run_pair(p, backend, cases.random_state(p), steps=10)
    assert_parity(p, ref, gpu)
    np.testing.assert_allclose(gpu.immersed_force, ref.immersed_force, rtol=1e-13)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_open_boundaries_match_oracle(backend, d):
    p, _ = cases.open_channel_case(NS, d)
    ref, gpu = run_pair(p, backend, cases.random_state(p, seed=1, u_scale=0.03))
    assert_parity(p, ref, gpu)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("case", ["bouzidi", "open"])
def test_dense_and_term_by_term_rules_both_match_the_oracle(backend, d, case):
    """The boundary warps evaluate rules in the dense per-node form by default; the term-by-term
    form stays for nodes whose rules read more than 32 distinct populations. Both against the
    oracle (float64), and against each other to round-off (the summation order differs)."""
    if case == "bouzidi":
        p, _ = cases.bouzidi(NS, d, "float64")
        state = cases.random_state(p)
    else:
        p, _ = cases.open_channel_case(NS, d)
        state = cases.random_state(p, seed=1, u_scale=0.03)
    ref, dense = run_pair(p, backend, state)
    _, terms = run_pair(p, backend, state, dense_rules=False)
    assert dense._special.tensors.get("ut_start") is not None
    assert terms._special.tensors.get("ut_start") is None
    assert_parity(p, ref, dense)
    assert_parity(p, ref, terms)
    fluid = p.fluid
    assert np.abs(dense.populations()[:, fluid] - terms.populations()[:, fluid]).max() < 1e-15


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_watchdog_reports_step_and_location(backend, d):
    sizes = {"nx": 8, "ny": 8} | ({"nz": 8} if d == 3 else {})
    s = lbm.make_solver(lbm.SimulationParams(**sizes, tau=0.8, dtype="float64"), backend=backend)
    rho = np.ones(s.shape)
    rho[(3, 5, 2)[:d]] = np.nan
    s.initialize(rho)
    with pytest.raises(lbm.SimulationDiverged) as info:
        s.run(10, check_every=2)
    assert info.value.step == 2
    assert len(info.value.location) == d


@pytest.mark.parametrize("backend", BACKENDS)
def test_vanishing_density_raises(backend):
    s = lbm.make_solver(lbm.SimulationParams(nx=8, ny=8, tau=0.8, dtype="float64"), backend=backend)
    rho = np.ones(s.shape)
    rho[1:4, 1:4] = -0.5
    s.initialize(rho)
    with pytest.raises(lbm.SimulationDiverged, match="density"):
        s.run(2, check_every=2)


@pytest.mark.parametrize("backend", BACKENDS)
def test_run_counts_steps_and_fires_callback(backend):
    s = lbm.make_solver(lbm.SimulationParams(nx=8, ny=8, tau=0.8), backend=backend)
    seen = []
    s.run(12, every=4, callback=lambda sv: seen.append(sv.time_step))
    assert s.time_step == 12 and seen == [4, 8, 12]


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_uniform_flow_is_an_exact_steady_state(backend, d):
    velocity = (0.05, -0.02, 0.01)[:d]
    sizes = {"nx": 8, "ny": 8} | ({"nz": 8} if d == 3 else {})
    s = lbm.make_solver(lbm.SimulationParams(**sizes, tau=0.8, dtype="float64"), backend=backend)
    s.initialize(1.0, *velocity)
    s.run(50)
    f = s.macroscopic()
    for got, want in zip(f.u, velocity, strict=True):
        np.testing.assert_allclose(got, want, atol=1e-14)
    np.testing.assert_allclose(f.rho, 1.0, atol=1e-14)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_body_force_accelerates_periodic_fluid_by_f_per_step(backend, d):
    force = (1e-5, -2e-5, 3e-5)[:d]
    sizes = {"nx": 8, "ny": 8} | ({"nz": 8} if d == 3 else {})
    s = lbm.make_solver(lbm.SimulationParams(**sizes, tau=0.8, dtype="float64", force=force), backend=backend)
    s.run(40)
    for got, fa in zip(s.macroscopic().u, force, strict=True):
        np.testing.assert_allclose(got, 40 * fa, rtol=1e-10)


@pytest.mark.parametrize("backend", BACKENDS)
def test_populations_round_trip_exactly(backend):
    p = cases.mixed(NS, "float64", "trt", 3)
    s = lbm.make_solver(p, backend=backend)
    s.initialize(*cases.random_state(p))
    s.run(6)
    f = s.populations()
    s2 = lbm.make_solver(p, backend=backend)
    s2.set_populations(f)
    np.testing.assert_array_equal(s2.populations(), f)
    s.run(6)
    s2.run(6)
    np.testing.assert_array_equal(s2.populations(), s.populations())


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_pull_and_aa_give_identical_bits(d, dtype):
    """Both variants compute the same per-node arithmetic on the same inputs."""
    p, _ = cases.bouzidi(NS, d, dtype)
    state = cases.random_state(p)
    a = lbm.make_solver(p, backend="cuda-naive")
    b = lbm.make_solver(p, backend="cuda-aa")
    for s in (a, b):
        s.initialize(*state)
        s.run(20)
    np.testing.assert_array_equal(a.populations()[:, p.fluid], b.populations()[:, p.fluid])


def test_tiled_backend_name_runs_the_pull_step():
    """The reference's 2D-only cuda-tiled name: the same bits as cuda-naive."""
    p = cases.mixed(NS, "float32", "trt", 2)
    a = lbm.make_solver(p, backend="cuda-tiled")
    b = lbm.make_solver(p, backend="cuda-naive")
    for s in (a, b):
        s.initialize(*cases.random_state(p))
        s.run(10)
    np.testing.assert_array_equal(a.populations(), b.populations())


@pytest.mark.parametrize("backend", BACKENDS)
def test_graph_and_eager_launches_agree(backend):
    p = cases.mixed(NS, "float32", "trt", 2)
    a = lbm.make_solver(p, backend=backend, graph=True)
    b = lbm.make_solver(p, backend=backend, graph=False)
    for s in (a, b):
        s.initialize(*cases.random_state(p))
        s.run(70)
    np.testing.assert_array_equal(a.populations(), b.populations())


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("pitch", [64, 96])
def test_padded_row_pitch_changes_nothing(backend, pitch):
    p, links = cases.bouzidi(NS, 2, "float64")
    probe = lbm.ForceProbe.build(p, links)
    a = lbm.make_solver(p, backend=backend)
    b = lbm.make_solver(p, backend=backend, pitch=pitch)
    for s in (a, b):
        s.initialize(*cases.random_state(p))
        s.run(10)
    np.testing.assert_array_equal(a.populations(), b.populations())
    np.testing.assert_array_equal(probe.evaluate(a), probe.evaluate(b))


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_16bit_storage_matches_emulating_oracle(backend, d, storage):
    """The oracle rounds to the storage format like the kernels do.

    float32 arithmetic differs by an ulp here and there (FMA contraction,
    summation order) and can flip a 16-bit rounding; after 10 steps the
    largest difference stays within 4 storage ulps of max|f| and 79-92 % of
    the stored values are bit-identical (measured), so > 70 % is required.
    """
    p = cases.mixed(NS, storage, "trt", d)
    ref, gpu = run_pair(p, backend, cases.random_state(p), steps=10)
    fluid = p.fluid
    a, b = ref.populations()[:, fluid], gpu.populations()[:, fluid]
    ulp = 2.0**-10 if storage == "float16" else 2.0**-7
    assert np.abs(a - b).max() <= 4 * ulp * np.abs(a).max()
    assert np.mean(a == b) > 0.7


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
@pytest.mark.parametrize("backend,size", [("cuda-naive", (16, 20, 16)), ("cuda-naive", (32, 20, 16)),
                                          ("cuda-naive", (64, 20, 16)), ("cuda-naive", (64, 21, 7)),
                                          ("cuda-aa", (64, 20, 16)), ("cuda-aa", (128, 20, 16)),
                                          ("cuda-aa", (64, 21, 7))])
def test_16bit_tma_kernels_with_walls_bodies_and_rules_match_the_oracle(backend, size, storage):
    """Grids the TMA-staged kernels take (nx a power of two): a channel with a moving wall,
    z walls, a Bouzidi sphere and a force, so tiles mix staged nodes, wall neighbours
    (bounce-back with the Ladd term), rule nodes (left to the boundary warps) and warps
    that fall back to the one-node path; several rows per warp at nx = 16 and 32 (which
    the node-pair kernel takes), an odd row count (a last tile with one row) and a thin
    z extent. Same bar as the emulating-oracle test above."""
    nx, ny, nz = size
    body = NS.sphere(nx / 2 - 0.3, (ny - 1) / 2 + 0.1, (nz - 1) / 2 + 0.2, min(4.1, (nz - 3) / 2))
    p, _ = cases.bouzidi(NS, 3, storage, size=size, body=body)
    ref, gpu = run_pair(p, backend, cases.random_state(p), steps=10)
    fluid = p.fluid
    a, b = ref.populations()[:, fluid], gpu.populations()[:, fluid]
    ulp = 2.0**-10 if storage == "float16" else 2.0**-7
    assert np.abs(a - b).max() <= 4 * ulp * np.abs(a).max()
    assert np.mean(a == b) > 0.7


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
@pytest.mark.parametrize("size", [(48, 20, 16), (200, 20, 12), (250, 12, 6), (96, 40)],
                         ids=lambda s: "x".join(map(str, s)))
def test_16bit_odd_half_on_widths_the_tma_kernel_does_not_take(size, storage):
    """The odd AA half's one-row-per-block kernel (even widths up to 256 that are not a power of two
    in [64, 256], and D2Q9): walls, a moving wall, a Bouzidi body and a force, against the emulating
    oracle within 4 storage ulps (as the TMA kernels' test)."""
    if len(size) == 3:
        nx, ny, nz = size
        body = NS.sphere(nx / 2 - 0.3, (ny - 1) / 2 + 0.1, (nz - 1) / 2 + 0.2, min(4.1, (nz - 3) / 2))
        p, _ = cases.bouzidi(NS, 3, storage, size=size, body=body)
    else:
        nx, ny = size
        p, _ = cases.bouzidi(NS, 2, storage, size=size, body=NS.circle(nx / 3 + 0.3, ny / 2 - 0.4, 6.2))
    state = cases.random_state(p)
    ref, gpu = run_pair(p, "cuda-aa", state, steps=10)
    fluid = p.fluid
    a, b = ref.populations()[:, fluid], gpu.populations()[:, fluid]
    ulp = 2.0**-10 if storage == "float16" else 2.0**-7
    assert np.abs(a - b).max() <= 4 * ulp * np.abs(a).max()
    assert np.mean(a == b) > 0.7


@pytest.mark.parametrize("storage", ["float16", "bfloat16"])
@pytest.mark.parametrize("nx", [48, 200, 250, 320])
def test_16bit_odd_row_kernel_gives_the_pull_steps_bits_in_a_duct(nx, storage):
    """In a duct (resting walls, a force) the AA pair with the one-row odd kernel stores the bits
    of two pull steps, as the TMA kernels do at 256^3 (with a moving wall the two schemes round the
    wall term at different points, so there only the oracle bound holds)."""
    p = cases.duct(NS, n=24, nx=nx, dtype=storage)
    state = cases.random_state(p)
    runs = []
    for backend in ("cuda-naive", "cuda-aa"):
        s = lbm.make_solver(p, backend=backend)
        s.initialize(*state)
        s.run(10)
        runs.append(s.populations())
    np.testing.assert_array_equal(runs[0], runs[1])


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("d", [2, 3])
def test_fused_and_split_launches_give_identical_bits(backend, d):
    """Boundary warps in the step launch or in a concurrent second kernel: same result."""
    p, _ = cases.bouzidi(NS, d, "float64")
    a = lbm.make_solver(p, backend=backend, launch="fused")
    b = lbm.make_solver(p, backend=backend, launch="split")
    for s in (a, b):
        s.initialize(*cases.random_state(p))
        s.run(12)
    np.testing.assert_array_equal(a.populations(), b.populations())


@pytest.mark.parametrize("case,dtype,collision", [
    ("ibm2", "float64", "trt"), ("ibm2", "float32", "trt"), ("ibm2", "float16", "trt"), ("ibm3", "float32", "trt"),
    ("ibm3", "bfloat16", "trt"), ("ibm2", "float32", "regularized"), ("cylinder", "float32", "trt"),
    ("cylinder", "float64", "trt")])
def test_immersed_body_step_in_one_launch_gives_the_boundary_launchs_bits(case, dtype, collision):
    """A pull step with an immersed body updates the body's stencil nodes in the launch that
    forms their force (lbm_step_pull_ibm), beside a boundary launch over the other special nodes
    (the cylinder's Zou-He inlet and outlet, in the dense rule form) and the bulk; the fused
    launch mode keeps the force followed by one boundary list. Same bits, over steps that feed
    each step's force back into the populations (16-bit storage: same stochastic rounding)."""
    import dataclasses

    if case == "cylinder":
        p = cases.cylinder_channel(NS, "ibm", nx=160, ny=60, dtype=dtype, center=(50.0, 30.0), radius=8.0)[0]
        state = cases.random_state(p, seed=3, u_scale=0.03)
    else:
        p = cases.ibm(NS, 2 if case == "ibm2" else 3, dtype)
        state = cases.random_state(p)
    p = dataclasses.replace(p, collision=collision)
    split = lbm.make_solver(p, backend="cuda-naive")
    fused = lbm.make_solver(p, backend="cuda-naive", launch="fused")
    assert split._ibm_split is not None and fused._ibm_split is not None
    rest, body = split._ibm_split
    assert body.n_special == split._ibm.tables.n_nodes
    assert rest.n_special == split._special.n_special - body.n_special
    if case == "cylinder":
        assert rest.n_special > 0 and "ut_start" in rest.tensors
    for s in (split, fused):
        s.initialize(*state)
        s.run(14)
    np.testing.assert_array_equal(split.populations(), fused.populations())
    np.testing.assert_array_equal(split.immersed_force, fused.immersed_force)


@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("block", [(32, 4), (64, 4), (128, 2), (32, 8), (256, 1)])
def test_block_shapes_give_identical_bits(backend, block):
    p = cases.mixed(NS, "float32", "trt", 3)
    a = lbm.make_solver(p, backend=backend)
    b = lbm.make_solver(p, backend=backend, block=block)
    for s in (a, b):
        s.initialize(*cases.random_state(p))
        s.run(6)
    np.testing.assert_array_equal(a.populations(), b.populations())
