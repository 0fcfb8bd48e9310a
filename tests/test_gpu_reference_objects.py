"""The drop-in, exercised with the reference's own objects (GPU).

The reference package, unmodified, in ``baseline/_ref`` (``oracle/reference_package.py``)
builds every input: ``SimulationParams``, the wall and body builders,
``bouzidi_rules``, ``open_channel``, ``ImmersedBoundary``, ``ForceProbe``. Its
``make_solver`` (``src/lbm/backends/__init__.py:62-83``) gets the registration
that the integration notes show -- backends ``cuda-b200`` and ``cuda-b200-aa``
returning ``lbm_b200.CudaSolver`` -- applied to the imported module for the
test only (``monkeypatch``; no file of the reference is touched). Each case
then runs on the reference's NumPy ``ReferenceSolver`` and on this package's
CUDA solver through that one entry point, and the reference's own readouts
(populations, ``macroscopic``, ``ForceProbe.evaluate``, ``immersed_force``)
are compared at the parity bounds. The last test runs the reference's own
Schaefer-Turek 2D-2 driver (``cases/cylinder_benchmark.py:231-255``) on the
CUDA solver and asserts the reference's own validation intervals.

Skipped where ``baseline/_ref`` is not installed.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import reference_package
from tests import cases
from tests.helpers import reference_ns

import lbm_b200

REF = reference_package.modules()

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(REF is None, reason="baseline/_ref (the reference package) is absent")]

ABS = {"float64": 1e-15, "float32": 1e-7}
REL = {"float64": 1e-14, "float32": 2e-6}
"""Against the reference's own float32 NumPy arithmetic (not the oracle's), whose summation order
differs from the kernels' fused multiply-adds: a Zou-He rule sums ~20 float32 terms, and 40 steps
of such differences reach ~1e-6 of max|f~| (measured 1.1e-6, 13 float32 ulps of max|f~|, on the 3D
open channel); the absolute bound is the reference's own."""
OURS = {"cuda-naive": "cuda-b200", "cuda-aa": "cuda-b200-aa"}


@pytest.fixture
def make_solver(monkeypatch):
    """The reference's make_solver with this package registered, as a maintainer would add it."""
    backends = REF.backends
    original = backends.make_solver

    def patched(params, backend="numpy", **options):
        if backend in ("cuda-b200", "cuda-b200-aa"):
            variant = "aa" if backend.endswith("-aa") else "pull"
            return lbm_b200.CudaSolver(params, variant=variant, **options)
        return original(params, backend, **options)

    monkeypatch.setattr(backends, "BACKENDS", (*backends.BACKENDS, "cuda-b200", "cuda-b200-aa"))
    monkeypatch.setattr(backends, "make_solver", patched)
    import lbm.cases.cylinder_benchmark as cyl  # noqa: PLC0415  (imported make_solver by name)

    monkeypatch.setattr(cyl, "make_solver", patched)
    return patched


def build(name, d, dtype):
    ns = reference_ns()
    links = None
    if name == "mixed":
        p = cases.mixed(ns, dtype, "trt", d)
    elif name == "bouzidi":
        p, links = cases.bouzidi(ns, d, dtype)
    elif name == "ibm":
        p = cases.ibm(ns, d, dtype)
    else:
        p, _ = cases.open_channel_case(ns, d, dtype=dtype)
    assert type(p).__module__.startswith("lbm."), "the inputs must be the reference's objects"
    return p, links


def assert_close(a, b, dtype):
    diff = np.abs(a - b).max()
    assert diff < ABS[dtype], diff
    assert diff <= REL[dtype] * np.abs(a).max(), diff


@pytest.mark.parametrize("backend", ["cuda-naive", "cuda-aa"])
@pytest.mark.parametrize("name", ["mixed", "bouzidi", "ibm", "open"])
@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_reference_inputs_run_on_the_cuda_backend_like_the_reference_solver(make_solver, backend, name, d, dtype):
    p, links = build(name, d, dtype)
    state = cases.random_state(p)
    ref = make_solver(p, backend="numpy")
    gpu = make_solver(p, backend=OURS[backend])
    assert isinstance(gpu, lbm_b200.CudaSolver)
    for s in (ref, gpu):
        s.initialize(*state)
        s.run(cases.EQUIVALENCE_STEPS)
    fluid = np.asarray(p.fluid)
    assert_close(ref.populations()[:, fluid], gpu.populations()[:, fluid], dtype)
    mr, mg = ref.macroscopic(), gpu.macroscopic()
    tol = 1e-13 if dtype == "float64" else 1e-5
    np.testing.assert_allclose(mg.rho, mr.rho, rtol=0, atol=tol)
    for a in range(d):
        np.testing.assert_allclose(mg.u[a], mr.u[a], rtol=0, atol=tol)
    if links is not None:  # the reference's ForceProbe, evaluated on both solvers
        probe = REF.forces.ForceProbe.build(p, links)
        want, got = probe.evaluate(ref), probe.evaluate(gpu)
        np.testing.assert_allclose(got, want, rtol=1e-10 if dtype == "float64" else 1e-4,
                                   atol=1e-14 if dtype == "float64" else 1e-8)
    if name == "ibm":
        np.testing.assert_allclose(gpu.immersed_force, ref.immersed_force,
                                   rtol=1e-10 if dtype == "float64" else 1e-4, atol=1e-14 if dtype == "float64" else 1e-8)


def test_reference_schaefer_turek_2d2_driver_on_the_cuda_backend(make_solver):
    """The reference's own 2D-2 driver and observer (inflow-profile start, C_D/C_L by its
    ForceProbe, St from lift zero crossings) on ``cuda-b200-aa``, N = 20, float32: the
    intervals of the reference's validation test (``tests/validation/test_cylinder_benchmark.py:28-32``)."""
    from lbm.cases.cylinder_benchmark import run_periodic  # noqa: PLC0415

    r = run_periodic(20, backend="cuda-b200-aa")
    assert 0.295 < r.strouhal < 0.305, r.strouhal
    assert r.cl_max == pytest.approx(1.0, rel=0.08)
    assert r.cd_max == pytest.approx(3.23, rel=0.03)
