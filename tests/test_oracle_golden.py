"""The oracle against golden vectors of the unmodified reference (CPU only).

``tests/golden/make_golden.py`` ran the reference's NumPy solver on these
cases; the oracle must reproduce its populations, macroscopic fields,
immersed-body force, force probe and watchdog report. Inputs are rebuilt here
with this package's builders, which also pins those builders.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import OracleDiverged, OracleSolver
from tests import cases
from tests.helpers import NS, golden

import lbm_b200 as lbm

TOL = {"float64": 1e-16, "float32": 2e-8}


def check_outputs(solver, ref, d, dtype):
    tol = TOL[dtype]
    f = solver.populations()
    assert f.dtype == np.dtype(dtype)
    np.testing.assert_allclose(f, ref["f"], rtol=0, atol=tol)
    rho, u = solver.macroscopic()
    np.testing.assert_allclose(rho, ref["rho"], rtol=0, atol=10 * tol)
    for a in range(d):
        np.testing.assert_allclose(u[a], ref[f"u{a}"], rtol=0, atol=10 * tol)


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize(("dtype", "collision"), [("float64", "trt"), ("float64", "bgk"), ("float32", "trt")])
def test_mixed_geometry(d, dtype, collision):
    ref = golden(f"mixed{d}d_{dtype}_{collision}")
    p = cases.mixed(NS, dtype, collision, d, None if d == 2 else (15, 13, 11))
    s = OracleSolver(p)
    s.initialize(*cases.random_state(p))
    s.run(int(ref["steps"]))
    check_outputs(s, ref, d, dtype)


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_bouzidi_body_and_force_probe(d, dtype):
    ref = golden(f"bouzidi{d}d_{dtype}")
    body = None if d == 2 else lbm.sphere(7.3, 6.6, 5.8, 3.1)
    p, links = cases.bouzidi(NS, d, dtype, None if d == 2 else (16, 14, 12), body)
    s = OracleSolver(p)
    s.initialize(*cases.random_state(p))
    s.run(int(ref["steps"]))
    check_outputs(s, ref, d, dtype)
    probe = lbm.ForceProbe.build(p, links)
    force = probe.weight.T @ s.evaluate_affine(probe.compiled("reference"))
    np.testing.assert_allclose(force, ref["probe_force"], rtol=1e-12 if dtype == "float64" else 1e-5, atol=1e-16)


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_immersed_boundary(d, dtype):
    ref = golden(f"ibm{d}d_{dtype}")
    body = None if d == 2 else lbm.sphere(6.7, 6.6, 5.9, 2.6)
    p = cases.ibm(NS, d, dtype, None if d == 2 else (14, 14, 12), body)
    s = OracleSolver(p)
    s.initialize(*cases.random_state(p))
    s.run(int(ref["steps"]))
    check_outputs(s, ref, d, dtype)
    np.testing.assert_allclose(s.immersed_force, ref["immersed_force"], rtol=1e-13 if dtype == "float64" else 1e-6)


@pytest.mark.parametrize("d", [2, 3])
def test_zou_he_open_channel(d):
    ref = golden(f"zouhe{d}d_float64")
    p, _ = cases.open_channel_case(NS, d)
    s = OracleSolver(p)
    s.initialize(*cases.random_state(p, seed=1, u_scale=0.03))
    s.run(int(ref["steps"]))
    check_outputs(s, ref, d, "float64")


def test_taylor_green_64():
    ref = golden("tgv64_float32")
    p, state = cases.tgv(NS, n=64)
    s = OracleSolver(p)
    s.initialize(*state)
    s.run(int(ref["steps"]))
    check_outputs(s, ref, 2, "float32")


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_duct_18(dtype):
    ref = golden(f"duct18_{dtype}")
    p = cases.duct(NS, n=18, nx=4, dtype=dtype, force=1e-5)
    s = OracleSolver(p)
    s.run(int(ref["steps"]))
    check_outputs(s, ref, 3, dtype)


def test_cavity_30():
    ref = golden("cavity30_float64")
    p = cases.cavity(NS, 30, 400.0, dtype="float64")
    s = OracleSolver(p)
    s.run(int(ref["steps"]))
    check_outputs(s, ref, 2, "float64")


@pytest.mark.parametrize("d", [2, 3])
def test_watchdog_reports_step_and_location(d):
    ref = golden(f"watchdog{d}d")
    sizes = {"nx": 8, "ny": 8} | ({"nz": 8} if d == 3 else {})
    p = lbm.SimulationParams(**sizes, tau=0.8, dtype="float64")
    s = OracleSolver(p)
    rho = np.ones(p.shape)
    rho[(3, 5, 2)[:d]] = np.nan
    s.initialize(rho)
    with pytest.raises(OracleDiverged) as info:
        s.run(10, check_every=5)
    assert info.value.step == int(ref["step"])
    assert info.value.location == tuple(int(v) for v in ref["location"])
