"""The FP64 NumPy adjoint with an immersed body, against central differences of the oracle (CPU).

The loss is the immersed body's drag (its body-force x component) averaged
over the last steps of a run from rest, in a channel with a Zou-He inlet; the
parameters are the inlet-speed scale U and a per-node Guo force field G. The
immersed-boundary force couples the stencil nodes' streamed populations into
their collision; the NumPy adjoint takes that term by complex steps through
the oracle's multi-direct passes. Both derivatives are checked against
central differences of the oracle's own forward runs (float64, h = 1e-4
relative).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.adjoint import OracleAdjoint

import lbm_b200 as lbm


def ibm_channel(scale, dtype="float64"):
    lat = lbm.D2Q9
    nx, ny = 18, 11
    solid = lbm.channel_walls(nx, ny)
    inflow = np.zeros((2, ny))
    inflow[0, 1:-1] = 0.04
    s2, rules, d_rules = lbm.zou_he_inlet_derivative(lat, solid, scale * inflow)
    body = lbm.ImmersedBoundary.from_ball(lbm.circle(7.3, 5.1, 2.1), spacing=1.0, iterations=3)
    p = lbm.SimulationParams(nx=nx, ny=ny, tau=0.6, collision="trt", solid=s2, dtype=dtype, link_rules=rules,
                             immersed=body)
    return p, d_rules


def drag(scale, G, steps, window):
    p, d_rules = ibm_channel(scale)
    adj = OracleAdjoint(p, None, None, 0, window, G, d_rules)
    return adj, adj.forward(steps)


def test_immersed_body_adjoint_matches_central_differences():
    p, _ = ibm_channel(1.0)
    rng = np.random.default_rng(3)
    G = 1e-5 * rng.standard_normal((p.d, *p.shape)) * p.fluid
    steps, window = 14, 6
    adj, loss = drag(1.0, G, steps, window)
    assert loss != 0.0
    dU, dG = adj.backward()
    h = 1e-4
    fd_U = (drag(1.0 + h, G, steps, window)[1] - drag(1.0 - h, G, steps, window)[1]) / (2 * h)
    assert dU == pytest.approx(fd_U, rel=1e-8)
    v = rng.standard_normal(G.shape) * p.fluid
    eps = h * np.abs(G).max()
    fd_G = (drag(1.0, G + eps * v, steps, window)[1] - drag(1.0, G - eps * v, steps, window)[1]) / (2 * eps)
    assert float((dG * v).sum()) == pytest.approx(fd_G, rel=1e-8)
    # the gradient reaches the stencil nodes' force field
    ibm = adj.solver.ibm
    assert np.abs(dG.reshape(p.d, -1)[:, ibm.nodes]).max() > 0.0


def test_loss_without_probe_needs_an_immersed_body():
    p, _ = ibm_channel(1.0)
    plain = lbm.SimulationParams(nx=p.nx, ny=p.ny, tau=0.6, collision="trt", solid=p.solid, dtype="float64")
    with pytest.raises(ValueError, match="immersed"):
        OracleAdjoint(plain, None, None, 0, 3, np.zeros((2, *p.shape)))
