"""Hand-written adjoint against the FP64 NumPy adjoint and finite differences (GPU).

The loss is the momentum-exchange drag on a Bouzidi body averaged over the
last steps of a run from rest; the parameters are the Zou-He inlet-speed
scale U and a per-node Guo force field G. The NumPy adjoint
(``oracle/adjoint.py``) differentiates the oracle by complex steps and an
explicit transposed-streaming scatter, independently of the CUDA kernels.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.adjoint import OracleAdjoint

import lbm_b200 as lbm
from lbm_b200.adjoint import AdjointRun, aligned_rules, drag_loss

pytestmark = pytest.mark.gpu


def channel_2d(dtype="float64"):
    lat = lbm.D2Q9
    nx, ny = 24, 14
    solid = lbm.channel_walls(nx, ny)
    body = lbm.circle(9.3, 6.6, 2.7)
    solid |= lbm.voxelize(body, solid.shape)
    inflow = np.zeros((2, ny))
    inflow[0, 1:-1] = 0.04

    def make(scale):
        s2, rules, d_rules = lbm.zou_he_inlet_derivative(lat, solid, scale * inflow)
        links = lbm.wall_links(lat, body, s2)
        all_rules, all_d = aligned_rules(rules, d_rules, lbm.bouzidi_rules(lat, links, s2))
        p = lbm.SimulationParams(nx=nx, ny=ny, tau=0.6, collision="trt", solid=s2, dtype=dtype, link_rules=all_rules)
        return p, all_d

    p, _ = make(1.0)
    links = lbm.wall_links(lat, body, p.solid)
    return make, links, p


def channel_3d(dtype="float64"):
    lat = lbm.D3Q19
    nx, ny, nz = 20, 12, 11
    solid = lbm.duct_walls(nx, ny, nz)
    body = lbm.sphere(7.2, 5.6, 5.3, 2.3)
    solid |= lbm.voxelize(body, solid.shape)
    inflow = np.zeros((3, nz, ny))
    inflow[0, 1:-1, 1:-1] = 0.04

    def make(scale):
        s2, rules, d_rules = lbm.zou_he_inlet_derivative(lat, solid, scale * inflow)
        links = lbm.wall_links(lat, body, s2)
        all_rules, all_d = aligned_rules(rules, d_rules, lbm.bouzidi_rules(lat, links, s2))
        p = lbm.SimulationParams(nx=nx, ny=ny, nz=nz, tau=0.6, collision="trt", solid=s2, dtype=dtype,
                                 link_rules=all_rules)
        return p, all_d

    p, _ = make(1.0)
    links = lbm.wall_links(lat, body, p.solid)
    return make, links, p


def oracle_gradients(make, links, G, steps, window):
    p, d_rules = make(1.0)
    probe = lbm.ForceProbe.build(p, links)
    comp = probe.compiled("reference")
    adj = OracleAdjoint(p, (comp.slots, comp.coeff, comp.constant), probe.weight, 0, window, G, d_rules)
    loss = adj.forward(steps)
    dU, dG = adj.backward()
    return loss, dU, dG


@pytest.mark.parametrize("case", [channel_2d, channel_3d], ids=["2d", "3d"])
def test_adjoint_matches_the_numpy_adjoint_in_float64(case):
    make, links, p = case("float64")
    rng = np.random.default_rng(0)
    G = 1e-5 * rng.standard_normal((p.d, *p.shape)) * p.fluid
    steps, window = 30, 12
    loss_ref, dU_ref, dG_ref = oracle_gradients(make, links, G, steps, window)
    run = AdjointRun(make, links, steps=steps, window=window, checkpoint=7)
    loss = run.forward(1.0, G)
    dU, dG = run.backward()
    assert loss == pytest.approx(loss_ref, rel=1e-12)
    assert dU == pytest.approx(dU_ref, rel=1e-10)
    fluid = p.fluid
    np.testing.assert_allclose(dG[:, fluid], dG_ref[:, fluid], rtol=0, atol=1e-10 * np.abs(dG_ref).max())


def test_adjoint_matches_central_finite_differences():
    """Central differences with h = 1e-4 relative, float64 runs (agreement <= 1e-4)."""
    make, links, p = channel_2d("float64")
    rng = np.random.default_rng(1)
    G = 1e-5 * rng.standard_normal((p.d, *p.shape)) * p.fluid
    steps, window = 40, 15
    run = AdjointRun(make, links, steps=steps, window=window, checkpoint=10)
    run.forward(1.0, G)
    dU, dG = run.backward()
    h = 1e-4
    fd_U = (run.forward(1.0 + h, G) - run.forward(1.0 - h, G)) / (2 * h)
    assert abs(dU - fd_U) <= 1e-4 * abs(fd_U)
    v = rng.standard_normal(G.shape) * p.fluid
    eps = 1e-4 * np.abs(G).max()
    fd_G = (run.forward(1.0, G + eps * v) - run.forward(1.0, G - eps * v)) / (2 * eps)
    assert abs((dG * v).sum() - fd_G) <= 1e-4 * abs(fd_G)


def test_checkpoint_interval_does_not_change_the_gradient():
    make, links, p = channel_2d("float64")
    G = np.zeros((p.d, *p.shape))
    out = []
    for k in (1, 8, 1000):
        run = AdjointRun(make, links, steps=24, window=10, checkpoint=k)
        run.forward(1.0, G)
        out.append(run.backward())
    for dU, dG in out[1:]:
        assert dU == out[0][0]
        np.testing.assert_array_equal(dG, out[0][1])


def test_float32_adjoint_is_close_to_the_float64_adjoint():
    make64, links, p = channel_2d("float64")
    make32, _, _ = channel_2d("float32")
    rng = np.random.default_rng(2)
    G = 1e-5 * rng.standard_normal((p.d, *p.shape)) * p.fluid
    a = AdjointRun(make64, links, steps=40, window=15)
    b = AdjointRun(make32, links, steps=40, window=15)
    a.forward(1.0, G)
    b.forward(1.0, G)
    dU64, dG64 = a.backward()
    dU32, dG32 = b.backward()
    assert dU32 == pytest.approx(dU64, rel=1e-4)
    assert np.abs(dG32 - dG64).max() <= 1e-4 * np.abs(dG64).max()


def test_torch_autograd_function():
    import torch

    make, links, p = channel_2d("float64")
    run = AdjointRun(make, links, steps=20, window=8)
    U = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    G = torch.zeros((p.d, *p.shape), dtype=torch.float64, requires_grad=True)
    loss = drag_loss(U, G, run)
    loss.backward()
    dU, dG = run.backward()
    assert U.grad.item() == pytest.approx(dU, rel=1e-14)
    np.testing.assert_allclose(G.grad.numpy(), dG, rtol=1e-14)


# ---------------------------------------------------------------- immersed bodies


def ibm_channel(d, dtype="float64", with_bouzidi=False):
    """Zou-He channel with an immersed body (3 multi-direct passes); optionally also a Bouzidi body."""
    if d == 2:
        lat, (nx, ny) = lbm.D2Q9, (20, 12)
        solid = lbm.channel_walls(nx, ny)
        inflow = np.zeros((2, ny))
        inflow[0, 1:-1] = 0.04
        ball = lbm.circle(7.3, 5.6, 2.1)
        wall_body = lbm.circle(15.2, 6.1, 1.8)
        sizes = {"nx": nx, "ny": ny}
    else:
        lat, (nx, ny, nz) = lbm.D3Q19, (16, 11, 11)
        solid = lbm.duct_walls(nx, ny, nz)
        inflow = np.zeros((3, nz, ny))
        inflow[0, 1:-1, 1:-1] = 0.04
        ball = lbm.sphere(6.4, 5.3, 5.1, 1.7)
        wall_body = lbm.sphere(11.6, 5.2, 5.4, 1.6)
        sizes = {"nx": nx, "ny": ny, "nz": nz}
    if with_bouzidi:
        solid = solid | lbm.voxelize(wall_body, solid.shape)
    body = lbm.ImmersedBoundary.from_ball(ball, spacing=1.0, iterations=3)

    def make(scale):
        s2, rules, d_rules = lbm.zou_he_inlet_derivative(lat, solid, scale * inflow)
        all_rules, all_d = rules, d_rules
        if with_bouzidi:
            links = lbm.wall_links(lat, wall_body, s2)
            all_rules, all_d = aligned_rules(rules, d_rules, lbm.bouzidi_rules(lat, links, s2))
        p = lbm.SimulationParams(**sizes, tau=0.6, collision="trt", solid=s2, dtype=dtype, link_rules=all_rules,
                                 immersed=body)
        return p, all_d

    p, _ = make(1.0)
    links = lbm.wall_links(lat, wall_body, p.solid) if with_bouzidi else None
    return make, links, p


def oracle_ibm_gradients(make, links, G, steps, window):
    p, d_rules = make(1.0)
    if links is None:
        adj = OracleAdjoint(p, None, None, 0, window, G, d_rules)
    else:
        probe = lbm.ForceProbe.build(p, links)
        comp = probe.compiled("reference")
        adj = OracleAdjoint(p, (comp.slots, comp.coeff, comp.constant), probe.weight, 0, window, G, d_rules)
    loss = adj.forward(steps)
    dU, dG = adj.backward()
    return loss, dU, dG


@pytest.mark.parametrize("d,with_bouzidi", [(2, False), (3, False), (2, True)],
                         ids=["2d-body-force", "3d-body-force", "2d-probe-with-immersed-body"])
def test_immersed_body_adjoint_matches_the_numpy_adjoint(d, with_bouzidi):
    """Loss: the immersed body's drag (or a Bouzidi body's probe drag with the immersed body in the flow)."""
    make, links, p = ibm_channel(d, "float64", with_bouzidi)
    rng = np.random.default_rng(4)
    G = 1e-5 * rng.standard_normal((p.d, *p.shape)) * p.fluid
    steps, window = 16, 6
    loss_ref, dU_ref, dG_ref = oracle_ibm_gradients(make, links, G, steps, window)
    run = AdjointRun(make, links, steps=steps, window=window, checkpoint=5)
    loss = run.forward(1.0, G)
    dU, dG = run.backward()
    assert loss == pytest.approx(loss_ref, rel=1e-12)
    assert dU == pytest.approx(dU_ref, rel=1e-10)
    fluid = p.fluid
    np.testing.assert_allclose(dG[:, fluid], dG_ref[:, fluid], rtol=0, atol=1e-10 * np.abs(dG_ref).max())


def test_immersed_body_adjoint_matches_central_finite_differences():
    """float64 GPU runs, h = 1e-4 relative; agreement <= 1e-6 (the target is 1e-4)."""
    make, links, p = ibm_channel(2, "float64")
    rng = np.random.default_rng(5)
    G = 1e-5 * rng.standard_normal((p.d, *p.shape)) * p.fluid
    steps, window = 60, 20
    run = AdjointRun(make, links, steps=steps, window=window, checkpoint=16)
    run.forward(1.0, G)
    dU, dG = run.backward()
    h = 1e-4
    fd_U = (run.forward(1.0 + h, G) - run.forward(1.0 - h, G)) / (2 * h)
    assert abs(dU - fd_U) <= 1e-6 * abs(fd_U)
    v = rng.standard_normal(G.shape) * p.fluid
    eps = 1e-4 * np.abs(G).max()
    fd_G = (run.forward(1.0, G + eps * v) - run.forward(1.0, G - eps * v)) / (2 * eps)
    assert abs((dG * v).sum() - fd_G) <= 1e-6 * abs(fd_G)


def test_float32_immersed_body_adjoint_is_close_to_float64():
    make64, links, p = ibm_channel(3, "float64")
    make32, _, _ = ibm_channel(3, "float32")
    rng = np.random.default_rng(6)
    G = 1e-5 * rng.standard_normal((p.d, *p.shape)) * p.fluid
    out = []
    for make in (make64, make32):
        run = AdjointRun(make, links, steps=40, window=15, checkpoint=10)
        run.forward(1.0, G)
        out.append(run.backward())
    (dU64, dG64), (dU32, dG32) = out
    assert dU32 == pytest.approx(dU64, rel=1e-4)
    assert np.abs(dG32 - dG64).max() <= 1e-4 * np.abs(dG64).max()


def test_immersed_body_loss_needs_an_immersed_body():
    make, links, p = channel_2d("float64")
    run = AdjointRun(make, None, steps=4, window=2)
    with pytest.raises(ValueError, match="immersed"):
        run.forward(1.0, None)


def test_dense_and_term_by_term_rules_give_the_same_gradient():
    """The adjoint evaluates rules and their U-derivatives in the dense per-node form when the
    forward solver has it; the term-by-term form must agree to round-off."""
    make, links, p = channel_3d("float64")
    rng = np.random.default_rng(7)
    G = 1e-5 * rng.standard_normal((p.d, *p.shape)) * p.fluid
    out = []
    for dense in (True, False):
        run = AdjointRun(make, links, steps=20, window=8, checkpoint=6, dense_rules=dense)
        loss = run.forward(1.0, G)
        out.append((loss, *run.backward()))
    (l1, u1, g1), (l2, u2, g2) = out
    assert l1 == pytest.approx(l2, rel=1e-13)
    assert u1 == pytest.approx(u2, rel=1e-12)
    assert np.abs(g1 - g2).max() <= 1e-12 * np.abs(g2).max()
