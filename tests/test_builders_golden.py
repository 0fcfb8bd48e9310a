"""Host-side input builders against the reference's outputs (CPU only).

Bouzidi rules, Zou-He rules, wall links, immersed-boundary markers/stencils
and force-probe slots of every memory layout must equal what the reference
package produced for the same geometry (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import numpy as np
import pytest

from tests import cases
from tests.helpers import NS, assert_rules_match, golden

import lbm_b200 as lbm
from oracle import reference_package


@pytest.mark.parametrize("d", [2, 3])
def test_bouzidi_rules_links_and_probe_layouts(d):
    ref = golden(f"bouzidi{d}d_float64")
    body = None if d == 2 else lbm.sphere(7.3, 6.6, 5.8, 3.1)
    p, links = cases.bouzidi(NS, d, "float64", None if d == 2 else (16, 14, 12), body)
    np.testing.assert_array_equal(links.node, ref["link_node"])
    np.testing.assert_array_equal(links.direction, ref["link_dir"])
    np.testing.assert_allclose(links.q, ref["link_q"], rtol=0, atol=1e-15)
    assert_rules_match(p.link_rules, ref, "rule_")
    probe = lbm.ForceProbe.build(p, links)
    np.testing.assert_array_equal(probe.weight, ref["probe_weight"])
    for layout in ("pull", "aa_odd", "aa_even"):
        comp = probe.compiled(layout)
        np.testing.assert_array_equal(comp.slots, ref[f"{layout}_slots"])
        np.testing.assert_allclose(comp.coeff, ref[f"{layout}_coeff"], rtol=0, atol=1e-15)
        np.testing.assert_allclose(comp.constant, ref[f"{layout}_const"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("d", [2, 3])
def test_zou_he_rules(d):
    ref = golden(f"zouhe{d}d_float64")
    p, _ = cases.open_channel_case(NS, d)
    np.testing.assert_array_equal(p.solid, ref["solid"])
    assert_rules_match(p.link_rules, ref, "rule_")


def test_cylinder_channel_rules():
    ref = golden("cylinder_bouzidi_rules")
    p, links, _ = cases.cylinder_channel(NS, "bouzidi")
    np.testing.assert_array_equal(p.solid, ref["solid"])
    np.testing.assert_array_equal(links.node, ref["link_node"])
    np.testing.assert_allclose(links.q, ref["link_q"], rtol=0, atol=1e-15)
    assert_rules_match(p.link_rules, ref, "rule_")


def test_cylinder_ibm_markers_and_open_rules():
    ref = golden("cylinder_ibm_markers")
    p, _, _ = cases.cylinder_channel(NS, "ibm")
    np.testing.assert_allclose(p.immersed.markers, ref["markers"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(p.immersed.areas, ref["areas"], rtol=1e-15)
    nodes, weights = p.immersed.stencil(p.shape)
    np.testing.assert_array_equal(nodes, ref["stencil_nodes"])
    np.testing.assert_allclose(weights, ref["stencil_weights"], rtol=0, atol=1e-15)
    assert_rules_match(p.link_rules, ref, "rule_")


def test_sphere_channel_rules():
    ref = golden("sphere_channel_small_rules")
    p, links, _ = cases.sphere_channel(NS, nx=40, ny=20, nz=18, radius=4.0)
    np.testing.assert_array_equal(p.solid, ref["solid"])
    np.testing.assert_array_equal(links.node, ref["link_node"])
    assert_rules_match(p.link_rules, ref, "rule_")


@pytest.mark.parametrize("d", [2, 3])
def test_ibm_markers_and_stencils(d):
    ref = golden(f"ibm{d}d_float64")
    body = None if d == 2 else lbm.sphere(6.7, 6.6, 5.9, 2.6)
    p = cases.ibm(NS, d, "float64", None if d == 2 else (14, 14, 12), body)
    np.testing.assert_allclose(p.immersed.markers, ref["markers"], rtol=0, atol=1e-13)
    nodes, weights = p.immersed.stencil(p.shape)
    np.testing.assert_array_equal(nodes, ref["stencil_nodes"])
    np.testing.assert_allclose(weights, ref["stencil_weights"], rtol=0, atol=1e-15)


def test_ibm_inverse_map_covers_every_stencil_entry():
    p = cases.ibm(NS, 2, "float64")
    t = lbm.ibm.build_tables(p.immersed, p.lattice, p.solid)
    pairs = set()
    for n in range(t.n_nodes):
        for k in range(t.inv_start[n], t.inv_start[n + 1]):
            pairs.add((int(t.inv_marker[k]), n))
    expected = {(m, int(t.stencil[m, s])) for m in range(t.n_markers) for s in range(t.stencil.shape[1])}
    assert pairs == expected
    assert t.inv_start[-1] == t.stencil.size


def test_zou_he_inlet_derivative_matches_finite_differences():
    lattice = lbm.D2Q9
    solid = lbm.channel_walls(12, 9)
    inflow = np.zeros((2, 9))
    inflow[0, 1:-1] = 0.04
    _, rules, d_rules = lbm.zou_he_inlet_derivative(lattice, solid, inflow)
    h = 1e-6
    _, plus = lbm.open_channel(lattice, solid, (1 + h) * inflow)
    _, minus = lbm.open_channel(lattice, solid, (1 - h) * inflow)
    base = {k: v for k, v in zip(zip(rules.node, rules.direction), range(len(rules)), strict=True)}

    def dense(r, idx):
        v = r.values
        out = {(int(k), int(y)): float(a) for k, y, a in zip(v.direction[idx], v.node[idx], v.coeff[idx], strict=True) if a != 0}
        return out, float(v.constant[idx])

    for key, idx in base.items():
        ip = int(np.flatnonzero((plus.node == key[0]) & (plus.direction == key[1]))[0])
        im = int(np.flatnonzero((minus.node == key[0]) & (minus.direction == key[1]))[0])
        tp, cp = dense(plus, ip)
        tm, cm = dense(minus, im)
        dt, dc = dense(d_rules, idx)
        assert abs((cp - cm) / (2 * h) - dc) < 1e-7
        for k in set(tp) | set(tm) | set(dt):
            assert abs((tp.get(k, 0.0) - tm.get(k, 0.0)) / (2 * h) - dt.get(k, 0.0)) < 1e-7


def test_params_validation_messages_match_the_reference():
    with pytest.raises(ValueError, match="must be positive"):
        lbm.SimulationParams(nx=0, ny=4, tau=0.8)
    with pytest.raises(ValueError, match="tau must be > 0.5"):
        lbm.SimulationParams(nx=4, ny=4, tau=0.5)
    with pytest.raises(ValueError, match="collision"):
        lbm.SimulationParams(nx=4, ny=4, tau=0.8, collision="mrt")
    with pytest.raises(ValueError, match="dtype"):
        lbm.SimulationParams(nx=4, ny=4, tau=0.8, dtype="int8")
    with pytest.raises(ValueError, match="force must have 3 components"):
        lbm.SimulationParams(nx=4, ny=4, nz=4, tau=0.8, force=(1e-5, 0.0))
    with pytest.raises(ValueError, match="lattice D3Q19 is 3D"):
        lbm.SimulationParams(nx=4, ny=4, tau=0.8, lattice="D3Q19")
    with pytest.warns(lbm.StabilityWarning):
        lbm.SimulationParams(nx=4, ny=4, tau=0.505)
    p = lbm.SimulationParams(nx=4, ny=4, tau=0.8, collision="trt")
    wp, wm = p.relaxation_rates
    assert wp == 1.25 and abs((1 / wp - 0.5) * (1 / wm - 0.5) - 3 / 16) < 1e-15
    assert lbm.SimulationParams(nx=4, ny=4, tau=0.8, dtype="float16").dtype == "float16"


def test_rules_validation():
    body, solid = lbm.circle(15.3, 10.4, 4.6), lbm.channel_walls(33, 21)
    solid = solid | lbm.voxelize(body, solid.shape)
    links = lbm.wall_links(lbm.D2Q9, body, solid)
    rules = lbm.bouzidi_rules(lbm.D2Q9, links, solid)
    with pytest.raises(ValueError, match="solid"):
        lbm.SimulationParams(nx=33, ny=21, tau=0.7, link_rules=rules)
    moving = np.zeros((2, 21, 33))
    moving[0] = 0.01
    with pytest.raises(ValueError, match="at rest"):
        lbm.SimulationParams(nx=33, ny=21, tau=0.7, solid=solid, wall_velocity=moving, link_rules=rules)
    with pytest.raises(ValueError, match="more than one"):
        lbm.LinkRules(np.array([5, 5]), np.array([3, 3]), lbm.AffineSet.from_lists([[(1, 0, 1.0)], [(1, 0, 1.0)]]))


def _compiled_map(target, slots, coeff, const):
    """{target slot: (constant, {term slot: coefficient})}, zero terms dropped, any rule order."""
    out = {}
    for t, s, c, k in zip(target, slots, coeff, const, strict=True):
        terms = {}
        for slot, a in zip(s, c, strict=True):
            if a != 0.0:
                terms[int(slot)] = terms.get(int(slot), 0.0) + float(a)
        out[int(t)] = (float(k), terms)
    return out


@pytest.mark.parametrize("layout", ["pull", "aa_odd", "aa_even"])
@pytest.mark.parametrize("case", ["bouzidi", "zouhe"])
@pytest.mark.parametrize("d", [2, 3])
def test_rules_compile_to_the_reference_prepass_slots(d, case, layout):
    """compile_rules (the pre-pass form that the GPU checker feeds to the reference's own
    rule kernels) gives the reference's targets, term slots, coefficients and constants."""
    from lbm_b200.link_rules import compile_rules

    ref = golden("compiled_rules")
    key = f"{case}{d}d_{layout}_"
    p, _ = cases.bouzidi(NS, d, "float64") if case == "bouzidi" else cases.open_channel_case(NS, d)
    c = compile_rules(p.lattice, p.link_rules, layout, p.solid, p.wall_velocity)
    ours = _compiled_map(c.target, c.values.slots, c.values.coeff, c.values.constant)
    theirs = _compiled_map(ref[key + "target"], ref[key + "slots"], ref[key + "coeff"], ref[key + "const"])
    assert ours.keys() == theirs.keys()
    for t, (k, terms) in theirs.items():
        k2, terms2 = ours[t]
        assert abs(k - k2) <= 1e-15, (t, k, k2)
        assert terms.keys() == terms2.keys(), t
        for slot, a in terms.items():
            assert abs(a - terms2[slot]) <= 1e-15, (t, slot)


@pytest.mark.skipif(not reference_package.available(), reason="baseline/_ref is absent")
@pytest.mark.parametrize("case", ["bouzidi2", "bouzidi3", "plain_moving", "cylinder"])
def test_force_probe_rows_equal_the_reference_builders(case):
    """ForceProbe.build (vectorised) gives the reference's rows term for term, for links with
    rules, links with plain bounce-back next to a moving wall, and the cylinder configuration."""
    from tests.helpers import reference_ns

    ref_ns = reference_ns()
    from lbm.forces import ForceProbe as RefProbe  # noqa: PLC0415

    def build(ns):
        if case.startswith("bouzidi"):
            return cases.bouzidi(ns, int(case[-1]), "float64")
        if case == "cylinder":
            p, links, _ = cases.cylinder_channel(ns, "bouzidi", dtype="float64")
            return p, links
        # plain bounce-back links into a body next to a moving lid (no rules)
        solid, wall = ns.cavity_walls(20, 0.05)
        body = ns.circle(10.2, 17.9, 3.1)
        solid = solid | ns.voxelize(body, solid.shape)
        links = ns.wall_links(ns.default_lattice(2), body, solid)
        return ns.SimulationParams(nx=22, ny=22, tau=0.7, solid=solid, wall_velocity=wall), links

    p, links = build(NS)
    rp, rlinks = build(ref_ns)
    ours, theirs = lbm.ForceProbe.build(p, links), RefProbe.build(rp, rlinks)
    np.testing.assert_array_equal(ours.weight, theirs.weight)
    np.testing.assert_array_equal(ours.values.direction, theirs.values.direction)
    np.testing.assert_array_equal(ours.values.node, theirs.values.node)
    np.testing.assert_allclose(ours.values.coeff, theirs.values.coeff, rtol=0, atol=1e-15)
    np.testing.assert_allclose(ours.values.constant, theirs.values.constant, rtol=0, atol=1e-15)
