"""Device-side rule compiler against the host builders and the reference's fixtures (GPU).

``lbm_b200.device_rules`` builds the ball voxelisation, the wall links with
their fractions and the Bouzidi rules on the device. They must equal the host
builders bit for bit (the kernels round every operation as NumPy does), and
so the reference's golden links and rules (``tests/golden``), which the host
builders are pinned to. The CUDA solver resolves force-probe terms to its own
buffers on the device (``lbm_compile_terms``); that must give the forces of the
host-compiled slots.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests import cases
from tests.helpers import NS, assert_rules_match, golden

import lbm_b200 as lbm
from lbm_b200 import device_rules as dev

pytestmark = pytest.mark.gpu


def host_and_device(lattice, body, solid):
    host_solid = solid | lbm.voxelize(body, solid.shape)
    host_links = lbm.wall_links(lattice, body, host_solid)
    host_rules = lbm.bouzidi_rules(lattice, host_links, host_solid)
    dev_solid, dev_links, dev_rules = dev.ball_channel(lattice, body, solid)
    return (host_solid, host_links, host_rules), (dev_solid, dev_links, dev_rules)


def assert_same(host, device):
    (hs, hl, hr), (ds, dl, dr) = host, device
    np.testing.assert_array_equal(ds, hs)
    np.testing.assert_array_equal(dl.node, hl.node)
    np.testing.assert_array_equal(dl.direction, hl.direction)
    np.testing.assert_array_equal(dl.q, hl.q)  # bit for bit
    np.testing.assert_array_equal(dr.node, hr.node)
    np.testing.assert_array_equal(dr.direction, hr.direction)
    for a, b in ((dr.values.direction, hr.values.direction), (dr.values.node, hr.values.node),
                 (dr.values.coeff, hr.values.coeff), (dr.values.constant, hr.values.constant)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("case", [
    ("D2Q9", (29, 45), (20.3, 13.6), 5.2),
    ("D2Q9", (164, 880), (200.0, 82.0), 20.0),
    ("D2Q9", (30, 31), (0.4, 15.2), 6.3),            # crosses the periodic x edge
    ("D3Q19", (16, 20, 24), (11.3, 9.6, 7.8), 4.1),
    ("D3Q19", (64, 64, 128), (32.0, 31.5, 31.5), 8.0),
    ("D3Q19", (40, 41, 43), (21.5, 20.0, 19.5), 12.25),
])
def test_device_builders_equal_the_host_builders_bit_for_bit(case):
    name, shape, centre, radius = case
    lattice = lbm.LATTICES[name]
    solid = lbm.channel_walls(shape[-1], shape[-2], shape[0] if len(shape) == 3 else None)
    body = lbm.Ball(centre, radius)
    host, device = host_and_device(lattice, body, solid)
    assert len(host[1]) > 0
    assert_same(host, device)


@pytest.mark.parametrize("d", [2, 3])
def test_device_links_and_rules_equal_the_reference_golden_fixtures(d):
    ref = golden(f"bouzidi{d}d_float64")
    body = None if d == 2 else lbm.sphere(7.3, 6.6, 5.8, 3.1)
    p, links = cases.bouzidi(NS, d, "float64", None if d == 2 else (16, 14, 12), body)
    body = body or lbm.circle(20.3, 13.6, 5.2)
    dl = dev.wall_links(p.lattice, body, p.solid)
    np.testing.assert_array_equal(dl.node, ref["link_node"])
    np.testing.assert_array_equal(dl.direction, ref["link_dir"])
    np.testing.assert_allclose(dl.q, ref["link_q"], rtol=0, atol=1e-15)
    rules = dev.bouzidi_rules(p.lattice, dl, p.solid)
    assert_rules_match(rules, ref, "rule_")


def test_a_fluid_node_inside_the_body_is_rejected():
    solid = lbm.channel_walls(40, 30)
    with pytest.raises(ValueError, match="must be marked solid"):
        dev.wall_links(lbm.D2Q9, lbm.circle(20.0, 15.0, 5.0), solid)


@pytest.mark.parametrize("backend", ["cuda-naive", "cuda-aa"])
@pytest.mark.parametrize("dtype", ["float64", "float16"])
def test_device_compiled_probe_equals_the_host_compiled_slots(backend, dtype):
    """probe.evaluate on the CUDA solver (terms resolved on the device) against the reduction of
    the host-compiled slots of the same state."""
    p, links = cases.bouzidi(NS, 3, dtype, size=(64, 20, 16), body=NS.sphere(31.7, 9.6, 7.7, 4.1))
    gpu = lbm.make_solver(p, backend=backend)
    gpu.initialize(*cases.random_state(p))
    gpu.run(6)
    probe = lbm.ForceProbe.build(p, links)
    via_device = probe.evaluate(gpu)
    via_host = gpu.reduce_affine(probe.compiled(gpu.state_layout), probe.weight)
    np.testing.assert_array_equal(via_device, via_host)
    np.testing.assert_allclose(via_host, probe.weight.T @ gpu.evaluate_affine(probe.compiled(gpu.state_layout)),
                               rtol=1e-12, atol=1e-18)


def assert_same_rules(device, host):
    np.testing.assert_array_equal(device.node, host.node)
    np.testing.assert_array_equal(device.direction, host.direction)
    for a, b in ((device.values.direction, host.values.direction), (device.values.node, host.values.node),
                 (device.values.coeff, host.values.coeff), (device.values.constant, host.values.constant)):
        assert a.shape == b.shape and a.dtype == b.dtype
        np.testing.assert_array_equal(a, b)  # bit for bit


def _open_cases():
    """(lattice, solid, inflow, rho_out): channels with walls, bodies at the open columns, a
    partly closed open layer, a fully periodic cross-section, the cylinder and sphere channels."""
    out = []
    for d in (2, 3):
        p, inflow = cases.open_channel_case(NS, d)
        nx, ny = 12, 9
        solid = lbm.channel_walls(nx, ny) if d == 2 else lbm.channel_walls(nx, ny, 5)
        out.append((f"small{d}d", p.lattice, solid, inflow, 1.003))
    rng = np.random.default_rng(5)
    solid = lbm.channel_walls(17, 13, 7)
    solid[2:4, 3:5, 1] = True       # a block on the inlet column
    solid[3, 6, 0] = True           # a closed node in the open inlet layer
    solid[1:3, 2:4, -2] = True      # a block on the outlet column
    inflow = rng.uniform(-0.02, 0.05, size=(3, 7, 13))
    out.append(("bodies3d", lbm.D3Q19, solid, inflow, 0.998))
    solid = np.zeros((11, 10), dtype=bool)  # periodic in y: no walls
    inflow = rng.uniform(0.0, 0.04, size=(2, 11))
    out.append(("periodic2d", lbm.D2Q9, solid, inflow, 1.0))
    solid = np.zeros((5, 6, 4), dtype=bool)  # the narrowest channel (nx = 4), periodic in y and z
    out.append(("narrow3d", lbm.D3Q19, solid, np.full((3, 5, 6), 0.03), 1.01))
    ny, nx = 164, 880
    y = np.arange(ny) - 0.5
    profile = np.where((y > 0) & (y < ny - 2), 4.0 * 0.05 * y * (ny - 2 - y) / (ny - 2) ** 2, 0.0)
    solid = np.zeros((ny, nx), dtype=bool)
    solid[0, :] = solid[-1, :] = True
    solid |= lbm.voxelize(lbm.circle(200.0, 82.0, 20.0), solid.shape)
    out.append(("cylinder", lbm.D2Q9, solid, np.stack([profile, np.zeros(ny)]), 1.0))
    solid = np.zeros((64, 64, 128), dtype=bool)
    solid[:, [0, -1], :] = True
    solid[[0, -1], :, :] = True
    inflow = np.zeros((3, 64, 64))
    inflow[0, 1:-1, 1:-1] = 0.04
    out.append(("sphere_channel", lbm.D3Q19, solid, inflow, 1.0))
    return out


@pytest.mark.parametrize("case", _open_cases(), ids=lambda c: c[0])
def test_device_open_channel_equals_the_host_builder_bit_for_bit(case):
    _, lattice, solid, inflow, rho_out = case
    hs, hr = lbm.open_channel(lattice, solid, inflow, rho_out=rho_out)
    ds, dr = dev.open_channel(lattice, solid, inflow, rho_out=rho_out)
    np.testing.assert_array_equal(ds, hs)
    assert len(hr) > 0
    assert_same_rules(dr, hr)


@pytest.mark.parametrize("d", [2, 3])
def test_device_open_channel_equals_the_reference_golden_rules(d):
    ref = golden(f"zouhe{d}d_float64")
    nx, ny, nz = 12, 9, 5
    solid = lbm.channel_walls(nx, ny) if d == 2 else lbm.channel_walls(nx, ny, nz)
    inflow = np.zeros((d, *solid.shape[:-1]))
    inflow[0], inflow[1] = 0.04, 0.01
    if d == 3:
        inflow[2] = -0.02
    ds, dr = dev.open_channel(lbm.LATTICES["D2Q9" if d == 2 else "D3Q19"], solid, inflow, rho_out=1.003)
    np.testing.assert_array_equal(ds, ref["solid"])
    assert_rules_match(dr, ref, "rule_")


def test_device_open_channel_rejects_what_the_host_builder_rejects():
    with pytest.raises(ValueError, match="at least 4 nodes"):
        dev.open_channel(lbm.D2Q9, np.zeros((6, 3), dtype=bool), 0.01)
