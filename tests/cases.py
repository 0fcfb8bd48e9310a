"""Test cases shared by the golden-vector generator and the parity tests.

Every builder takes a namespace ``ns`` that provides ``SimulationParams``,
``channel_walls``, ``cavity_walls``, ``voxelize``, ``circle``, ``sphere``,
``wall_links``, ``bouzidi_rules``, ``open_channel``, ``ImmersedBoundary`` and
``default_lattice``. ``tests/golden/make_golden.py`` passes the reference
package's modules, the tests pass this repository's package, so both build
the same inputs from the same geometry code. The mixed/Bouzidi/IBM/Zou-He
cases follow the reference's own GPU-equivalence tests
(``tests/test_cuda_backend.py:106-151``, ``tests/test_geometry_link_rules.py:121-150``,
``tests/test_ibm.py:319-338``, ``tests/test_open_boundaries.py:393-406``).
"""

from __future__ import annotations

import math

import numpy as np

EQUIVALENCE_STEPS = 40


def mixed(ns, dtype="float64", collision="trt", d=2, size=None):
    """Walls, a moving lid/plate, an obstacle and a body force; not block-aligned."""
    if d == 2:
        nx, ny = size or (45, 29)
        solid = ns.channel_walls(nx, ny)
        solid[10:16, 12:19] = True
        wall = np.zeros((2, ny, nx))
        wall[0, -1, :] = 0.05
        sizes, force = {"nx": nx, "ny": ny}, (1e-5, -2e-6)
    else:
        nx, ny, nz = size or (24, 20, 16)
        solid = ns.channel_walls(nx, ny, nz)
        solid[0, :, :] = True
        solid[-1, :, :] = True
        z0, y0, x0 = nz * 6 // 16, ny * 7 // 20, nx * 9 // 24
        solid[z0 : z0 + max(2, nz // 4), y0 : y0 + max(2, ny // 4), x0 : x0 + max(2, nx * 5 // 24)] = True
        wall = np.zeros((3, nz, ny, nx))
        wall[0, :, -1, :] = 0.05
        wall[2, :, -1, :] = -0.02
        sizes, force = {"nx": nx, "ny": ny, "nz": nz}, (1e-5, -2e-6, 3e-6)
    return ns.SimulationParams(
        **sizes, tau=0.7, collision=collision, force=force, solid=solid, wall_velocity=wall, dtype=dtype
    )


def bouzidi(ns, d=2, dtype="float64", size=None, body=None):
    """Channel, moving wall, Bouzidi body and force (reference ``bouzidi_params``)."""
    if d == 2:
        nx, ny = size or (45, 29)
        solid = ns.channel_walls(nx, ny)
        body = body or ns.circle(20.3, 13.6, 5.2)
        wall = np.zeros((2, ny, nx))
        wall[0, -1, :] = 0.05
        sizes, force = {"nx": nx, "ny": ny}, (1e-5, -2e-6)
    else:
        nx, ny, nz = size or (24, 20, 16)
        solid = ns.channel_walls(nx, ny, nz)
        body = body or ns.sphere(11.3, 9.6, 7.8, 4.1)
        solid[0] = True
        solid[-1] = True
        wall = np.zeros((3, nz, ny, nx))
        wall[0, :, -1, :] = 0.05
        wall[2, :, -1, :] = -0.02
        sizes, force = {"nx": nx, "ny": ny, "nz": nz}, (1e-5, -2e-6, 3e-6)
    lattice = ns.default_lattice(d)
    solid = solid | ns.voxelize(body, solid.shape)
    links = ns.wall_links(lattice, body, solid)
    params = ns.SimulationParams(
        **sizes, tau=0.7, collision="trt", force=force, solid=solid, wall_velocity=wall, dtype=dtype,
        link_rules=ns.bouzidi_rules(lattice, links, solid),
    )
    return params, links


def ibm(ns, d=2, dtype="float64", size=None, body=None):
    """Channel, moving wall, IBM body and force (reference ``ibm_params``)."""
    if d == 2:
        nx, ny = size or (45, 29)
        solid = ns.channel_walls(nx, ny)
        body = body or ns.circle(20.3, 13.6, 5.2)
        wall, force = np.zeros((2, ny, nx)), (1e-5, -2e-6)
        wall[0, -1] = 0.05
        sizes = {"nx": nx, "ny": ny}
    else:
        nx, ny, nz = size or (24, 20, 16)
        solid = ns.channel_walls(nx, ny, nz)
        body = body or ns.sphere(11.3, 9.6, 7.8, 3.6)
        wall, force = np.zeros((3, nz, ny, nx)), (1e-5, -2e-6, 3e-6)
        wall[0, :, -1] = 0.05
        sizes = {"nx": nx, "ny": ny, "nz": nz}
    return ns.SimulationParams(
        **sizes, tau=0.7, collision="trt", force=force, solid=solid, wall_velocity=wall, dtype=dtype,
        immersed=ns.ImmersedBoundary.from_ball(body),
    )


def open_channel_case(ns, d=2, rho_out=1.003, dtype="float64"):
    """Zou-He inlet/outlet channel (reference ``small_open_channel``)."""
    lattice = ns.default_lattice(d)
    nx, ny, nz = 12, 9, 5
    solid = ns.channel_walls(nx, ny) if d == 2 else ns.channel_walls(nx, ny, nz)
    inflow = np.zeros((d, *solid.shape[:-1]))
    inflow[0], inflow[1] = 0.04, 0.01
    if d == 3:
        inflow[2] = -0.02
    solid, rules = ns.open_channel(lattice, solid, inflow, rho_out=rho_out)
    sizes = {"nx": nx, "ny": ny} | ({"nz": nz} if d == 3 else {})
    params = ns.SimulationParams(**sizes, tau=0.7, collision="trt", solid=solid, dtype=dtype, link_rules=rules)
    return params, inflow


def cylinder_channel(ns, method="bouzidi", nx=880, ny=164, dtype="float32", u_max=0.05, iterations=3,
                     center=(200.0, 82.0), radius=20.0):
    """Config: D2Q9 channel 880 x 164, cylinder D = 40 at (200, 82), Zou-He in/out, Re = 100.

    Parabolic inflow as the reference's Schaefer-Turek builder
    (``cases/cylinder_benchmark.py:107-113``): walls halfway at y = 0.5 and
    ny - 1.5, profile 4 U y (H - y)/H^2 with y = j - 1/2.
    """
    lattice = ns.default_lattice(2)
    height = ny - 2
    y = np.arange(ny) - 0.5
    profile = np.where((y > 0) & (y < height), 4.0 * u_max * y * (height - y) / height**2, 0.0)
    inflow = np.stack([profile, np.zeros(ny)])
    solid = np.zeros((ny, nx), dtype=bool)
    solid[0, :] = solid[-1, :] = True
    body = ns.circle(*center, radius)
    immersed = None
    if method == "ibm":
        immersed = ns.ImmersedBoundary.from_ball(body, spacing=1.0, iterations=iterations)
    else:
        solid |= ns.voxelize(body, solid.shape)
    solid, open_rules = ns.open_channel(lattice, solid, inflow)
    rules = open_rules
    links = None
    if method == "bouzidi":
        links = ns.wall_links(lattice, body, solid)
        rules = ns.LinkRules.concat(open_rules, ns.bouzidi_rules(lattice, links, solid))
    u_mean = 2.0 * u_max / 3.0
    nu = u_mean * 40.0 / 100.0
    tau = 3.0 * nu + 0.5
    params = ns.SimulationParams(
        nx=nx, ny=ny, tau=tau, collision="trt", solid=solid, dtype=dtype, link_rules=rules, immersed=immersed
    )
    return params, links, inflow


def schaefer_turek(ns, test="2D-2", n=20, u_max=0.05, dtype="float32", collision="trt"):
    """The Schaefer-Turek DFG cylinder benchmark at N nodes per diameter, Bouzidi cylinder
    (the reference's ``cases/cylinder_benchmark.py:93-130``, ``build``).

    Channel H = 0.41, L = 2.2, D = 0.1 centred at (0.2, 0.2), nu = 1e-3 (SI); dx = D / N; the
    x = 0 layer is the Zou-He velocity inlet acting at x = 1, the last layer the pressure outlet;
    channel walls halfway at y = 0.5 and ny - 1.5. 2D-2: U_m = 1.5 m/s, Re = 100.
    Returns (params, cylinder links, u_mean, inflow profile u_x(y)).
    """
    height_si, length_si, diameter_si, centre_si, nu_si = 0.41, 2.2, 0.1, (0.2, 0.2), 1e-3
    u_m_si = {"2D-1": 0.3, "2D-2": 1.5}[test]
    dx = diameter_si / n
    ny = round(height_si / dx) + 2
    nx = round(length_si / dx) + 3
    height = ny - 2
    y = np.arange(ny) - 0.5
    profile = np.where((y > 0) & (y < height), 4.0 * u_max * y * (height - y) / height**2, 0.0)
    inflow = np.stack([profile, np.zeros(ny)])
    solid = np.zeros((ny, nx), dtype=bool)
    solid[0, :] = solid[-1, :] = True
    body = ns.circle(1.0 + centre_si[0] / dx, 0.5 + centre_si[1] / dx, 0.5 * n)
    solid |= ns.voxelize(body, solid.shape)
    lattice = ns.default_lattice(2)
    solid, open_rules = ns.open_channel(lattice, solid, inflow)
    links = ns.wall_links(lattice, body, solid)
    rules = ns.LinkRules.concat(open_rules, ns.bouzidi_rules(lattice, links, solid))
    u_mean = 2.0 * u_max / 3.0
    reynolds = u_m_si * 2.0 / 3.0 * diameter_si / nu_si
    nu = u_mean * n / reynolds
    params = ns.SimulationParams(nx=nx, ny=ny, tau=3.0 * nu + 0.5, collision=collision, solid=solid, dtype=dtype,
                                 link_rules=rules)
    return params, links, u_mean, profile


def lift_period(t, cl):
    """Mean period of C_L(t) from its upward zero crossings, each located by linear interpolation
    between the samples around it (the reference's ``cylinder_benchmark.lift_period``)."""
    t, cl = np.asarray(t, dtype=np.float64), np.asarray(cl, dtype=np.float64)
    up = np.flatnonzero((cl[:-1] < 0) & (cl[1:] >= 0))
    if len(up) < 2:
        raise ValueError("need at least two upward zero crossings of C_L to measure a period")
    crossings = t[up] - cl[up] * (t[up + 1] - t[up]) / (cl[up + 1] - cl[up])
    return float(np.mean(np.diff(crossings)))


def sphere_channel(ns, nx=128, ny=64, nz=64, radius=8.0, u_in=0.04, tau=0.6, dtype="float32"):
    """Config: D3Q19 channel 128 x 64 x 64, Bouzidi sphere r = 8, Zou-He inlet U, outlet rho = 1."""
    lattice = ns.default_lattice(3)
    solid = np.zeros((nz, ny, nx), dtype=bool)
    solid[:, [0, -1], :] = True
    solid[[0, -1], :, :] = True
    body = ns.sphere(nx / 4.0, (ny - 1) / 2.0, (nz - 1) / 2.0, radius)
    solid |= ns.voxelize(body, solid.shape)
    inflow = np.zeros((3, nz, ny))
    inflow[0] = u_in
    inflow[:, [0, -1], :] = 0.0
    inflow[:, :, [0, -1]] = 0.0
    solid, open_rules = ns.open_channel(lattice, solid, inflow)
    links = ns.wall_links(lattice, body, solid)
    rules = ns.LinkRules.concat(open_rules, ns.bouzidi_rules(lattice, links, solid))
    params = ns.SimulationParams(
        nx=nx, ny=ny, nz=nz, tau=tau, collision="trt", solid=solid, dtype=dtype, link_rules=rules
    )
    return params, links, inflow


def duct(ns, n=256, nx=None, dtype="float32", tau=0.9, force=1e-6):
    """Config: D3Q19 square duct, walls at y, z = 0 and n-1, periodic in x, F = (force, 0, 0)."""
    nx = n if nx is None else nx
    solid = np.zeros((n, n, nx), dtype=bool)
    solid[:, [0, -1], :] = True
    solid[[0, -1], :, :] = True
    return ns.SimulationParams(
        nx=nx, ny=n, nz=n, tau=tau, collision="trt", force=(force, 0.0, 0.0), solid=solid, dtype=dtype
    )


def tgv(ns, n=512, dtype="float32", tau=0.8, u0=0.01):
    """Config: D2Q9 TRT Taylor-Green vortex, u0 (sin kx cos ky, -cos kx sin ky), k = 2 pi / n."""
    params = ns.SimulationParams(nx=n, ny=n, tau=tau, collision="trt", dtype=dtype)
    k = 2.0 * math.pi / n
    y, x = np.mgrid[0:n, 0:n].astype(np.float64)
    ux = u0 * np.sin(k * x) * np.cos(k * y)
    uy = -u0 * np.cos(k * x) * np.sin(k * y)
    return params, (1.0, ux, uy)


def cavity(ns, n, re, lid=0.1, dtype="float32"):
    """Config: D2Q9 TRT lid-driven cavity of side n, tau = 3 lid n / Re + 1/2."""
    solid, wall = ns.cavity_walls(n, lid)
    tau = 3.0 * lid * n / re + 0.5
    return ns.SimulationParams(
        nx=n + 2, ny=n + 2, tau=tau, collision="trt", solid=solid, wall_velocity=wall, dtype=dtype
    )


def random_state(params, seed=0, rho_scale=0.01, u_scale=0.02):
    """rho = 1 + 0.01 N, u = 0.02 N (reference ``tests/test_cuda_backend.py:154-159``)."""
    rng = np.random.default_rng(seed)
    shape = params.shape
    rho = 1 + rho_scale * rng.standard_normal(shape)
    u = u_scale * rng.standard_normal((params.d, *shape))
    return (rho, *u)
