"""Device-side rule compiler: body voxelisation, wall links, Bouzidi and Zou-He rules built on the GPU.

The host builders (``geometry.voxelize``, ``geometry.wall_links``,
``link_rules.bouzidi_rules``, ``open_boundaries.open_channel``; reference
``src/lbm/geometry.py:140-206``, ``link_rules.py:154-188``,
``open_boundaries.py:96-186``) walk every node of the grid in NumPy: for a 256^3
duct with a sphere that is tens of seconds of set-up before the first step.
These functions take the same arguments and return the same objects (host
NumPy arrays, equal bit for bit: the kernels in ``csrc/compile.cu`` round
every operation as NumPy does), but do the per-node work on the device:

* ``voxelize(body, shape)`` -- ``lbm_ball_voxelize``;
* ``wall_links(lattice, body, solid)`` -- ``lbm_ball_links_count`` + ``_write``
  (links grouped by direction, nodes ascending, wall fractions q);
* ``bouzidi_rules(lattice, links, solid)`` -- ``lbm_bouzidi_links``;
* ``ball_channel(...)`` -- the three in sequence on one device-resident mask;
* ``open_channel(lattice, solid, inflow, rho_out)`` -- ``lbm_zou_he_count`` +
  ``_write``: the Zou-He inlet and outlet rules of an open channel.

Bodies are balls (``Ball``: circles and spheres), the body type of the
reference's builders that the benchmark configurations use.
"""

from __future__ import annotations

import numpy as np

from . import _native as N
from .geometry import Ball, WallLinks
from .lattice import VelocitySet, as_lattice
from .link_rules import AffineSet, LinkRules


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("the device-side rule compiler needs a CUDA device")
    N.load()
    return torch


def _grid(lattice: VelocitySet, shape) -> N.Grid:
    shape = tuple(int(v) for v in shape)
    nx, ny = shape[-1], shape[-2]
    nz = shape[0] if len(shape) == 3 else 1
    return N.Grid(N.LATTICE_CODE[lattice.name], N.LBM_F64, nx, ny, nz, nx, nx * ny * nz)


def _ball(body) -> tuple[float, float, float, float]:
    if not isinstance(body, Ball) and not hasattr(body, "radius"):
        raise TypeError("the device-side compiler handles balls (circles and spheres)")
    c = tuple(float(v) for v in body.center) + (0.0,)
    return c[0], c[1], c[2], float(body.radius) ** 2


def _mask_on_device(torch, solid):
    if isinstance(solid, torch.Tensor):
        return solid.to("cuda", torch.uint8).contiguous().reshape(-1)
    return torch.from_numpy(np.ascontiguousarray(np.asarray(solid, dtype=np.uint8)).reshape(-1)).to("cuda")


def _stream(torch) -> int:
    return torch.cuda.current_stream().cuda_stream


def voxelize_device(body, shape, solid=None):
    """Device uint8 mask (flat, natural node order) of ``solid`` (or zeros) with the ball set."""
    torch = _torch()
    lat = as_lattice("D2Q9" if len(shape) == 2 else "D3Q19")
    mask = _mask_on_device(torch, solid) if solid is not None else torch.zeros(int(np.prod(shape)), dtype=torch.uint8,
                                                                                   device="cuda")
    cx, cy, cz, r2 = _ball(body)
    N.call("lbm_ball_voxelize", N.C.byref(_grid(lat, shape)), cx, cy, cz, r2, N.ptr(mask), _stream(torch))
    return mask


def voxelize(body, shape) -> np.ndarray:
    """Boolean mask of the nodes inside the ball (``geometry.voxelize``), computed on the device."""
    if len(shape) != body.d:
        raise ValueError(f"grid shape {shape} does not match a {body.d}D body")
    return voxelize_device(body, shape).cpu().numpy().astype(bool).reshape(shape)


def wall_links_device(lattice: VelocitySet, body, mask, shape):
    """(node, direction, q) device tensors of every link from a fluid node into the ball; ``mask`` is
    the device uint8 solid mask (natural order). Raises if a node inside the ball is not solid."""
    torch = _torch()
    lattice = as_lattice(lattice)
    grid = _grid(lattice, shape)
    cx, cy, cz, r2 = _ball(body)
    lib = N.load()
    n_scratch = int(lib.lbm_ball_links_scratch(N.C.byref(grid)))
    if n_scratch <= 0:
        raise N.NativeError("lbm_ball_links_scratch: invalid grid")
    scratch = torch.empty(n_scratch, dtype=torch.int64, device="cuda")
    stream = _stream(torch)
    N.call("lbm_ball_links_count", N.C.byref(grid), N.ptr(mask), cx, cy, cz, r2, N.ptr(scratch), stream)
    m = lattice.q * ((grid.qstride + 255) // 256)  # the per-(direction, block) counts come first
    count, stray = (int(v) for v in scratch[m:m + 2].cpu().tolist())
    if stray:
        raise ValueError("every node inside the body must be marked solid")
    node = torch.empty(count, dtype=torch.int64, device="cuda")
    direction = torch.empty(count, dtype=torch.int32, device="cuda")
    q = torch.empty(count, dtype=torch.float64, device="cuda")
    if count:
        N.call("lbm_ball_links_write", N.C.byref(grid), N.ptr(mask), cx, cy, cz, r2, N.ptr(scratch), N.ptr(node),
               N.ptr(direction), N.ptr(q), stream)
    return node, direction, q


def wall_links(lattice: VelocitySet, body, solid) -> WallLinks:
    """``geometry.wall_links`` on the device: same links, same order, same fractions."""
    lattice = as_lattice(lattice)
    shape = np.asarray(solid).shape
    if lattice.d != body.d or len(shape) != body.d:
        raise ValueError(f"{lattice.name}, a {body.d}D body and grid {shape} must agree")
    torch = _torch()
    node, direction, q = wall_links_device(lattice, body, _mask_on_device(torch, solid), shape)
    return WallLinks(node.cpu().numpy(), direction.cpu().numpy().astype(np.int64), q.cpu().numpy())


def _bouzidi_arrays(lattice, mask, shape, node, direction, q):
    torch = _torch()
    n = int(node.numel())
    keep = torch.empty(n, dtype=torch.uint8, device="cuda")
    tdir = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    tnode = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    coeff = torch.empty((n, 2), dtype=torch.float64, device="cuda")
    N.call("lbm_bouzidi_links", N.C.byref(_grid(lattice, shape)), N.ptr(mask), n, N.ptr(node), N.ptr(direction),
           N.ptr(q), N.ptr(keep), N.ptr(tdir), N.ptr(tnode), N.ptr(coeff), _stream(torch))
    k = keep.cpu().numpy().astype(bool)
    return (node.cpu().numpy()[k], direction.cpu().numpy().astype(np.int64)[k], tdir.cpu().numpy()[k],
            tnode.cpu().numpy()[k], coeff.cpu().numpy()[k])


def bouzidi_rules(lattice: VelocitySet, links: WallLinks, solid) -> LinkRules:
    """``link_rules.bouzidi_rules`` on the device: same rules, same order, same coefficients."""
    torch = _torch()
    lattice = as_lattice(lattice)
    shape = np.asarray(solid).shape
    to = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)  # noqa: E731
    x, j, tdir, tnode, coeff = _bouzidi_arrays(lattice, _mask_on_device(torch, solid), shape,
                                               to(links.node, torch.int64), to(links.direction, torch.int32),
                                               to(links.q, torch.float64))
    return LinkRules(x, j, AffineSet.from_dense(tdir, tnode, coeff, np.zeros(x.size)))


def ball_channel(lattice: VelocitySet, body, solid):
    """Voxelise the ball into ``solid`` and build its wall links and Bouzidi rules, the mask kept on
    the device in between: ``(solid, links, rules)`` as ``voxelize`` + ``wall_links`` +
    ``bouzidi_rules`` return them."""
    torch = _torch()
    lattice = as_lattice(lattice)
    solid = np.asarray(solid, dtype=bool)
    shape = solid.shape
    mask = voxelize_device(body, shape, solid)
    node, direction, q = wall_links_device(lattice, body, mask, shape)
    x, j, tdir, tnode, coeff = _bouzidi_arrays(lattice, mask, shape, node, direction, q)
    links = WallLinks(node.cpu().numpy(), direction.cpu().numpy().astype(np.int64), q.cpu().numpy())
    rules = LinkRules(x, j, AffineSet.from_dense(tdir, tnode, coeff, np.zeros(x.size)))
    return mask.cpu().numpy().astype(bool).reshape(shape), links, rules


def _zou_he_column(torch, lattice, mask, shape, column, sign, layer_x, layer, velocity, rho_out):
    """Pass 1 of one open column: (grid, scratch, arguments, rule rows, widest rule)."""
    grid = _grid(lattice, shape)
    lib = N.load()
    n_scratch = int(lib.lbm_zou_he_scratch(N.C.byref(grid)))
    if n_scratch <= 0:
        raise N.NativeError("lbm_zou_he_scratch: invalid grid")
    scratch = torch.empty(n_scratch, dtype=torch.int64, device="cuda")
    plane = _mask_on_device(torch, layer)
    args = (N.C.byref(grid), N.ptr(mask), column, sign, layer_x, N.ptr(plane), N.ptr(velocity), float(rho_out))
    N.call("lbm_zou_he_count", *args, N.ptr(scratch), _stream(torch))
    n = int(np.prod(shape[:-1]))
    nodes, width = (int(v) for v in scratch[n:n + 2].cpu().tolist())
    n_unknown = sum(1 for c in lattice.c if sign * c[0] == 1)
    return (args, scratch, plane), nodes * n_unknown, width


def open_channel(lattice: VelocitySet, solid, inflow, rho_out: float = 1.0):
    """``open_boundaries.open_channel`` on the device: the same closed mask and the same rules --
    rule order, packed terms, coefficients and constants bit for bit (reference
    ``open_boundaries.py:96-186``). ``inflow`` broadcasts to (d, *cross_section) and acts at
    x = 1; ``rho_out`` is imposed at x = nx - 2. One thread per node of each open column
    (``lbm_zou_he_count`` + ``lbm_zou_he_write``); the x = 0 and x = nx - 1 layers are closed on the
    host, as ``open_channel`` does."""
    from .open_boundaries import _layers

    torch = _torch()
    lattice = as_lattice(lattice)
    closed, inlet, outlet = _layers(solid)
    shape = closed.shape
    if len(shape) != lattice.d:
        raise ValueError(f"{lattice.name} needs a {lattice.d}D mask, got shape {shape}")
    nx = shape[-1]
    mask = _mask_on_device(torch, closed)
    cross = shape[:-1]
    vel = np.array(np.broadcast_to(np.asarray(inflow, dtype=np.float64), (lattice.d, *cross)))  # a writable copy
    velocity = torch.from_numpy(vel.reshape(lattice.d, -1)).to("cuda")
    columns = [_zou_he_column(torch, lattice, mask, shape, 1, +1, 0, inlet[..., 0], velocity, 1.0),
               _zou_he_column(torch, lattice, mask, shape, nx - 2, -1, nx - 1, outlet[..., -1], None, rho_out)]
    rows = sum(r for _, r, _ in columns)
    width = max([max(w, 1) for _, r, w in columns if r], default=1)
    node = torch.empty(rows, dtype=torch.int64, device="cuda")
    direction = torch.empty(rows, dtype=torch.int64, device="cuda")
    tdir = torch.empty((rows, width), dtype=torch.int64, device="cuda")
    tnode = torch.empty((rows, width), dtype=torch.int64, device="cuda")
    coeff = torch.empty((rows, width), dtype=torch.float64, device="cuda")
    const = torch.empty(rows, dtype=torch.float64, device="cuda")
    start = 0
    for (args, scratch, _plane), r, _ in columns:
        if r:
            sl = slice(start, start + r)
            N.call("lbm_zou_he_write", *args, N.ptr(scratch), width, N.ptr(node[sl]), N.ptr(direction[sl]),
                   N.ptr(tdir[sl]), N.ptr(tnode[sl]), N.ptr(coeff[sl]), N.ptr(const[sl]), _stream(torch))
        start += r
    host = lambda t: t.cpu().numpy()  # noqa: E731
    rules = LinkRules(host(node), host(direction), AffineSet.from_dense(host(tdir), host(tnode), host(coeff),
                                                                        host(const)))
    return closed, rules
