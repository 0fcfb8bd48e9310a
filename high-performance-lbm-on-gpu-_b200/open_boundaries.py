"""Zou-He velocity inlet and pressure outlet as link rules (Hecht-Harting form).

Same boundary scheme as the reference (``src/lbm/open_boundaries.py:96-186``):
the x = 0 and x = nx - 1 layers become resting solid nodes and every unknown
population (c.n = +1) of the first/last fluid column is an affine rule in the
streamed populations s_k of its node::

    rho (1 - u_n) = S_0 + 2 S_-                 (mass and normal momentum)
    f_j = s_opp(j) + 6 w_j (c_j . rho u) - sum_t (c_j . t) N_t
    N_t = 1/2 sum_{c.n = 0} s_k (c_k . t) - rho u_t / 3

Inlet: u prescribed, rho = (S_0 + 2 S_-)/(1 - u_n). Outlet: rho prescribed,
tangential u = 0. Corner nodes get the full treatment.

The builder here is vectorised over the nodes of a column: every rule is a
coefficient vector over the Q streamed populations of its node, and each
streamed population is one (direction, node) term (a pull from x - c_k, or the
bounce-back reflection f*_opp(k)(x) when x - c_k is solid). Keys never
collide, so no term merging is needed. ``zou_he_inlet_derivative`` returns the
exact derivative of the inlet rules with respect to a scale of the inflow
velocity, used by the adjoint.
"""

from __future__ import annotations

import numpy as np

from .geometry import neighbour_index
from .lattice import VelocitySet
from .link_rules import AffineSet, LinkRules


def _column_nodes(solid: np.ndarray, column: int) -> np.ndarray:
    """Flat indices of the fluid nodes of x column ``column`` (ascending)."""
    shape = solid.shape
    cross = np.flatnonzero(~solid[..., column].ravel())
    coords = np.unravel_index(cross, solid[..., column].shape)
    return np.ravel_multi_index((*coords, np.full(cross.size, column)), shape)


def _stream_keys(lattice: VelocitySet, solid_flat, nodes, shape):
    """(direction, node) of the streamed population s_k at each node: (M, Q) each."""
    q = lattice.q
    opp = np.asarray(lattice.opposite)
    key_dir = np.empty((nodes.size, q), dtype=np.int64)
    key_node = np.empty((nodes.size, q), dtype=np.int64)
    for k in range(q):
        src = neighbour_index(nodes, [-v for v in lattice.c[k]], shape)
        blocked = solid_flat[src]
        key_dir[:, k] = np.where(blocked, opp[k], k)
        key_node[:, k] = np.where(blocked, nodes, src)
    return key_dir, key_node


def _weighted_sum(a, key_w):
    """sum_k a[m, r, k] key_w[m, k], summed over k left to right: one fixed order on every host,
    which the device-side builder (``csrc/compile.cu``, ``zh_row``) follows."""
    acc = a[..., 0] * key_w[:, None, 0]
    for k in range(1, a.shape[-1]):
        acc = acc + a[..., k] * key_w[:, None, k]
    return acc


def _zou_he_coefficients(lattice, solid, layer_mask, column, sign, velocity=None, rho_out=None, dvel=None):
    """Rules of one open column as dense coefficient arrays.

    Returns ``(nodes, directions, key_dir, key_node, coeff, const, dcoeff, dconst)``
    with ``coeff`` of shape (R, Q) over the streamed keys of each rule's node;
    ``dcoeff``/``dconst`` are derivatives w.r.t. a scale of ``velocity`` when
    ``dvel`` (= d velocity / d scale) is given.
    """
    shape = solid.shape
    d, q = lattice.d, lattice.q
    solid_flat = solid.ravel()
    layer_flat = layer_mask.ravel()
    c = np.asarray(lattice.c, dtype=np.int64)
    w = np.asarray(lattice.w, dtype=np.float64)
    opp = np.asarray(lattice.opposite)
    c_n = sign * c[:, 0]
    zero_n = (c_n == 0).astype(np.float64)
    minus_n = (c_n == -1).astype(np.float64)
    unknown = np.flatnonzero(c_n == 1)

    nodes = _column_nodes(solid, column)
    # A node gets rules only if some unknown population streams in from the open layer.
    touches = np.zeros(nodes.size, dtype=bool)
    for j in unknown:
        touches |= layer_flat[neighbour_index(nodes, [-v for v in lattice.c[j]], shape)]
    nodes = nodes[touches]
    m = nodes.size
    key_dir, key_node = _stream_keys(lattice, solid_flat, nodes, shape)

    known = np.broadcast_to(zero_n + 2.0 * minus_n, (m, q))  # coefficients of S_0 + 2 S_-
    coords = np.unravel_index(nodes, shape)
    derive = dvel is not None
    if velocity is not None:
        u = np.stack([velocity[a][coords] for a in range(d)])  # (d, m)
        du = np.stack([dvel[a][coords] for a in range(d)]) if derive else np.zeros_like(u)
        denom = 1.0 - sign * u[0]
        rho_c = known / denom[:, None]
        rho_k = np.zeros(m)
        drho_c = known * (sign * du[0] / denom**2)[:, None]
        rho_u_c = [rho_c * u[a][:, None] for a in range(d)]
        rho_u_k = [np.zeros(m) for _ in range(d)]
        drho_u_c = [drho_c * u[a][:, None] + rho_c * du[a][:, None] for a in range(d)]
        drho_u_k = [np.zeros(m) for _ in range(d)]
    else:
        rho_u_c = [-sign * known] + [np.zeros((m, q)) for _ in range(d - 1)]
        rho_u_k = [np.full(m, sign * rho_out)] + [np.zeros(m) for _ in range(d - 1)]
        drho_u_c = [np.zeros((m, q)) for _ in range(d)]
        drho_u_k = [np.zeros(m) for _ in range(d)]

    # N_t = 1/2 sum_{c.n=0} s_k c_kt - rho u_t / 3
    trans_c, trans_k, dtrans_c, dtrans_k = {}, {}, {}, {}
    for t in range(1, d):
        trans_c[t] = 0.5 * zero_n * c[:, t] - rho_u_c[t] / 3.0
        trans_k[t] = -rho_u_k[t] / 3.0
        dtrans_c[t] = -drho_u_c[t] / 3.0
        dtrans_k[t] = -drho_u_k[t] / 3.0

    coeff = np.zeros((m, unknown.size, q))
    const = np.zeros((m, unknown.size))
    dcoeff = np.zeros_like(coeff)
    dconst = np.zeros_like(const)
    for r, j in enumerate(unknown):
        coeff[:, r, opp[j]] += 1.0
        for a in range(d):
            if c[j, a]:
                s = 6.0 * w[j] * c[j, a]
                coeff[:, r] += s * rho_u_c[a]
                const[:, r] += s * rho_u_k[a]
                dcoeff[:, r] += s * drho_u_c[a]
                dconst[:, r] += s * drho_u_k[a]
        for t in range(1, d):
            if c[j, t]:
                coeff[:, r] -= c[j, t] * trans_c[t]
                const[:, r] -= c[j, t] * trans_k[t]
                dcoeff[:, r] -= c[j, t] * dtrans_c[t]
                dconst[:, r] -= c[j, t] * dtrans_k[t]
    # Shifted storage f~ = f - w: const_shifted = const - w_j + sum_k a_k w_k
    key_w = w[key_dir]  # (m, q)
    const = const - w[unknown][None, :] + _weighted_sum(coeff, key_w)
    dconst = dconst + _weighted_sum(dcoeff, key_w)

    node_out = np.repeat(nodes, unknown.size)
    dir_out = np.tile(unknown, m)
    return (
        node_out,
        dir_out,
        np.repeat(key_dir, unknown.size, axis=0),
        np.repeat(key_node, unknown.size, axis=0),
        coeff.reshape(-1, q),
        const.reshape(-1),
        dcoeff.reshape(-1, q),
        dconst.reshape(-1),
    )


def _as_rules(node, direction, key_dir, key_node, coeff, const) -> LinkRules:
    """Drop zero coefficients and pack terms to the front of each row."""
    nz = coeff != 0.0
    width = max(int(nz.sum(axis=1).max(initial=1)), 1)
    order = np.argsort(~nz, axis=1, kind="stable")[:, :width]
    kd = np.take_along_axis(key_dir, order, axis=1)
    kn = np.take_along_axis(key_node, order, axis=1)
    cf = np.take_along_axis(coeff, order, axis=1)
    live = np.take_along_axis(nz, order, axis=1)
    kd = np.where(live, kd, 0)
    kn = np.where(live, kn, 0)
    cf = np.where(live, cf, 0.0)
    return LinkRules(
        np.asarray(node, dtype=np.int64),
        np.asarray(direction, dtype=np.int64),
        AffineSet.from_dense(kd, kn, cf, const),
    )


def _layers(solid):
    solid = np.array(solid, dtype=bool)
    if solid.shape[-1] < 4:
        raise ValueError("an open channel needs at least 4 nodes along x")
    inlet = np.zeros_like(solid)
    outlet = np.zeros_like(solid)
    inlet[..., 0] = ~solid[..., 0]
    outlet[..., -1] = ~solid[..., -1]
    solid[..., 0] = True
    solid[..., -1] = True
    return solid, inlet, outlet


def _inflow_field(lattice, shape, inflow):
    velocity = np.zeros((lattice.d, *shape))
    velocity[..., 1] = np.broadcast_to(np.asarray(inflow, dtype=np.float64), velocity[..., 1].shape)
    return velocity


def open_channel(lattice: VelocitySet, solid: np.ndarray, inflow, rho_out: float = 1.0):
    """Close the x = 0 and x = nx-1 layers; return ``(solid, rules)`` (``open_boundaries.py:156-186``).

    ``inflow`` broadcasts to (d, *cross_section) and acts at x = 1; ``rho_out``
    is imposed at x = nx - 2.
    """
    solid, inlet, outlet = _layers(solid)
    velocity = _inflow_field(lattice, solid.shape, inflow)
    a = _zou_he_coefficients(lattice, solid, inlet, 1, +1, velocity=velocity)
    b = _zou_he_coefficients(lattice, solid, outlet, solid.shape[-1] - 2, -1, rho_out=rho_out)
    rules = LinkRules.concat(_as_rules(*a[:6]), _as_rules(*b[:6]))
    return solid, rules


def zou_he_inlet_derivative(lattice: VelocitySet, solid: np.ndarray, inflow, rho_out: float = 1.0):
    """Rules of ``open_channel`` plus their derivative w.r.t. a scale s of the inflow.

    With inflow(s) = s * inflow, returns ``(solid, rules, d_rules)`` where
    ``d_rules`` has the same (node, direction, term) layout as ``rules`` and
    holds d coeff / ds and d constant / ds at s = 1 (outlet rows are zero).
    The terms of ``d_rules`` are not packed, so padding entries may carry
    zero coefficients.
    """
    solid, inlet, outlet = _layers(solid)
    velocity = _inflow_field(lattice, solid.shape, inflow)
    a = _zou_he_coefficients(lattice, solid, inlet, 1, +1, velocity=velocity, dvel=velocity)
    b = _zou_he_coefficients(lattice, solid, outlet, solid.shape[-1] - 2, -1, rho_out=rho_out, dvel=velocity)
    node = np.concatenate([a[0], b[0]])
    direction = np.concatenate([a[1], b[1]])
    key_dir = np.concatenate([a[2], b[2]])
    key_node = np.concatenate([a[3], b[3]])
    coeff = np.concatenate([a[4], b[4]])
    const = np.concatenate([a[5], b[5]])
    dcoeff = np.concatenate([a[6], b[6]])
    dconst = np.concatenate([a[7], b[7]])
    rules = LinkRules(node, direction, AffineSet.from_dense(key_dir, key_node, coeff, const))
    d_rules = LinkRules(node, direction, AffineSet.from_dense(key_dir, key_node, dcoeff, dconst))
    return solid, rules, d_rules
