"""NumPy restatement of the reference LBM step -- TEST INFRASTRUCTURE ONLY.

Each function cites the reference file:line it restates (paths relative to the
reference project). Written against plain NumPy; every array keeps the
simulation dtype so float32 runs round like the reference's float32 runs.

16-bit storage ("float16", "bfloat16") has no counterpart in the reference.
The oracle emulates it: arithmetic in float32, populations rounded to the
storage format after every step exactly as the CUDA kernels store them
(``stochastic_round``: the same hash of node, step and direction, so the
rounding decisions are replayed bit for bit; the initial state is rounded to
nearest, ``quantize``), so the GPU path can be checked bit-for-tolerance.
"""

from __future__ import annotations

import numpy as np

FP16_SCALE = 2.0**14
"""Power-of-two factor applied before rounding to float16 (keeps small f~ out of subnormals)."""


class OracleDiverged(RuntimeError):
    def __init__(self, step, location, reason):
        self.step, self.location, self.reason = step, location, reason
        super().__init__(f"simulation diverged by step {step}: {reason} at node {location}")


def compute_dtype(dtype: str):
    return np.float64 if dtype == "float64" else np.float32


def quantize(f: np.ndarray, dtype: str) -> np.ndarray:
    """Round float32 values to the storage format and back (no-op for float32/float64)."""
    if dtype == "float16":
        scaled = (f.astype(np.float32) * np.float32(FP16_SCALE)).astype(np.float16)
        return scaled.astype(np.float32) * np.float32(1.0 / FP16_SCALE)
    if dtype == "bfloat16":
        bits = np.ascontiguousarray(f, dtype=np.float32).view(np.uint32).astype(np.uint64)
        bias = 0x7FFF + ((bits >> 16) & 1)
        rounded = ((bits + bias) & 0xFFFF0000).astype(np.uint32)
        return rounded.view(np.float32)
    return f


SR_MULT = 0x9E3779B9


def lowbias32(x):
    """32-bit integer hash "lowbias32" of C. Wellons' hash-prospector (uint32 in, uint32 out)."""
    x = np.asarray(x, dtype=np.uint32).copy()
    x ^= x >> np.uint32(16)
    x *= np.uint32(0x7FEB352D)
    x ^= x >> np.uint32(15)
    x *= np.uint32(0x846CA68B)
    x ^= x >> np.uint32(16)
    return x


def sr_keys(q: int) -> np.ndarray:
    """Per-direction keys K_i = lowbias32(i + 1)."""
    return lowbias32(np.arange(1, q + 1, dtype=np.uint32))


def _float16_stochastic(v: np.ndarray, r: np.ndarray) -> np.ndarray:
    """float32 -> float16 as cvt.rs rounds: |v| + r 2^-13 ulp(|v|), truncated; >= 65536 -> inf."""
    a = np.abs(v.astype(np.float64))
    _, ex = np.frexp(a)
    ulp = np.ldexp(1.0, np.maximum(ex - 1, -14) - 10)
    with np.errstate(invalid="ignore"):
        y = a + r.astype(np.float64) * ulp / 8192.0
        q = np.floor(y / ulp) * ulp
    q = np.where(q >= 65536.0, np.inf, q)
    return np.copysign(q, v).astype(np.float16)


def stochastic_round(f: np.ndarray, dtype: str, step: int) -> np.ndarray:
    """Stochastic rounding of post-collision populations to 16-bit storage, as the step kernels store them.

    f has shape (q, *shape) in natural order (x last). Nodes pair up along x
    (x even with x + 1): pair = row * ceil(nx / 2) + x // 2, h =
    lowbias32(pair ^ lowbias32(step)) and direction i draws the 32-bit word
    (h ^ K_i) * 0x9E3779B9; the even node takes bits 0-12 (float16, after the
    2^14 scale; 0-15 for bfloat16) as r, the odd node bits 16-28 (16-31).
    float16: |v| + r 2^-13 ulp(|v|) truncated toward zero, magnitudes that
    reach 65536 infinite; bfloat16: r added to the float32 bit pattern, then
    truncated. float32/float64 storage is returned unchanged.
    """
    if dtype not in ("float16", "bfloat16"):
        return f
    q = f.shape[0]
    nx = f.shape[-1]
    rows = int(np.prod(f.shape[1:-1], dtype=np.int64))
    flat = f.reshape(q, rows, nx)
    x = np.arange(nx, dtype=np.int64)
    pair = (np.arange(rows, dtype=np.int64)[:, None] * ((nx + 1) // 2) + (x // 2)[None, :]).astype(np.uint32)
    odd = np.broadcast_to((x & 1).astype(bool)[None, :], (rows, nx))
    h = lowbias32(pair ^ lowbias32(np.uint32(step & 0xFFFFFFFF)))
    keys = sr_keys(q)
    out = np.empty(flat.shape, dtype=np.float32)
    with np.errstate(over="ignore"):
        for i in range(q):
            word = (h ^ keys[i]) * np.uint32(SR_MULT)
            xi = flat[i].astype(np.float32)
            if dtype == "float16":
                r = np.where(odd, (word >> np.uint32(16)) & np.uint32(0x1FFF), word & np.uint32(0x1FFF))
                scaled = xi * np.float32(FP16_SCALE)
                out[i] = _float16_stochastic(scaled, r).astype(np.float32) * np.float32(1.0 / FP16_SCALE)
            else:
                r = np.where(odd, word >> np.uint32(16), word & np.uint32(0xFFFF))
                bits = (xi.view(np.uint32).astype(np.uint64) + r.astype(np.uint64)) >> np.uint64(16) << np.uint64(16)
                out[i] = bits.astype(np.uint32).view(np.float32)
    return out.reshape(f.shape)


def _dot(c, vec):
    """c . vec skipping zero components (reference ``equilibrium.py:23-30``)."""
    return sum(ca * va for ca, va in zip(c, vec, strict=True) if ca)


def equilibrium(lattice, drho, u):
    """Shifted 2nd-order equilibrium w_i [drho + rho (3cu + 4.5 (cu)^2 - 1.5 u.u)] (``equilibrium.py:40-58``)."""
    rho = 1.0 + drho
    usq = 1.5 * sum(ua * ua for ua in u)
    out = []
    for ci, wi in zip(lattice.c, lattice.w, strict=True):
        cu = 3.0 * _dot(ci, u)
        out.append(wi * (drho + rho * (cu + 0.5 * cu * cu - usq)))
    return np.stack(out)


def _momentum(lattice, f):
    return tuple(
        sum(ca * f[i] for i, ca in enumerate(lattice.component(a)) if ca) for a in range(lattice.d)
    )


def _is_zero(v) -> bool:
    return isinstance(v, (int, float)) and v == 0.0


def guo_source(lattice, u, force, wp, wm):
    """Guo source split into even/odd parts (``forcing.py:37-56``)."""
    u_dot_f = sum(ua * fa for ua, fa in zip(u, force, strict=True))
    ap, am = 1.0 - 0.5 * wp, 1.0 - 0.5 * wm
    out = []
    for ci, wi in zip(lattice.c, lattice.w, strict=True):
        cf = _dot(ci, force)
        cu = _dot(ci, u)
        out.append(wi * (ap * (9.0 * cu * cf - 3.0 * u_dot_f) + am * (3.0 * cf)))
    return np.stack(out)


def collide(lattice, f, wp, wm, force):
    """TRT + Guo on every node of f (q, ...) (``collision.py:59-88``)."""
    drho = f.sum(axis=0)
    rho = 1.0 + drho
    u = tuple((ja + 0.5 * fa) / rho for ja, fa in zip(_momentum(lattice, f), force, strict=True))
    neq = f - equilibrium(lattice, drho, u)
    neq_o = neq[list(lattice.opposite)]
    post = f - (0.5 * wp) * (neq + neq_o) - (0.5 * wm) * (neq - neq_o)
    if any(not _is_zero(fa) for fa in force):
        post = post + guo_source(lattice, u, force, wp, wm)
    return post


def collide_regularized(lattice, f, wp, force):
    """Regularised collision with Guo forcing on every node of f (q, ...).

    Not in the reference (its roadmap item 3, README "High Reynolds numbers");
    restated from the published method: projective regularisation, J. Latt and
    B. Chopard, Math. Comput. Simul. 72 (2006) 165-168 (also T. Krueger et al.,
    The Lattice Boltzmann Method, Springer 2017, sec. 10.6.5). The
    non-equilibrium part f^neq = f - feq (feq as in ``equilibrium``, u = (j +
    F/2)/rho) is replaced by its projection on the Hermite polynomials up to
    second order, w_i [3 c_i . m1 + 4.5 (c_i c_i - I/3) : Pi] with m1 = sum c
    f^neq and Pi = sum c c f^neq, which then relaxes at rate wp; the Guo source
    is split as in ``guo_source``. Since m1 = -F/2, the odd part of the update
    is 1.5 w c.F whatever the odd rate:
        f*_i = feq_i + 1.5 w_i c_i.F + (1 - wp) 4.5 w_i (c_i.Pi.c_i - tr Pi / 3)
               + (1 - wp/2) w_i (9 (c_i.u)(c_i.F) - 3 u.F)
    """
    d = lattice.d
    drho = f.sum(axis=0)
    rho = 1.0 + drho
    u = tuple((ja + 0.5 * fa) / rho for ja, fa in zip(_momentum(lattice, f), force, strict=True))
    neq = f - equilibrium(lattice, drho, u)
    c = np.asarray(lattice.c)
    pi = {}
    for a in range(d):
        for b in range(a, d):
            pi[a, b] = sum(c[i, a] * c[i, b] * neq[i] for i in range(lattice.q) if c[i, a] * c[i, b])
    trace = sum(pi[a, a] for a in range(d))
    u_dot_f = sum(ua * fa for ua, fa in zip(u, force, strict=True))
    out = []
    for i, wi in enumerate(lattice.w):
        ci = c[i]
        cpc = sum(ci[a] * ci[b] * pi[min(a, b), max(a, b)] for a in range(d) for b in range(d) if ci[a] * ci[b])
        cf = _dot(ci, force)
        cu = _dot(ci, u)
        feq = wi * (drho + rho * (3.0 * cu + 4.5 * cu * cu - 1.5 * sum(ua * ua for ua in u)))
        out.append(feq + 1.5 * wi * cf + (1.0 - wp) * 4.5 * wi * (cpc - trace / 3.0)
                   + (1.0 - 0.5 * wp) * wi * (9.0 * cu * cf - 3.0 * u_dot_f))
    return np.stack(out).astype(f.dtype)


def _chimera(am, a0, ap, u):
    """Central moments of orders 0, 1, 2 along one axis of the three populations with c = -1, 0, +1,
    about velocity u (the 'chimera' transformation of the cumulant method)."""
    k0 = (am + a0) + ap
    s = ap - am
    k1 = s - u * k0
    k2 = ((ap + am) - (2.0 * u) * s) + (u * u) * k0
    return k0, k1, k2


def _chimera_inverse(k0, k1, k2, u):
    """The populations (c = -1, 0, +1) of central moments (k0, k1, k2) about u."""
    s = k1 + u * k0
    p = (k2 + (2.0 * u) * s) - (u * u) * k0
    return 0.5 * (p - s), k0 - p, 0.5 * (p + s)


def collide_cumulant(lattice, f, wp, force):
    """Cumulant collision on every node of f (9, ...), D2Q9 only.

    Not in the reference (its roadmap item 3, README "High Reynolds numbers");
    restated from the published method: the cumulant lattice Boltzmann
    equation, M. Geier, M. Schoenherr, A. Pasquali, M. Krafczyk, Comput. Math.
    Appl. 70 (2015) 507-547 (its central-moment 'chimera' transformation,
    sec. 3, and forcing by the half-force velocity shift, sec. 2.4), written for
    the 2D tensor-product lattice D2Q9, whose nine populations carry the
    nine moments of orders (m, n), m, n <= 2. With u = (j + F/2)/rho and the
    central moments k_mn = sum_i f_i (c_ix - u_x)^m (c_iy - u_y)^n:

    * second order: k20 - k02 and k11 relax with wp (shear viscosity
      (1/wp - 1/2)/3), k20 + k02 is set to its equilibrium 2 rho/3 (bulk rate 1);
    * third order k21, k12 -> 0 and the fourth-order cumulant
      C22 = k22/rho - (k20 k02 + 2 k11^2)/rho^2 -> 0 (rates 1), so k22* = (k20* k02* + 2 k11*^2)/rho;
    * first order mirrored, k10* = -k10 (= F_x/2: the post-collision momentum is j + F).

    The cumulant relations use the second-order central moments about u (the
    first-order ones, -F/2, enter at O(F^2), as in the published scheme).

    Evaluated on shifted populations f~ = f - w, in deviations only, so that
    round-off stays at the scale of f~ (as in the TRT form): the chimera
    transformation along x then y gives the central moments k~ of f~ about u;
    those of the weights are M_m(u_x) M_n(u_y), M = (1, -u, 1/3 + u^2)
    (w_ij = W_i W_j, W = (1/6, 2/3, 1/6)), and every post-collision moment is
    written directly as its difference from the weights' one, p = k* - M M:
        p00 = drho, p10 = 2 u_x - k~10, p01 = 2 u_y - k~01,
        D* = (1 - wp) ((k~20 - k~02) + (u_x^2 - u_y^2)), k11* = (1 - wp) (k~11 + u_x u_y),
        a = drho/3 + D*/2, b = drho/3 - D*/2,
        p20 = a - u_x^2, p02 = b - u_y^2, p11 = k11* - u_x u_y,
        p21 = u_y (1/3 + u_x^2), p12 = u_x (1/3 + u_y^2),
        p22 = (drho/9 + a b + 2 k11*^2)/rho - (u_x^2 + u_y^2)/3 - u_x^2 u_y^2;
    then the inverse chimera along y, then x.
    """
    if lattice.q != 9:
        raise ValueError("the cumulant collision is built for D2Q9")
    c = lattice.c
    index = {tuple(ci): i for i, ci in enumerate(c)}
    dt = f.dtype.type
    drho = f.sum(axis=0)
    rho = dt(1.0) + drho
    jx, jy = _momentum(lattice, f)
    ux = (jx + 0.5 * force[0]) / rho
    uy = (jy + 0.5 * force[1]) / rho
    # along x, per row cy = -1, 0, 1; then along y: k[m][n]
    rows = [_chimera(f[index[(-1, cy)]], f[index[(0, cy)]], f[index[(1, cy)]], ux) for cy in (-1, 0, 1)]
    k = [_chimera(rows[0][m], rows[1][m], rows[2][m], uy) for m in range(3)]
    third = dt(1.0 / 3.0)
    uxx, uyy, uxy = ux * ux, uy * uy, ux * uy
    keep = dt(1.0) - dt(wp)
    dev = keep * ((k[2][0] - k[0][2]) + (uxx - uyy))
    k11 = keep * (k[1][1] + uxy)
    d3 = drho * third
    a = d3 + dt(0.5) * dev
    b = d3 - dt(0.5) * dev
    x = (drho * dt(1.0 / 9.0) + a * b) + dt(2.0) * (k11 * k11)
    p22 = (x / rho - (uxx + uyy) * third) - uxx * uyy
    post = [[drho, dt(2.0) * uy - k[0][1], b - uyy],
            [dt(2.0) * ux - k[1][0], k11 - uxy, ux * (third + uyy)],
            [a - uxx, uy * (third + uxx), p22]]
    cols = [_chimera_inverse(post[m][0], post[m][1], post[m][2], uy) for m in range(3)]  # cols[m][b]
    out = np.empty_like(f)
    for r, cy in enumerate((-1, 0, 1)):
        am, a0, ap = _chimera_inverse(cols[0][r], cols[1][r], cols[2][r], ux)
        out[index[(-1, cy)]], out[index[(0, cy)]], out[index[(1, cy)]] = am, a0, ap
    return out


def stream_pull(lattice, f):
    """f_i(x) = f*_i(x - c_i), periodic (``streaming.py:32-37``)."""
    axes = tuple(range(lattice.d))
    return np.stack([np.roll(f[i], tuple(reversed(ci)), axis=axes) for i, ci in enumerate(lattice.c)])


def bounce_back_links(lattice, solid, wall, dtype):
    """Fluid-to-solid link mask and Ladd term 6 w_i (c_i . u_w) (``boundaries.py:53-72``)."""
    fluid = ~solid
    axes = tuple(range(lattice.d))
    masks, terms = [], []
    for ci, wi in zip(lattice.c, lattice.w, strict=True):
        shift = tuple(reversed(ci))
        from_solid = np.roll(solid, shift, axis=axes) & fluid
        cu = sum(ca * np.roll(wall[a].astype(dtype), shift, axis=axes) for a, ca in enumerate(ci) if ca)
        term = (2.0 * wi / lattice.cs2) * cu
        masks.append(from_solid)
        terms.append(np.where(from_solid, term, 0.0).astype(dtype))
    return np.stack(masks), np.stack(terms)


def _neighbour(nodes, c, shape):
    coords = np.unravel_index(np.asarray(nodes, dtype=np.int64), shape)
    moved = tuple((coords[a] + int(s)) % shape[a] for a, s in enumerate(tuple(c)[::-1]))
    return np.ravel_multi_index(moved, shape)


def _roma(r):
    a = np.abs(np.asarray(r, dtype=np.float64))
    inner = (1.0 + np.sqrt(np.maximum(1.0 - 3.0 * a * a, 0.0))) / 3.0
    outer = (5.0 - 3.0 * a - np.sqrt(np.maximum(1.0 - 3.0 * (1.0 - a) ** 2, 0.0))) / 6.0
    return np.where(a <= 0.5, inner, np.where(a <= 1.5, outer, 0.0))


def _bincount(index, weights, n):
    """np.bincount with real or complex weights (complex: real and imaginary parts separately)."""
    if np.iscomplexobj(weights):
        return np.bincount(index, weights=weights.real, minlength=n) + 1j * np.bincount(index, weights=weights.imag, minlength=n)
    return np.bincount(index, weights=weights, minlength=n)


class _Ibm:
    """Direct-forcing IBM state (``ibm.py:123-214``), reference layout only."""

    def __init__(self, params, cdt):
        body = params.immersed
        lattice = params.lattice
        shape = params.shape
        d = lattice.d
        base = np.floor(body.markers - 0.5).astype(np.int64)
        offsets = np.indices((3,) * d).reshape(d, -1).T
        pts = base[:, None, :] + offsets[None]
        weights = np.prod(_roma(pts - body.markers[:, None, :]), axis=-1)
        flat = np.ravel_multi_index(tuple(pts[..., a] for a in range(d))[::-1], shape)
        nodes, inverse = np.unique(flat, return_inverse=True)
        self.nodes = nodes
        self.inverse = inverse.reshape(flat.shape)
        self.weights = weights.astype(cdt)
        self.areas = np.asarray(body.areas).astype(cdt)
        self.iterations = int(body.iterations)
        self.uniform = tuple(float(v) for v in params.force)
        self.d = d
        self.sources = np.stack([_neighbour(nodes, [-v for v in ck], shape) for ck in lattice.c])
        self.c = np.asarray(lattice.c)
        self.body_force = np.zeros(d)

    def moments(self, f):
        """rho and j (d, n) of the streamed populations at the stencil nodes (``ibm.py:160-173``)."""
        q = self.sources.shape[0]
        streamed = f.reshape(q, -1)[np.arange(q)[:, None], self.sources]  # (q, n)
        drho = streamed.sum(axis=0)
        rho = 1.0 + drho
        j = [sum(self.c[k, a] * streamed[k] for k in range(q) if self.c[k, a]) for a in range(self.d)]
        return rho, j

    def force_from_moments(self, rho, j):
        """Multi-direct passes (``ibm.py:189-214``): node force (d, n) and body force (d,).

        Complex inputs are allowed (the adjoint differentiates this by complex steps).
        """
        n = self.nodes.size
        u_star = np.stack([(j[a] + 0.5 * self.uniform[a]) / rho for a in range(self.d)])
        rho_marker = (self.weights * rho[self.inverse]).sum(axis=1)
        force = np.zeros((self.d, n), dtype=u_star.dtype)
        total = np.zeros(self.d, dtype=u_star.dtype)
        flat_inv = self.inverse.reshape(-1)
        for _ in range(self.iterations):
            u = u_star + force / (2.0 * rho)
            u_marker = (self.weights[None] * u[:, self.inverse]).sum(axis=2)
            f_marker = 2.0 * rho_marker * (0.0 - u_marker) * self.areas
            total = total + f_marker.sum(axis=1)
            spread = (self.weights[None] * f_marker[:, :, None]).reshape(self.d, -1)
            for a in range(self.d):
                force[a] = force[a] + _bincount(flat_inv, spread[a], n)
        return force, -total

    def force_field(self, f):
        force, self.body_force = self.force_from_moments(*self.moments(f))
        return force


class OracleSolver:
    """The reference solver's semantics on NumPy (``solver.py:61-292``).

    Accepts any parameter object with the reference's ``SimulationParams``
    attributes. ``force_field`` (optional, shape (d, *shape)) adds a per-node
    Guo force on top of the uniform one (an extension used by the adjoint).
    """

    def __init__(self, params, force_field=None):
        self.params = params
        self.lattice = params.lattice
        self.dtype = params.dtype
        self.cdt = compute_dtype(params.dtype)
        self.fluid = ~np.asarray(params.solid, dtype=bool)
        self.solid = np.asarray(params.solid, dtype=bool)
        self.mask, self.wall_term = bounce_back_links(self.lattice, self.solid, np.asarray(params.wall_velocity), self.cdt)
        self.rates = params.relaxation_rates
        self.time_step = 0
        n = int(np.prod(params.shape))
        self.n_nodes = n
        self.rules = None
        rules = params.link_rules
        if rules is not None and len(rules):
            v = rules.values
            slots = np.asarray(v.direction) * n + np.asarray(v.node)
            target = np.asarray(rules.direction) * n + np.asarray(rules.node)
            self.rules = (target, slots, np.asarray(v.coeff).astype(self.cdt), np.asarray(v.constant).astype(self.cdt))
        self.ibm = _Ibm(params, self.cdt) if params.immersed is not None else None
        self.field = None
        if self.ibm is not None:
            self.field = np.zeros((self.lattice.d, *params.shape), dtype=self.cdt)
        self.extra_force = None
        if force_field is not None:
            self.extra_force = np.asarray(force_field, dtype=self.cdt).reshape(self.lattice.d, *params.shape)
        self.initialize()

    # ---------------------------------------------------------------- state
    def initialize(self, rho=1.0, ux=0.0, uy=0.0, uz=0.0):
        """Equilibrium at u + F/(2 rho), combined in float64, cast once (``solver.py:101-117``)."""
        p = self.params
        d = self.lattice.d
        if d == 2 and np.any(np.asarray(uz) != 0):
            raise ValueError("a 2D simulation has no z velocity; leave uz at 0")
        comps = (ux, uy, uz)[:d]
        rho = np.broadcast_to(np.asarray(rho, dtype=np.float64), p.shape)
        force = self._force_components(np.float64)
        u = [np.broadcast_to(np.asarray(ua, dtype=np.float64), p.shape) + 0.5 * fa / rho for ua, fa in zip(comps, force, strict=True)]
        drho = np.asarray(rho - 1.0, dtype=self.cdt)
        f = equilibrium(self.lattice, drho, tuple(np.asarray(a, dtype=self.cdt) for a in u))
        self.f = quantize(f, self.dtype)
        self.time_step = 0
        self.round_step = 0

    def set_populations(self, f):
        self.f = np.array(f, dtype=self.cdt, copy=True)
        self.round_step = 0

    def _force_components(self, dt):
        """Uniform force, plus the per-node extension field (not the IBM field)."""
        force = tuple(float(v) for v in self.params.force)
        if self.extra_force is None:
            return force
        return tuple(force[a] + self.extra_force[a].astype(dt) for a in range(self.lattice.d))

    def collision_force(self):
        force = self._force_components(self.cdt)
        if self.field is None:
            return force
        return tuple(force[a] + self.field[a] for a in range(self.lattice.d))

    # ---------------------------------------------------------------- step
    def step(self):
        """One step (``solver.py:257-274``): IBM field, pull, bounce-back, rules, collide."""
        lattice = self.lattice
        f = self.f
        force = self._force_components(self.cdt)
        if self.ibm is not None:
            local = self.ibm.force_field(f)
            self.field.reshape(lattice.d, -1)[:, self.ibm.nodes] = local
            force = self.collision_force()
        streamed = stream_pull(lattice, f)
        reflected = f[list(lattice.opposite)] + self.wall_term
        streamed = np.where(self.mask, reflected, streamed)
        if self.rules is not None:
            target, slots, coeff, const = self.rules
            values = const + (coeff * f.reshape(-1)[slots]).sum(axis=1)
            streamed.reshape(-1)[target] = values
        model = getattr(self.params, "collision", "bgk")
        if model == "regularized":
            post = collide_regularized(lattice, streamed, self.rates[0], force)
        elif model == "cumulant":
            post = collide_cumulant(lattice, streamed, self.rates[0], force)
        else:
            post = collide(lattice, streamed, self.rates[0], self.rates[1], force)
        self.f = stochastic_round(np.where(self.fluid, post, f), self.dtype, self.round_step)
        self.round_step += 1

    def run(self, steps, check_every=500):
        done = 0
        while done < steps:
            k = min(check_every - done % check_every, steps - done)
            for _ in range(k):
                self.step()
            self.time_step += k
            done += k
            self.check_health()

    def check_health(self):
        """NaN / rho <= 0 watchdog (``solver.py:162-172``)."""
        drho = self.f.sum(axis=0)
        bad_nf = ~np.isfinite(drho) & self.fluid
        bad = bad_nf | ((drho <= -1.0) & self.fluid)
        if not bad.any():
            return
        loc = tuple(int(i) for i in np.unravel_index(int(np.argmax(bad)), self.params.shape))
        reason = "non-finite populations" if bad_nf.any() else "non-positive density"
        raise OracleDiverged(self.time_step, loc, reason)

    # ---------------------------------------------------------------- readouts
    def populations(self):
        return np.array(self.f, copy=True)

    def macroscopic(self):
        """rho = 1 + sum f~*, rho u = sum c f* - F/2; solid -> (1, 0) (``diagnostics.py:72-80``)."""
        f = self.f
        force = self.collision_force()
        rho = 1.0 + f.sum(axis=0)
        u = tuple((ja - 0.5 * fa) / rho for ja, fa in zip(_momentum(self.lattice, f), force, strict=True))
        return np.where(self.solid, 1.0, rho), tuple(np.where(self.solid, 0.0, ua) for ua in u)

    def evaluate_affine(self, compiled):
        """const + sum coeff * f[slots] in the state dtype (``link_rules.py:269-272``)."""
        slots = np.asarray(compiled.slots)
        coeff = np.asarray(compiled.coeff).astype(self.cdt)
        const = np.asarray(compiled.constant).astype(self.cdt)
        return (const + (coeff * self.f.reshape(-1)[slots]).sum(axis=1)).astype(np.float64)

    @property
    def immersed_force(self):
        if self.ibm is None:
            raise AttributeError("this simulation has no immersed body")
        return np.asarray(self.ibm.body_force, dtype=np.float64)
