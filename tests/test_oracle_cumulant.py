"""The oracle's cumulant collision against the defining properties of the published method (CPU).

The reference has no cumulant collision, so ``oracle.lbm_oracle.collide_cumulant``
(the cumulant method of Geier et al. 2015 on D2Q9) is pinned here by what
defines it, on random D2Q9 states in float64:

* the chimera transformation gives the central moments sum_i f_i (c_ix - u_x)^m
  (c_iy - u_y)^n, and its inverse undoes it;
* mass is conserved and momentum changes by exactly the force;
* after the collision, about u = (j + F/2)/rho: the shear moments k20 - k02 and
  k11 are (1 - w) times their values before, k20 + k02 = 2 rho/3, the
  third-order moments vanish (no force) and so does the fourth-order cumulant;
* the product-form equilibrium rho W(u_x) W(u_y) is a fixed point;
* a Taylor-Green vortex decays at the lattice viscosity (1/w - 1/2)/3.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import OracleSolver
from oracle.lbm_oracle import _chimera, _chimera_inverse, _momentum, collide_cumulant, equilibrium

import lbm_b200 as lbm

SHAPE = (6, 7)
L = lbm.D2Q9


def random_state(rng, amp=1e-3):
    drho = 0.02 * rng.standard_normal(SHAPE)
    u = tuple(0.05 * rng.standard_normal(SHAPE) for _ in range(2))
    return equilibrium(L, drho, u) + amp * rng.standard_normal((9, *SHAPE))


def central_moment(f, u, m, n):
    """sum_i f_i (c_ix - u_x)^m (c_iy - u_y)^n of full populations f."""
    return sum(f[i] * (c[0] - u[0]) ** m * (c[1] - u[1]) ** n for i, c in enumerate(L.c))


def full(f_shifted):
    return f_shifted + np.asarray(L.w).reshape(-1, 1, 1)


def test_chimera_round_trip():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((3, 50))
    u = 0.1 * rng.standard_normal(50)
    k = _chimera(a[0], a[1], a[2], u)
    back = _chimera_inverse(*k, u)
    np.testing.assert_allclose(np.stack(back), a, rtol=0, atol=1e-14)
    # (c - u)^m moments of the three populations
    for m in range(3):
        want = sum(a[i] * (c - u) ** m for i, c in enumerate((-1, 0, 1)))
        np.testing.assert_allclose(k[m], want, rtol=0, atol=1e-14)


@pytest.mark.parametrize("forced", [False, True])
def test_mass_and_momentum(forced):
    rng = np.random.default_rng(1)
    f = random_state(rng)
    force = tuple(1e-4 * rng.standard_normal(SHAPE) for _ in range(2)) if forced else (0.0, 0.0)
    post = collide_cumulant(L, f, 1 / 0.7, force)
    np.testing.assert_allclose(post.sum(axis=0), f.sum(axis=0), rtol=0, atol=1e-15)
    for a, (j0, j1) in enumerate(zip(_momentum(L, f), _momentum(L, post), strict=True)):
        np.testing.assert_allclose(j1, j0 + force[a], rtol=0, atol=1e-15)


def test_moments_after_the_collision():
    rng = np.random.default_rng(2)
    f = random_state(rng, amp=3e-3)
    w = 1 / 0.58
    post = collide_cumulant(L, f, w, (0.0, 0.0))
    rho = 1.0 + f.sum(axis=0)
    u = tuple(j / rho for j in _momentum(L, f))
    pre_full, post_full = full(f), full(post)
    km = {mn: central_moment(pre_full, u, *mn) for mn in ((2, 0), (0, 2), (1, 1))}
    kp = {mn: central_moment(post_full, u, *mn) for mn in ((2, 0), (0, 2), (1, 1), (2, 1), (1, 2), (2, 2))}
    tol = dict(rtol=0, atol=2e-15)
    np.testing.assert_allclose(kp[2, 0] - kp[0, 2], (1 - w) * (km[2, 0] - km[0, 2]), **tol)
    np.testing.assert_allclose(kp[1, 1], (1 - w) * km[1, 1], **tol)
    np.testing.assert_allclose(kp[2, 0] + kp[0, 2], 2 * rho / 3, **tol)
    np.testing.assert_allclose(kp[2, 1], 0.0, **tol)
    np.testing.assert_allclose(kp[1, 2], 0.0, **tol)
    c22 = kp[2, 2] / rho - (kp[2, 0] * kp[0, 2] + 2 * kp[1, 1] ** 2) / rho**2
    np.testing.assert_allclose(c22, 0.0, **tol)
    # BGK would keep a (1 - w) share of the third-order moments
    assert np.abs(central_moment(pre_full, u, 2, 1)).max() > 1e-4


def test_product_equilibrium_is_a_fixed_point():
    rng = np.random.default_rng(3)
    rho = 1.0 + 0.02 * rng.standard_normal(SHAPE)
    u = [0.05 * rng.standard_normal(SHAPE) for _ in range(2)]

    def weight(c, v):  # one-dimensional equilibrium factor, c = -1, 0, 1
        return (2.0 / 3.0 - v * v) if c == 0 else 0.5 * (1.0 / 3.0 + v * v + c * v)

    feq = np.stack([rho * weight(c[0], u[0]) * weight(c[1], u[1]) for c in L.c]) - np.asarray(L.w).reshape(-1, 1, 1)
    np.testing.assert_allclose(collide_cumulant(L, feq, 1 / 0.53, (0.0, 0.0)), feq, rtol=0, atol=1e-15)


def test_taylor_green_decays_at_the_lattice_viscosity():
    """Within the O(k^2) discretisation error of the lattice (0.11 % at 64^2, as BGK's 0.13 %)."""
    n, tau, u0, steps = 64, 0.8, 0.01, 400
    params = lbm.SimulationParams(nx=n, ny=n, tau=tau, collision="cumulant", dtype="float64")
    k = 2 * np.pi / n
    x = np.arange(n)
    X, Y = np.meshgrid(x, x)
    ux = u0 * np.sin(k * X) * np.cos(k * Y)
    uy = -u0 * np.cos(k * X) * np.sin(k * Y)
    s = OracleSolver(params)
    s.initialize(1.0, ux, uy)
    for _ in range(steps):
        s.step()
    _, u = s.macroscopic()
    amp = float(np.sum(u[0] * ux) / np.sum(ux * ux))
    exact = np.exp(-2 * params.viscosity * k * k * steps)
    assert abs(amp - exact) < 2e-3 * exact, (amp, exact)


def test_params_take_the_cumulant_model_on_d2q9_only():
    assert lbm.SimulationParams(nx=4, ny=4, tau=0.8, collision="cumulant").relaxation_rates == (1.25, 1.25)
    with pytest.raises(ValueError, match="cumulant collision is built for D2Q9"):
        lbm.SimulationParams(nx=4, ny=4, nz=4, tau=0.8, collision="cumulant")
