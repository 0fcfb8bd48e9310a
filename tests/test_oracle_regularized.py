"""The oracle's regularised collision against the defining properties of the published method (CPU).

The reference has no regularised collision, so ``oracle.lbm_oracle.collide_regularized``
(projective regularisation, Latt & Chopard 2006, with Guo forcing) is pinned
here by what defines it, on random states of D2Q9 and D3Q19 in float64:

* it conserves mass, and changes momentum by exactly the force;
* a non-equilibrium part that lies in the second-order Hermite space passes
  unchanged, so the update equals BGK's;
* any non-equilibrium content outside that space (a "ghost" moment orthogonal
  to the Hermite polynomials up to second order) leaves no trace.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.lbm_oracle import _momentum, collide, collide_regularized, equilibrium

import lbm_b200 as lbm

SHAPE = (5, 6, 7)


def random_moments(lattice, rng):
    shape = SHAPE[-lattice.d:]
    drho = 0.02 * rng.standard_normal(shape)
    u = tuple(0.05 * rng.standard_normal(shape) for _ in range(lattice.d))
    return drho, u


def hermite2(lattice, pi):
    """w_i 4.5 (c_i c_i - I/3) : pi for a symmetric field pi[a][b]."""
    c = np.asarray(lattice.c, dtype=np.float64)
    out = []
    for i, wi in enumerate(lattice.w):
        v = sum((c[i, a] * c[i, b] - (a == b) / 3.0) * pi[a][b] for a in range(lattice.d) for b in range(lattice.d))
        out.append(4.5 * wi * v)
    return np.stack(out)


def ghost(lattice, amp):
    """A population pattern orthogonal (sum over i, unweighted) to 1, c_i and c_i c_i: no mass,
    momentum or stress, i.e. no content in the Hermite space up to second order."""
    c = np.asarray(lattice.c, dtype=np.float64)
    basis = [np.ones(lattice.q)] + [c[:, a] for a in range(lattice.d)]
    basis += [c[:, a] * c[:, b] for a in range(lattice.d) for b in range(a, lattice.d)]
    m = np.stack(basis, axis=1)
    rng = np.random.default_rng(7)
    v = rng.standard_normal(lattice.q)
    v -= m @ np.linalg.lstsq(m, v, rcond=None)[0]
    assert np.abs(m.T @ v).max() < 1e-12
    return v.reshape(-1, *([1] * lattice.d)) * amp


@pytest.mark.parametrize("lattice", [lbm.D2Q9, lbm.D3Q19])
@pytest.mark.parametrize("forced", [False, True])
def test_mass_and_momentum(lattice, forced):
    rng = np.random.default_rng(1)
    drho, u = random_moments(lattice, rng)
    f = equilibrium(lattice, drho, u) + 1e-3 * rng.standard_normal((lattice.q, *drho.shape))
    force = tuple(1e-4 * rng.standard_normal(drho.shape) for _ in range(lattice.d)) if forced else (0.0,) * lattice.d
    post = collide_regularized(lattice, f, 1 / 0.7, force)
    np.testing.assert_allclose(post.sum(axis=0), f.sum(axis=0), rtol=0, atol=1e-15)
    for a, (j0, j1) in enumerate(zip(_momentum(lattice, f), _momentum(lattice, post), strict=True)):
        np.testing.assert_allclose(j1, j0 + force[a], rtol=0, atol=1e-15)


@pytest.mark.parametrize("lattice", [lbm.D2Q9, lbm.D3Q19])
def test_second_order_non_equilibrium_relaxes_like_bgk(lattice):
    rng = np.random.default_rng(2)
    drho, u = random_moments(lattice, rng)
    d = lattice.d
    pi = [[None] * d for _ in range(d)]
    for a in range(d):
        for b in range(a, d):
            pi[a][b] = pi[b][a] = 1e-3 * rng.standard_normal(drho.shape)
    f = equilibrium(lattice, drho, u) + hermite2(lattice, pi)
    force = (0.0,) * d
    wp = 1 / 0.62
    np.testing.assert_allclose(collide_regularized(lattice, f, wp, force), collide(lattice, f, wp, wp, force),
                               rtol=0, atol=1e-15)


@pytest.mark.parametrize("lattice", [lbm.D2Q9, lbm.D3Q19])
def test_higher_order_non_equilibrium_is_filtered(lattice):
    rng = np.random.default_rng(3)
    drho, u = random_moments(lattice, rng)
    feq = equilibrium(lattice, drho, u)
    force = tuple(1e-4 * rng.standard_normal(drho.shape) for _ in range(lattice.d))
    wp = 1 / 0.55
    clean = collide_regularized(lattice, feq, wp, force)
    noisy = collide_regularized(lattice, feq + ghost(lattice, 1e-3), wp, force)
    np.testing.assert_allclose(noisy, clean, rtol=0, atol=1e-15)
    # BGK keeps a (1 - wp) share of the same ghost content
    assert np.abs(collide(lattice, feq + ghost(lattice, 1e-3), wp, wp, force) - collide(lattice, feq, wp, wp, force)).max() > 1e-5
