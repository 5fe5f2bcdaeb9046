"""Quadrature rules and basis: ports of the reference's tests/TestQuadraturePolynomialReproduction.m
and tests/TestSpectralBasis.m."""
from __future__ import annotations

import math

import numpy as np
import pytest


@pytest.mark.parametrize("m", range(5))
@pytest.mark.parametrize("kind", ["legendre", "lobatto"])
def test_polynomial_reproduction(m, kind):
    """tests/TestQuadraturePolynomialReproduction.m:13-49: exact to degree 4 on [1.5, 4.5], 1e-12."""
    from cf_b200 import quadrature

    a, b, N = 1.5, 4.5, 5
    qr = quadrature.legendre(N, a, b, include_boundaries=True) if kind == "legendre" else quadrature.lobatto(N, a, b)
    approx = float(np.dot(qr.w, (m + 1) * qr.x**m))
    assert abs(approx - (b ** (m + 1) - a ** (m + 1))) < 1e-12


@pytest.mark.parametrize("m", range(5))
def test_halfrange_hermite_reproduction(m):
    """tests/TestQuadraturePolynomialReproduction.m:51-81 (beta = 1.25, N = 5), 1e-12."""
    from cf_b200 import quadrature

    beta = 1.25
    qr = quadrature.halfrange_hermite(5, beta)
    exact = math.gamma(m + 1.5) / (2 * beta ** (m + 1.5))
    assert abs(exact - float(np.dot(qr.w, qr.x ** (2 * m)))) < 1e-12


@pytest.mark.parametrize("n,alpha", [(5, 0.5), (20, 0.5), (40, 1.0 / 2.0), (31, 0.0)])
def test_generalized_laguerre_against_scipy(n, alpha):
    from scipy.special import roots_genlaguerre

    from cf_b200 import quadrature

    qr = quadrature.generalized_laguerre(n, alpha)
    x, w = roots_genlaguerre(n, alpha)
    assert np.max(np.abs(qr.x - x) / x) < 1e-12
    assert np.max(np.abs(qr.w - w) / np.abs(w).max()) < 1e-12


def test_basis_sizes():
    """tests/TestSpectralBasis.m:7-17"""
    from cf_b200 import basis

    assert basis.n_q(3) == 16 and 3 * basis.n_q(3) == 48


def test_basis_orthonormal():
    """tests/TestSpectralBasis.m:19-89 (K_max=3, L_max=4): the mass matrix is the identity.

    The reference integrates the angles with a Lebedev rule; a Gauss-Legendre x uniform-azimuth
    product rule of the same exactness is used here.  Its assertion is rel. Frobenius < 1e-8."""
    from cf_b200 import basis, quadrature

    K, L = 4, 4
    n_rad = max(15, 2 * 3 + L + 2)
    rad = quadrature.generalized_laguerre(n_rad, 0.5)
    r = np.sqrt(rad.x)
    w_rad = rad.w / 2
    pol = quadrature.legendre(L + 2, -1.0, 1.0)
    n_azi = 2 * L + 2
    phi = 2 * math.pi * np.arange(n_azi) / n_azi
    Rr, CT, PH = np.meshgrid(r, pol.x, phi, indexing="ij")
    ST = np.sqrt(1 - CT**2)
    v = np.stack([Rr * ST * np.cos(PH), Rr * ST * np.sin(PH), Rr * CT], -1).reshape(-1, 3)
    W = (w_rad[:, None, None] * pol.w[None, :, None] * (2 * math.pi / n_azi) * np.ones_like(PH)).ravel()
    Psi = basis.evaluate(K, L, v)
    M = Psi.T @ (W[:, None] * Psi)
    off = M - np.diag(np.diag(M))
    assert np.linalg.norm(off) / np.linalg.norm(np.diag(M)) < 1e-8
    assert np.max(np.abs(M - np.eye(M.shape[0]))) < 1e-11


def test_real_sh_matches_scipy():
    from scipy.special import sph_harm_y

    from cf_b200 import basis

    rng = np.random.default_rng(0)
    th = rng.uniform(0, math.pi, 50)
    ph = rng.uniform(0, 2 * math.pi, 50)
    L = 6
    Y = basis.real_sh(L, th, ph)
    for l in range(L + 1):
        for m in range(-l, l + 1):
            c = sph_harm_y(l, abs(m), th, ph)  # includes the Condon-Shortley phase
            if m > 0:
                ref = math.sqrt(2) * c.real
            elif m < 0:
                ref = math.sqrt(2) * c.imag
            else:
                ref = c.real
            assert np.max(np.abs(Y[:, basis.q_index(l, m) - 1] - ref)) < 1e-12
