"""Spectral basis conventions and projections of velocity distributions.

Restates the reference's basis (src/SpectralBasis.m, src/SphericalHarmonics.m):

    phi_{k,l,m}(v) = N_kl * L_k^{(l+1/2)}(|v|^2) * |v|^l * Y_lm(v_hat)

with real spherical harmonics Y_lm (Condon-Shortley phase; m>0 -> cos, m<0 -> sin;
src/SphericalHarmonics.m:15-50), the angular index ``q = l^2 + l + m + 1``
(1-based; src/SphericalHarmonics.m:57) and the global coefficient index
``k*N_Q + q`` (src/SpectralBasis.m:54).  A cell's coefficient vector is stored
column-major as ``[N_Q x K]``: element (q, k) at ``(q-1) + k*N_Q``.

The coefficients of a distribution f(v) are those of ``f(v) / e^{-|v|^2}``
(tutorial_collisions_spectral_properties.m:156-158), obtained with a 3D product
quadrature (generalised Laguerre x Gauss-Legendre x uniform azimuth,
tutorial_collisions_spectral_properties.m:101-136).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import quadrature


def n_q(L: int) -> int:
    return (L + 1) ** 2


def q_index(l: int, m: int) -> int:
    """1-based angular index q for (l, m)."""
    return l * l + l + m + 1


def q_to_l(q):
    """Degree l of a 1-based angular index (the reference's floor(sqrt(q-1)))."""
    return np.floor(np.sqrt(np.asarray(q, dtype=np.float64) - 1.0)).astype(np.int64)


def radial_norm(k: int, l: int) -> float:
    """Orthonormalisation N_kl = (0.5 Gamma(k+l+3/2)/k!)^{-1/2} (src/SpectralBasis.m:44-52)."""
    al = l + 0.5
    ln_mii = -math.log(2.0) + math.lgamma(k + al + 1.0) - math.lgamma(k + 1.0)
    return math.exp(-0.5 * ln_mii)


def laguerre(k: int, alpha: float, x: np.ndarray) -> np.ndarray:
    """Generalised Laguerre L_k^{(alpha)}(x) by the recurrence of src/SpectralBasis.m:143-162."""
    x = np.asarray(x, dtype=np.float64)
    if k == 0:
        return np.ones_like(x)
    prev2 = np.ones_like(x)
    prev1 = 1.0 + alpha - x
    if k == 1:
        return prev1
    val = prev1
    for i in range(1, k):
        val = ((2 * i + 1 + alpha - x) * prev1 - (i + alpha) * prev2) / (i + 1)
        prev2, prev1 = prev1, val
    return val


def assoc_legendre_all(L: int, x: np.ndarray) -> np.ndarray:
    """P_l^m(x) with the Condon-Shortley phase for 0 <= m <= l <= L.

    Returns an array of shape [L+1, L+1, len(x)] indexed [l, m].  This is the
    function MATLAB's ``legendre(l, x)`` returns row by row (used by
    src/SphericalHarmonics.m:25); the recurrences are the standard ones (also used
    by src/mex/compute_rtensor_sumfac_mex.cpp:36-55).
    """
    x = np.asarray(x, dtype=np.float64)
    P = np.zeros((L + 1, L + 1) + x.shape)
    somx2 = np.sqrt(np.maximum((1.0 - x) * (1.0 + x), 0.0))
    pmm = np.ones_like(x)
    fact = 1.0
    for m in range(L + 1):
        if m > 0:
            pmm = pmm * (-fact * somx2)
            fact += 2.0
        P[m, m] = pmm
        if m + 1 <= L:
            P[m + 1, m] = x * (2 * m + 1) * pmm
        for ll in range(m + 2, L + 1):
            P[ll, m] = (x * (2 * ll - 1) * P[ll - 1, m] - (ll + m - 1) * P[ll - 2, m]) / (ll - m)
    return P


def sh_norm(l: int, m: int) -> float:
    am = abs(m)
    base = math.sqrt((2 * l + 1) / (4.0 * math.pi) * math.exp(math.lgamma(l - am + 1) - math.lgamma(l + am + 1)))
    return base if m == 0 else math.sqrt(2.0) * base


def real_sh(L: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Real spherical harmonics [N_points x N_Q] (src/SphericalHarmonics.m:15-50)."""
    theta = np.asarray(theta, dtype=np.float64).ravel()
    phi = np.asarray(phi, dtype=np.float64).ravel()
    P = assoc_legendre_all(L, np.cos(theta))
    Y = np.zeros((theta.size, n_q(L)))
    for l in range(L + 1):
        for m in range(-l, l + 1):
            am = abs(m)
            col = q_index(l, m) - 1
            nrm = math.sqrt((2 * l + 1) / (4.0 * math.pi) * math.exp(math.lgamma(l - am + 1) - math.lgamma(l + am + 1)))
            if m > 0:
                Y[:, col] = math.sqrt(2.0) * nrm * P[l, am] * np.cos(am * phi)
            elif m == 0:
                Y[:, col] = nrm * P[l, 0]
            else:
                Y[:, col] = math.sqrt(2.0) * nrm * P[l, am] * np.sin(am * phi)
    return Y


def evaluate(K: int, L: int, v: np.ndarray) -> np.ndarray:
    """Basis values Psi[N_points x K*N_Q] at velocities v [N_points x 3] (src/SpectralBasis.m:25-58)."""
    v = np.asarray(v, dtype=np.float64)
    r2 = np.sum(v * v, axis=1)
    r = np.sqrt(r2) + np.finfo(np.float64).eps
    theta = np.arccos(v[:, 2] / r)
    phi = np.arctan2(v[:, 1], v[:, 0])
    Y = real_sh(L, theta, phi)
    NQ = n_q(L)
    Psi = np.zeros((v.shape[0], K * NQ))
    for l in range(L + 1):
        cols = np.arange(l * l, (l + 1) ** 2)
        solid = (r**l)[:, None] * Y[:, cols]
        for k in range(K):
            Lk = laguerre(k, l + 0.5, r2)
            Psi[:, k * NQ + cols] = radial_norm(k, l) * Lk[:, None] * solid
    return Psi


@dataclass
class Grid3D:
    v: np.ndarray  # [N x 3]
    w: np.ndarray  # [N] weights including the e^{-|v|^2} Laguerre weight


def product_grid(n_rad: int = 60, n_pol: int = 30, n_azi: int = 30) -> Grid3D:
    """Spherical product grid (tutorial_collisions_spectral_properties.m:101-136)."""
    rad = quadrature.generalized_laguerre(n_rad, 0.5)
    r = np.sqrt(rad.x)
    w_rad = rad.w / 2.0
    pol = quadrature.legendre(n_pol, -1.0, 1.0)
    ct = pol.x
    st = np.sqrt(1.0 - ct**2)
    phi = np.linspace(0.0, 2.0 * math.pi, n_azi + 1)[:-1]
    w_azi = 2.0 * math.pi / n_azi
    R, CT, PH = np.meshgrid(r, ct, phi, indexing="ij")
    ST = np.sqrt(1.0 - CT**2)
    v = np.stack([R * ST * np.cos(PH), R * ST * np.sin(PH), R * CT], axis=-1).reshape(-1, 3)
    W = (w_rad[:, None, None] * pol.w[None, :, None] * w_azi * np.ones_like(PH)).reshape(-1)
    return Grid3D(v, W)


def project(K: int, L: int, F: np.ndarray, grid: Grid3D, Psi: np.ndarray | None = None) -> np.ndarray:
    """Coefficients c = Psi^T (W .* F) of F(v) = f(v)/e^{-|v|^2}, returned as [N_Q x K] (column-major q fastest).

    ``F`` may be [N] for one distribution or [N x B] for several.
    """
    if Psi is None:
        Psi = evaluate(K, L, grid.v)
    F = np.asarray(F, dtype=np.float64)
    c = Psi.T @ (grid.w[:, None] * (F if F.ndim == 2 else F[:, None]))
    NQ = n_q(L)
    out = c.reshape(K, NQ, -1).transpose(1, 0, 2)  # [N_Q, K, B]
    return out[..., 0] if F.ndim == 1 else out


def maxwellian_F(v: np.ndarray, density: float, drift, temperature: float) -> np.ndarray:
    """F(v) = f_M(v) / e^{-|v|^2} for a Maxwellian n (pi T)^{-3/2} exp(-|v-u|^2/T).

    With density 1, drift u and T = 1 this is the shifted Maxwellian of
    tutorial_collisions_spectral_properties.m:155-156.
    """
    u = np.asarray(drift, dtype=np.float64).reshape(1, 3)
    d2 = np.sum((v - u) ** 2, axis=1)
    v2 = np.sum(v * v, axis=1)
    return density * (math.pi * temperature) ** -1.5 * np.exp(-d2 / temperature + v2)


def bimaxwellian_F(v: np.ndarray, density: float, t_par: float, t_perp: float) -> np.ndarray:
    """F(v) for a bi-Maxwellian with temperature t_par along z and t_perp across."""
    v2 = np.sum(v * v, axis=1)
    e = -(v[:, 0] ** 2 + v[:, 1] ** 2) / t_perp - v[:, 2] ** 2 / t_par + v2
    return density * math.pi**-1.5 * (t_perp ** -1.0) * (t_par ** -0.5) * np.exp(e)


def invariant_indices(NQ: int) -> np.ndarray:
    """0-based global indices of mass, momentum (3) and energy in the coefficient vector.

    The reference lists them as 1, 2, 3, 4 and N_Q+1
    (tutorial_collisions_spectral_properties.m:139-144).
    """
    return np.array([0, 1, 2, 3, NQ], dtype=np.int64)
