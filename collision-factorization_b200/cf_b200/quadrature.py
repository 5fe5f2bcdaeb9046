"""One-dimensional Gauss rules used to build and project the spectral operator.

Restates the reference's ``Gauss`` class (src/Gauss.m).  These rules produce the
5D quadrature grids that the reduced radial tensor R is computed on
(src/GeneralCollisionTensor.m:67-79) and the 3D grids that seeded Maxwellians are
projected with (tutorial_collisions_spectral_properties.m:101-136).  Each rule
follows the reference's own iteration, so nodes and weights agree with it to
rounding.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

_EPS = np.finfo(np.float64).eps


@dataclass
class Rule:
    x: np.ndarray
    w: np.ndarray


def legendre(n: int, a: float = -1.0, b: float = 1.0, include_boundaries: bool = False) -> Rule:
    """Gauss-Legendre rule with ``n`` nodes on [a, b].

    Newton iteration on the Legendre three-term recurrence from the
    Chebyshev-like initial guess, as in src/Gauss.m:38-105.
    """
    if n < 1:
        raise ValueError("legendre: need at least one node")
    nn = n - 1
    n1, n2 = nn + 1, nn + 2
    xu = np.linspace(-1.0, 1.0, n1) if n1 > 1 else np.array([1.0])
    y = np.cos((2.0 * np.arange(nn + 1) + 1.0) * math.pi / (2 * nn + 2)) + (0.27 / n1) * np.sin(
        math.pi * xu * nn / n2
    )
    y0 = np.full_like(y, 2.0)
    lp = np.zeros_like(y)
    for _ in range(200):
        if not np.max(np.abs(y - y0)) > _EPS:
            break
        lcol_prev = np.ones_like(y)  # L(:,1)
        lcol = y.copy()  # L(:,2)
        for k in range(2, n1 + 1):
            lnext = ((2 * k - 1) * y * lcol - (k - 1) * lcol_prev) / k
            lcol_prev, lcol = lcol, lnext
        # lcol is L(:,N2), lcol_prev is L(:,N1)
        lp = n2 * (lcol_prev - y * lcol) / (1.0 - y**2)
        y0 = y
        y = y0 - lcol / lp
    x = np.flipud((a * (1.0 - y) + b * (1.0 + y)) / 2.0)
    w = np.flipud((b - a) / ((1.0 - y**2) * lp**2) * (n2 / n1) ** 2)
    if include_boundaries:
        x = np.concatenate(([a], x, [b]))
        w = np.concatenate(([0.0], w, [0.0]))
    return Rule(x, w)


def lobatto(n: int, a: float = -1.0, b: float = 1.0) -> Rule:
    """Gauss-Lobatto-Legendre rule with ``n`` nodes on [a, b] (src/Gauss.m:7-36)."""
    if n < 2:
        raise ValueError("lobatto: need at least two nodes")
    n1 = n
    nn = n - 1
    x = np.cos(math.pi * np.arange(nn + 1) / nn)
    xold = np.full_like(x, 2.0)
    P = np.zeros((n1, n1))
    for _ in range(200):
        if not np.max(np.abs(x - xold)) > _EPS:
            break
        xold = x
        P[:, 0] = 1.0
        P[:, 1] = x
        for k in range(2, nn + 1):
            P[:, k] = ((2 * k - 1) * x * P[:, k - 1] - (k - 1) * P[:, k - 2]) / k
        x = xold - (x * P[:, n1 - 1] - P[:, nn - 1]) / (n1 * P[:, n1 - 1])
    xs = np.flipud((a * (1.0 - x) + b * (1.0 + x)) / 2.0)
    w = (b - a) / (nn * n1 * P[:, n1 - 1] ** 2)
    return Rule(xs, w)


def generalized_laguerre(n: int, alpha: float = 0.0) -> Rule:
    """Generalised Gauss-Laguerre rule for x^alpha e^-x on [0, inf).

    Golub-Welsch eigenvalues as initial roots, up to 15 Newton polishing steps on
    the three-term recurrence and weights from the derivative, as in
    src/Gauss.m:128-173 (the weights use the derivative evaluated before the last
    Newton update, exactly like the reference).
    """
    if n < 1:
        raise ValueError("generalized_laguerre: need at least one node")
    i = np.arange(1, n + 1, dtype=np.float64)
    diag = 2.0 * i - 1.0 + alpha
    off = np.sqrt(i[: n - 1] * (i[: n - 1] + alpha))
    J = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
    x = np.sort(np.linalg.eigvalsh(J))
    lp1 = -np.ones(n)
    for _ in range(15):
        l0 = np.ones(n)
        l1 = 1.0 + alpha - x
        lp0 = np.zeros(n)
        lp1 = -np.ones(n)
        for k in range(2, n + 1):
            l2 = ((2 * k - 1 + alpha - x) * l1 - (k - 1 + alpha) * l0) / k
            lp2 = ((2 * k - 1 + alpha - x) * lp1 - l1 - (k - 1 + alpha) * lp0) / k
            l0, l1 = l1, l2
            lp0, lp1 = lp1, lp2
        dx = l1 / lp1
        x = x - dx
        if np.max(np.abs(dx)) < 1e-15:
            break
    ln_const = math.lgamma(n + alpha + 1.0) - math.lgamma(n + 1.0)
    w = math.exp(ln_const) / (x * lp1**2)
    return Rule(x, w)


def halfrange_hermite(n: int, beta: float = 1.0) -> Rule:
    """Rule for int_0^inf f(x) x^2 e^{-beta x^2} dx (src/Gauss.m:177-195)."""
    lag = generalized_laguerre(n, 0.5)
    return Rule(np.sqrt(lag.x / beta), lag.w / (2.0 * beta**1.5))
