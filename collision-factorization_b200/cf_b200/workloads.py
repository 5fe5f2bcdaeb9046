"""Seeded synthetic inputs for the benchmark configurations.

Every generator takes an explicit seed (numpy ``default_rng``) so that tests, the benchmark and the
fixture scripts see identical cells.  Cell arrays are returned as ``[B, K, N_Q]`` C-ordered float64,
which is the same memory as the reference's column-major ``[N_Q x K x B]``.

* ``maxwellian_cells``  -- a seeded Maxwellian per cell (small drift, temperature near 1) plus a
  perturbation with coefficients N(0,1) * exp(-decay*(k+l)) at a given amplitude (the
  hard-sphere batch configuration).
* ``two_maxwellian_mixture`` -- one f: two Maxwellians with drifts N(0, 0.5^2)^3 and temperatures
  U[0.5, 1.5], renormalised to unit density (the CPU-runnable configuration).
* ``bimaxwellian_cells`` -- anisotropic bi-Maxwellians, T_par/T_perp ~ U[0.5, 2] (precision form).
* ``stress_cells``  -- Maxwellian plus a seeded L=2 stress perturbation (implicit relaxation),
  generalising tutorial_stress_relaxation.m:63-65.
* ``synthetic_R``  -- a seeded stand-in for the reduced radial tensor with the reference's
  conservation rows zeroed, for resolutions where the reference's CPU quadrature
  (compute_rtensor_sumfac_mex) is too slow to run.
"""
from __future__ import annotations

import math

import numpy as np

from . import basis


def _grid_for(L: int):
    n_ang = max(2 * L + 4, 16)
    return basis.product_grid(n_rad=40, n_pol=n_ang, n_azi=n_ang)


def project_maxwellians(K: int, L: int, drifts: np.ndarray, temps: np.ndarray, densities=None) -> np.ndarray:
    """Coefficients [n, K, N_Q] of Maxwellians with the given drifts [n x 3] and temperatures [n]."""
    grid = _grid_for(L)
    Psi = basis.evaluate(K, L, grid.v)
    n = drifts.shape[0]
    dens = np.ones(n) if densities is None else np.asarray(densities, dtype=np.float64)
    F = np.stack([basis.maxwellian_F(grid.v, dens[i], drifts[i], temps[i]) for i in range(n)], axis=1)
    c = basis.project(K, L, F, grid, Psi)  # [NQ, K, n]
    return np.ascontiguousarray(c.transpose(2, 1, 0))


def perturbation(K: int, L: int, B: int, rng: np.random.Generator, amplitude: float, decay: float) -> np.ndarray:
    NQ = basis.n_q(L)
    l_of_q = basis.q_to_l(np.arange(1, NQ + 1))
    k = np.arange(K)[:, None]
    w = np.exp(-decay * (k + l_of_q[None, :]))  # [K, NQ]
    return amplitude * rng.standard_normal((B, K, NQ)) * w[None]


def maxwellian_cells(K: int, L: int, B: int, seed: int, amplitude: float = 1e-2, decay: float = 0.6,
                     drift_sd: float = 0.1, t_range=(0.9, 1.1), n_base: int = 32) -> np.ndarray:
    """[B, K, N_Q]: seeded Maxwellian (one of n_base) + amplitude * N(0,1) exp(-decay (k+l))."""
    rng = np.random.default_rng(seed)
    nb = min(n_base, B) if B > 0 else 0
    drifts = rng.normal(0.0, drift_sd, size=(nb, 3))
    temps = rng.uniform(t_range[0], t_range[1], size=nb)
    base = project_maxwellians(K, L, drifts, temps) if nb else np.zeros((0, K, basis.n_q(L)))
    which = rng.integers(0, max(nb, 1), size=B)
    cells = base[which] if nb else np.zeros((0, K, basis.n_q(L)))
    return np.ascontiguousarray(cells + perturbation(K, L, B, rng, amplitude, decay))


def two_maxwellian_mixture(K: int, L: int, seed: int) -> np.ndarray:
    """[K, N_Q] coefficients of 0.5 M(u1,T1) + 0.5 M(u2,T2), renormalised to unit density."""
    rng = np.random.default_rng(seed)
    drifts = rng.normal(0.0, 0.5, size=(2, 3))
    temps = rng.uniform(0.5, 1.5, size=2)
    c = project_maxwellians(K, L, drifts, temps, densities=[0.5, 0.5])
    f = c.sum(axis=0)
    # unit density: scale so the mass coefficient equals that of a unit-density Maxwellian
    unit = project_maxwellians(K, L, np.zeros((1, 3)), np.ones(1))[0]
    return np.ascontiguousarray(f * (unit[0, 0] / f[0, 0]))


def project_axisymmetric(K: int, L: int, F_of, n_rad: int = 48, n_pol: int | None = None) -> np.ndarray:
    """[K, N_Q] coefficients of an axisymmetric F(r, cos theta) (only m = 0 modes are nonzero)."""
    from . import quadrature

    n_pol = n_pol or max(2 * L + 8, 24)
    rad = quadrature.generalized_laguerre(n_rad, 0.5)
    r = np.sqrt(rad.x)
    w_rad = rad.w / 2.0
    pol = quadrature.legendre(n_pol, -1.0, 1.0)
    R, CT = np.meshgrid(r, pol.x, indexing="ij")
    W = (w_rad[:, None] * pol.w[None, :] * 2.0 * math.pi).ravel()
    Fv = F_of(R.ravel(), CT.ravel())
    P = basis.assoc_legendre_all(L, CT.ravel())
    NQ = basis.n_q(L)
    out = np.zeros((K, NQ))
    rr = R.ravel()
    for l in range(L + 1):
        q = basis.q_index(l, 0) - 1
        Y = math.sqrt((2 * l + 1) / (4.0 * math.pi)) * P[l, 0]
        for k in range(K):
            phi = basis.radial_norm(k, l) * basis.laguerre(k, l + 0.5, rr * rr) * rr**l * Y
            out[k, q] = np.sum(W * Fv * phi)
    return out


def bimaxwellian_cells(K: int, L: int, B: int, seed: int, n_base: int = 32) -> np.ndarray:
    """[B, K, N_Q] projections of bi-Maxwellians with T_par/T_perp ~ U[0.5, 2] (energy kept at 3/2)."""
    rng = np.random.default_rng(seed)
    nb = min(n_base, max(B, 1))
    ratios = rng.uniform(0.5, 2.0, size=nb)
    base = []
    for a in ratios:
        t_perp = 3.0 / (2.0 + a)  # 2 T_perp + T_par = 3 (unit temperature)
        t_par = a * t_perp

        def F(r, ct, t_par=t_par, t_perp=t_perp):
            vz2 = (r * ct) ** 2
            vp2 = r * r - vz2
            return math.pi**-1.5 / (t_perp * math.sqrt(t_par)) * np.exp(-vp2 / t_perp - vz2 / t_par + r * r)

        base.append(project_axisymmetric(K, L, F))
    base = np.stack(base)
    which = rng.integers(0, nb, size=B)
    return np.ascontiguousarray(base[which])


def stress_cells(K: int, L: int, B: int, seed: int, amplitude: float = 0.1) -> np.ndarray:
    """[B, K, N_Q]: absolute Maxwellian c[0,0] = 1 plus a seeded L=2 stress (all five m) of the given size.

    tutorial_stress_relaxation.m:63-65 sets c_eq(1) = 1 and one L=2, m=0 coefficient to 0.1; here the
    five L=2, k=0 coefficients of each cell are amplitude * N(0,1)/sqrt(5).
    """
    rng = np.random.default_rng(seed)
    NQ = basis.n_q(L)
    c = np.zeros((B, K, NQ))
    c[:, 0, 0] = 1.0
    if L >= 2:
        c[:, 0, 4:9] = amplitude * rng.standard_normal((B, 5)) / math.sqrt(5.0)
    return c


def synthetic_R(l_triplets: np.ndarray, K: int, seed: int, scale: float = 1.0, decay: float = 0.35) -> np.ndarray:
    """Seeded [K x K x K x N_L] (Fortran order) with the conservation rows of
    src/GeneralCollisionTensor.m:184-191 zeroed (k1 = 0, 1 when l1 = 0; k1 = 0 when l1 = 1)."""
    rng = np.random.default_rng(seed)
    N_L = l_triplets.shape[0]
    k = np.arange(K)
    w = np.exp(-decay * (k[:, None, None] + k[None, :, None] + k[None, None, :]))
    R = scale * rng.standard_normal((K, K, K, N_L)) * w[..., None]
    for t in range(N_L):
        l1 = int(l_triplets[t, 0])
        if l1 == 0:
            R[: min(2, K), :, :, t] = 0.0
        elif l1 == 1:
            R[0, :, :, t] = 0.0
    return np.asfortranarray(R)


RAGGED_BUCKETS = ((4, 4), (6, 6), (8, 6), (10, 8))  # (L, K)
RAGGED_WEIGHTS = (0.4, 0.3, 0.2, 0.1)


def ragged_assignment(B: int, seed: int, weights=RAGGED_WEIGHTS) -> np.ndarray:
    """Bucket index of each of B cells, drawn with the given proportions."""
    rng = np.random.default_rng(seed)
    return rng.choice(len(weights), size=B, p=np.asarray(weights) / np.sum(weights))
