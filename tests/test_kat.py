"""Known-answer tests of the operator the path contracts (CPU, oracle side).

The reference prints these in its tutorials without asserting them; here they are asserted on the
operators whose R comes from the reference's own quadrature MEX (tests/golden/op_*.npz):

* Wang Chang-Uhlenbeck spectrum (tests/TestWCUEigenvalues.m, AbsTol 1e-10);
* H-theorem: exactly 5 zero eigenvalues and none positive (tutorial_collisions_spectral_properties.m:53-64);
* Galilean invariance of the 5 invariant entries of Q for shifted Maxwellians (:96-183, < 1e-12);
* Chapman-Enskog bracket matrix and viscosity factors (tutorial_chapman_enscog_decay_rates.m:46-91);
* BKW transient against the analytic solution (tutorial_collisions_bwu_solution.m:47-104);
* conservation during nonlinear stress relaxation (tutorial_stress_relaxation.m:77-91,162-168).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_op


def dense_of(name):
    from cf_b200.geometry import Geometry
    from oracle import rtensor

    d = load_op(name)
    geo = Geometry(d["L"], d["labels"], d["vals"], d["ic_map"], d["l_triplets"])
    return d, rtensor.assemble_dense(geo, d["R"], d["K"])


def wcu_spectrum(K_max: int, L_max: int) -> np.ndarray:
    """Analytic Maxwell-molecule spectrum (tests/TestWCUEigenvalues.m:101-147)."""
    from cf_b200 import basis, quadrature

    qr = quadrature.legendre(200, -1.0, 1.0)
    c = np.sqrt((1 + qr.x) / 2)
    s = np.sqrt((1 - qr.x) / 2)
    lam = []
    for l in range(L_max + 1):
        Pc = basis.assoc_legendre_all(l, c)[l, 0]
        Ps = basis.assoc_legendre_all(l, s)[l, 0]
        for k in range(K_max + 1):
            val = 2 * math.pi * np.sum(qr.w * (c ** (2 * k + l) * Pc + s ** (2 * k + l) * Ps - 1))
            if (k, l) in ((0, 0), (0, 1), (1, 0)):
                val = 0.0
            lam += [val] * (2 * l + 1)
    return np.sort(np.array(lam))[::-1]


def test_wcu_eigenvalues():
    d, Cd = dense_of("wcu_k2_l2_g0")
    J = Cd[:, :, 0] + Cd[:, 0, :]
    lam = np.sort(np.linalg.eigvals(J).real)[::-1]
    lam = lam / abs(lam[5])
    ref = wcu_spectrum(2, 2)
    ref = ref / abs(ref[5])
    assert np.max(np.abs(lam[:5])) < 1e-10
    assert np.max(np.abs(lam - ref)) < 1e-10


def test_h_theorem_five_zero_modes_none_positive():
    for name in ("wcu_k2_l2_g0", "hs_k4_l4_g1"):
        d, Cd = dense_of(name)
        J = Cd[:, :, 0] + Cd[:, 0, :]
        lam = np.linalg.eigvals(J).real
        lam = lam / np.sort(np.abs(lam))[5]
        assert np.sum(np.abs(lam) < 1e-10) == 5, name
        assert np.sum(lam > 1e-10) == 0, name


def test_galilean_invariance_of_invariants():
    """Shifted Maxwellians U in {0, 0.1, 0.3, 0.6}: the 5 invariant entries of Q vanish (< 1e-12)."""
    from cf_b200 import basis
    from oracle.reference import Oracle

    d = load_op("hs_k4_l4_g1")
    K, L, NQ = d["K"], d["L"], d["NQ"]
    grid = basis.product_grid(60, 30, 30)
    Psi = basis.evaluate(K, L, grid.v)
    orc = Oracle()
    inv = basis.invariant_indices(NQ)
    for U in (0.0, 0.1, 0.3, 0.6):
        F = basis.maxwellian_F(grid.v, 1.0, [U, 0.0, 0.0], 1.0)
        f = np.asfortranarray(basis.project(K, L, F, grid, Psi))
        Q = np.zeros((NQ, K), order="F")
        orc.af(Q, f, d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
        assert np.max(np.abs(Q.ravel(order="F")[inv])) < 1e-12
        if U == 0.0:
            assert np.max(np.abs(Q)) < 1e-12  # the Maxwellian is an equilibrium


def test_chapman_enskog_bracket_matrix_and_viscosity():
    """Hard spheres, K_max = 4, L = 4: the L = 2 block of J_eq is the Chapman-Cowling bracket matrix."""
    d, Cd = dense_of("hs_k4_l4_g1")
    K, NQ = d["K"], d["NQ"]
    J = Cd[:, :, 0] + Cd[:, 0, :]
    idx = np.arange(K) * NQ + 6  # q = 7 (l = 2, m = 0)
    H = J[np.ix_(idx, idx)]
    H = H / H[0, 0]
    # orthonormal Laguerre basis vs the Sonine normalisation: D = diag(1, -sqrt(2/7))
    D = np.diag([1.0, -math.sqrt(2.0 / 7.0)])
    H_ana = D @ np.array([[1.0, 0.25], [0.25, 205.0 / 48.0]]) @ D
    assert np.max(np.abs(H[:2, :2] - H_ana)) < 1e-10
    f_mu = [np.linalg.inv(H[:k, :k])[0, 0] for k in range(1, K + 1)]
    assert abs(f_mu[0] - 1.0) < 1e-14
    assert abs(f_mu[1] - 205.0 / 202.0) < 1e-10
    assert all(b > a for a, b in zip(f_mu, f_mu[1:]))
    assert abs(f_mu[-1] - 1.016034) < 1e-5


def project_bkw(alpha: float, K: int, L: int) -> np.ndarray:
    """Isotropic projection of the BKW solution (tutorial_collisions_bwu_solution.m:237-269)."""
    from cf_b200 import basis, quadrature

    NQ = basis.n_q(L)
    qr = quadrature.generalized_laguerre(80, 0.5)
    c = np.zeros(K * NQ)
    v = np.stack([np.sqrt(qr.x), np.zeros_like(qr.x), np.zeros_like(qr.x)], axis=1)
    Psi = basis.evaluate(K, L, v)
    a = alpha
    F = math.pi**-1.5 * (1 - a) ** -1.5 * np.exp(-qr.x * a / (1 - a)) * (1 + (a / (1 - a)) * (qr.x / (1 - a) - 1.5))
    step = (2 * math.pi * qr.w * F)[:, None] * Psi
    for k in range(K):
        c[k * NQ] = np.sum(step[:, k * NQ])
    return c


def test_bkw_transient():
    """RK2 from alpha_0 = 0.25 to t = 4/mu tracks alpha(t) = alpha_0 e^{-mu t / 2}."""
    d, Cd = dense_of("bkw_k5_l1_g0")
    K, L, NQ = d["K"], d["L"], d["NQ"]
    N = K * NQ
    Cf = Cd.reshape(N, N * N, order="F")
    ceq = project_bkw(0.0, K, L)
    Jeq = Cd[:, :, 0] * ceq[0] + Cd[:, 0, :] * ceq[0]
    mu = abs(Jeq[2 * NQ, 2 * NQ])
    assert abs(mu - 4.0 * math.pi / 3.0) < 1e-10
    a0 = 0.25
    c = project_bkw(a0, K, L)
    dt = 0.001 / mu
    for i in range(4000):
        q1 = Cf @ np.outer(c, c).ravel(order="F")
        ct = c + dt * q1
        q2 = Cf @ np.outer(ct, ct).ravel(order="F")
        c = c + 0.5 * dt * (q1 + q2)
        if (i + 1) % 1000 == 0:
            ca = project_bkw(a0 * math.exp(-mu / 2 * (i + 1) * dt), K, L)
            assert np.max(np.abs(c - ca)) / np.max(np.abs(ca)) < 1e-7
    inv = basis_inv(NQ)
    assert np.max(np.abs(c[inv] - project_bkw(a0, K, L)[inv])) < 1e-13


def basis_inv(NQ):
    from cf_b200 import basis

    return basis.invariant_indices(NQ)


def test_stress_relaxation_conserves_invariants():
    """Hard spheres K_max = 4, L = 4: c_eq + 0.1 at (k=0, q=7), RK2 for 200 steps of 0.005/mu."""
    d, Cd = dense_of("hs_k4_l4_g1")
    K, NQ = d["K"], d["NQ"]
    N = K * NQ
    Cf = Cd.reshape(N, N * N, order="F")
    J = Cd[:, :, 0] + Cd[:, 0, :]
    mu = abs(J[6, 6])
    c = np.zeros(N)
    c[0] = 1.0
    c[6] = 0.1
    c0 = c.copy()
    dt = 0.005 / mu
    for _ in range(200):
        q1 = Cf @ np.outer(c, c).ravel(order="F")
        ct = c + dt * q1
        q2 = Cf @ np.outer(ct, ct).ravel(order="F")
        c = c + 0.5 * dt * (q1 + q2)
    inv = basis_inv(NQ)
    assert np.max(np.abs(c[inv] - c0[inv])) < 1e-13
    assert abs(c[6]) < 0.1 * math.exp(-0.5)  # the stress has relaxed past e^-1/2 by t = 1/mu
