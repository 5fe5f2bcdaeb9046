"""The reference's spectral known answers on the GPU operator.

J_eq = dQ/df at the absolute Maxwellian is assembled column by column from the library's batched
J.v (one cell per unit vector), then checked like the reference's own tests check its dense tensor:
the Maxwell-molecule spectrum (tests/TestWCUEigenvalues.m:30-60), the five zero modes and no
positive eigenvalue, and the Chapman-Enskog bracket matrix of the l = 2 block
(tutorial_chapman_enscog_decay_rates.m:42-58).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_op
from test_kat import wcu_spectrum

pytestmark = pytest.mark.gpu


def _jeq_gpu(name: str):
    """Dense J_eq (column-major basis index q + N_Q k) from unit-vector probes through cf_jv_device."""
    import torch

    import cf_b200

    d = load_op(name)
    K, NQ = d["K"], d["NQ"]
    N = K * NQ
    op = cf_b200.CollisionOperator(d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    f = torch.zeros((N, K, NQ), dtype=torch.float64, device="cuda")
    f[:, 0, 0] = 1.0
    E = torch.zeros_like(f)
    for j in range(N):
        E[j, j // NQ, j % NQ] = 1.0
    cols = op.jv(f, E).cpu().numpy()  # [j, k, q]
    op.close()
    J = np.stack([cols[j].T.ravel(order="F") for j in range(N)], axis=1)
    return d, J


def test_wcu_spectrum_on_gpu_operator(cuda_available):
    d, J = _jeq_gpu("wcu_k2_l2_g0")
    lam = np.sort(np.linalg.eigvals(J).real)[::-1]
    lam = lam / abs(lam[5])
    ref = wcu_spectrum(2, 2)
    ref = ref / abs(ref[5])
    assert np.max(np.abs(lam[:5])) < 1e-10
    assert np.max(np.abs(lam - ref)) < 1e-10


@pytest.mark.parametrize("name", ["wcu_k2_l2_g0", "hs_k4_l4_g1"])
def test_h_theorem_on_gpu_operator(name, cuda_available):
    d, J = _jeq_gpu(name)
    lam = np.linalg.eigvals(J).real
    lam = lam / np.sort(np.abs(lam))[5]
    assert np.sum(np.abs(lam) < 1e-10) == 5
    assert np.sum(lam > 1e-10) == 0


def test_chapman_enskog_bracket_on_gpu_operator(cuda_available):
    d, J = _jeq_gpu("hs_k4_l4_g1")
    K, NQ = d["K"], d["NQ"]
    idx = np.arange(K) * NQ + 6  # q = 7 (l = 2, m = 0)
    H = J[np.ix_(idx, idx)]
    H = H / H[0, 0]
    D = np.diag([1.0, -math.sqrt(2.0 / 7.0)])
    H_ana = D @ np.array([[1.0, 0.25], [0.25, 205.0 / 48.0]]) @ D
    assert np.max(np.abs(H[:2, :2] - H_ana)) < 1e-10
    f_mu = [np.linalg.inv(H[:k, :k])[0, 0] for k in range(1, K + 1)]
    assert abs(f_mu[1] - 205.0 / 202.0) < 1e-10
