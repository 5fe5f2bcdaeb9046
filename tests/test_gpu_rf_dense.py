"""The radial-first dense form (CF_FORM_RF_DENSE, csrc/rfdense.cu): the radial step of
radial_first_collision_kernel_mex.cpp:41-59 factored out of the COO entries as one dense
[K^2 x K] x [K x cells] product per (l-triplet, q2), then K^2 per entry; FP64 on the folded operator.

Tolerance: 1e-12 normwise per cell against the oracle's restatement of the reference's angular-first
kernel (both forms compute the same Q; the FP64 bar of the parity suite).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL_FP64 = 1e-12
PATH_RF_DENSE = 13


def _setup(L, K, R=None, seed=3):
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    if R is None:
        R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed)
    return geo, np.asfortranarray(R)


def _oracle(geo, R, K, cells, oracle_lib):
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    return np.ascontiguousarray(Qo.transpose(2, 1, 0))


@pytest.mark.parametrize("L,K,B", [(4, 4, 37), (6, 12, 33), (3, 5, 70), (8, 8, 41)])
def test_rf_dense_vs_oracle(L, K, B, cuda_available, oracle_lib):
    """Device entry, ragged last cell block; invariants exactly zero."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(L, K, np.load(GOLDEN / "R_hs_k7_l8_pad20.npy") if (L, K) == (8, 8) else None, seed=L + K)
    cells = workloads.maxwellian_cells(K, L, B, seed=K)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    f = torch.from_numpy(cells).cuda()
    Q = torch.zeros_like(f)
    op.q(f, out=Q, form="rf_dense")
    torch.cuda.synchronize()
    assert op.info()["last_path"] == PATH_RF_DENSE
    Qn = Q.cpu().numpy()
    assert per_cell_err(Qn, ref) <= TOL_FP64, per_cell_err(Qn, ref)
    assert np.all(Qn.reshape(B, -1)[:, [0, 1, 2, 3, geo.n_q]] == 0.0)
    op.close()


def test_rf_dense_accumulates_deterministic_and_batch_sizes(cuda_available, oracle_lib):
    """out += Q(f) on a nonzero Q; the same bits twice; a larger batch after a smaller one and a
    smaller one after that (the scratch grows and is reused) give the same per-cell results."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    L, K = 5, 6
    geo, R = _setup(L, K, seed=9)
    cells = workloads.maxwellian_cells(K, L, 130, seed=4)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    q0 = np.random.default_rng(2).standard_normal(cells.shape)
    outs = []
    for n in (130, 130, 17, 130, 64):
        f = torch.from_numpy(cells[:n].copy()).cuda()
        Q = torch.from_numpy(q0[:n].copy()).cuda()
        op.q(f, out=Q, form="rf_dense")
        torch.cuda.synchronize()
        outs.append(Q.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    for o in outs:
        n = o.shape[0]
        assert np.array_equal(o, outs[0][:n])
    assert per_cell_err(outs[0] - q0, ref) <= 1e-11
    op.close()


def test_rf_dense_host_entry(cuda_available, oracle_lib):
    """The MEX-compatible batched host entry (column-major arrays) in this form."""
    import cf_b200
    from cf_b200 import workloads

    L, K, B = 4, 8, 1100
    geo, R = _setup(L, K, seed=12)
    cells = workloads.maxwellian_cells(K, L, B, seed=3)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    Qg = np.asfortranarray(np.full_like(f, 0.25))
    cf_b200.contract_batched(Qg, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, form="rf_dense")
    Qg -= 0.25
    assert per_cell_err(np.ascontiguousarray(Qg.transpose(2, 1, 0)), ref) <= TOL_FP64


@pytest.mark.skipif(not (GOLDEN / "R_hs_k11_l16_pad20.npy").exists(), reason="L = 16, K = 12 R fixture absent")
def test_rf_dense_precision_configuration(cuda_available, oracle_lib):
    """Hard spheres, L = 16, K = 12 (R from the GPU quadrature), 9 bi-Maxwellian cells."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(16, 12, np.load(GOLDEN / "R_hs_k11_l16_pad20.npy"))
    cells = workloads.bimaxwellian_cells(12, 16, 9, seed=20260)
    ref = _oracle(geo, R, 12, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    f = torch.from_numpy(cells).cuda()
    Q = torch.zeros_like(f)
    op.q(f, out=Q, form="rf_dense")
    torch.cuda.synchronize()
    assert per_cell_err(Q.cpu().numpy(), ref) <= TOL_FP64
    op.close()
