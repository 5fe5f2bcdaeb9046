"""The BF16-split forms on the band kernel (af_bf16_band_kernel): the K^3 step on the BF16 tensor
cores through tcgen05.mma (kind::f16) with R_t and Phi as BF16 hi + lo and an FP32 accumulator in
tensor memory; the Phi step in FP64.  Taken automatically at K = 4 and 12, on kernel path 'band' at
K = 8.

Tolerance: 1e-4 normwise per cell against the oracle's restatement of the reference's angular-first
kernel, the bar of the BF16-split forms (two BF16 terms carry about 16 significant bits, the sums
run in FP32); the conservation rows of Q are exactly zero, as in every form.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL_BF16 = 1e-4
PATH_BAND_BF16 = 12


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


def _invariants_zero(Q, n_q):
    B = Q.shape[0]
    return np.all(Q.reshape(B, -1)[:, [0, 1, 2, 3, n_q]] == 0.0)


@pytest.mark.parametrize("L,K", [(6, 12), (3, 12), (6, 4), (2, 4), (8, 8)])
def test_bf16_band_kernel_vs_oracle(L, K, cuda_available, oracle_lib):
    """Plain and folded BF16-split forms through the device entry, 37 cells (a ragged last group)."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(L, K, np.load(GOLDEN / "R_hs_k7_l8_pad20.npy") if (L, K) == (8, 8) else None, seed=L + K)
    cells = workloads.maxwellian_cells(K, L, 37, seed=K, amplitude=0.05)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    if K == 8:
        op.set_kernel_path("band")
    f = torch.from_numpy(cells).cuda()
    for form in ("af_bf16", "af_sym_bf16"):
        Q = torch.zeros_like(f)
        op.q(f, out=Q, form=form)
        torch.cuda.synchronize()
        assert op.info()["last_path"] == PATH_BAND_BF16, form
        Qn = Q.cpu().numpy()
        err = per_cell_err(Qn, ref)
        assert 1e-12 < err <= TOL_BF16, (form, err)
        assert _invariants_zero(Qn, geo.n_q), form
    op.close()


def test_bf16_band_host_entry_accumulates(cuda_available, oracle_lib):
    """The host entry (column-major arrays, Q_out = Q_in + Q(f)) at K = 12, both BF16-split forms."""
    import cf_b200
    from cf_b200 import workloads

    L, K, B = 5, 12, 45
    geo, R = _setup(L, K, seed=11)
    cells = workloads.maxwellian_cells(K, L, B, seed=4, amplitude=0.05)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    args = (geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    for form in ("af_bf16", "af_sym_bf16"):
        Qg = np.asfortranarray(np.full_like(f, 0.125))
        cf_b200.contract_batched(Qg, f, *args, form=form)
        Qg -= 0.125
        Qc = np.ascontiguousarray(Qg.transpose(2, 1, 0))
        assert per_cell_err(Qc, ref) <= TOL_BF16, form


@pytest.mark.skipif(not (GOLDEN / "R_hs_k11_l16_pad20.npy").exists(), reason="L = 16, K = 12 R fixture absent")
def test_bf16_band_precision_configuration(cuda_available, oracle_lib):
    """Hard spheres, L = 16, K = 12 (R from the GPU quadrature), bi-Maxwellian cells: the BF16-split
    forms of the precision configuration on a 9-cell sample the oracle finishes in seconds."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(16, 12, np.load(GOLDEN / "R_hs_k11_l16_pad20.npy"))
    cells = workloads.bimaxwellian_cells(12, 16, 9, seed=20260)
    ref = _oracle(geo, R, 12, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    f = torch.from_numpy(cells).cuda()
    for form in ("af_bf16", "af_sym_bf16"):
        Q = torch.zeros_like(f)
        op.q(f, out=Q, form=form)
        torch.cuda.synchronize()
        Qn = Q.cpu().numpy()
        assert per_cell_err(Qn, ref) <= TOL_BF16, (form, per_cell_err(Qn, ref))
        assert _invariants_zero(Qn, geo.n_q), form
    op.close()


def test_bf16_band_deterministic_and_linear_in_scale(cuda_available):
    """Two runs give the same bits; Q(2 f) = 4 Q(f) exactly (scaling by 2 is exact in BF16, FP32 and
    FP64), at a batch of 4099 cells (a ragged last cell group)."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    L, K, B = 6, 12, 4099
    geo, R = _setup(L, K, seed=7)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    f = torch.from_numpy(workloads.maxwellian_cells(K, L, B, seed=5, amplitude=0.05)).cuda()
    outs = []
    for scale in (1.0, 1.0, 2.0):
        Q = torch.zeros_like(f)
        op.q(f * scale, out=Q, form="af_sym_bf16")
        torch.cuda.synchronize()
        outs.append(Q)
    assert torch.equal(outs[0], outs[1])
    assert torch.equal(outs[2], 4.0 * outs[0])
    op.close()
