"""The FP64 band kernel (af_band64_kernel): the fast angular-first Q forms on l1-band work units with
f resident in shared memory and R_t staged per l-triplet by bulk copies, on kernel path 'band'
(K = 4, 8 or 12).

Tolerance: 1e-12 normwise per cell against the oracle's restatement of the reference's angular-first
kernel, the FP64 bar of the parity suite.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL_FP64 = 1e-12
PATH_BAND = 11


def _setup(L, K, R=None, seed=3):
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    if R is None:
        R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed)
    return geo, np.asfortranarray(R)


def _device_q(op, cells, form):
    import torch

    f = torch.from_numpy(cells).cuda()
    Q = torch.zeros_like(f)
    op.q(f, out=Q, form=form)
    torch.cuda.synchronize()
    return Q.cpu().numpy()


def _oracle(geo, R, K, cells, oracle_lib):
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    return np.ascontiguousarray(Qo.transpose(2, 1, 0))


@pytest.mark.parametrize("L,K", [(6, 12), (3, 12), (8, 8), (6, 4)])
def test_band_kernel_vs_oracle(L, K, cuda_available, oracle_lib):
    """Plain and folded fast forms on the band kernel, 37 cells (a ragged last 4-cell group)."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(L, K, np.load(GOLDEN / "R_hs_k7_l8_pad20.npy") if (L, K) == (8, 8) else None, seed=L + K)
    cells = workloads.maxwellian_cells(K, L, 37, seed=K)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    op.set_kernel_path("band")
    for form in ("af", "af_sym"):
        Q = _device_q(op, cells, form)
        assert op.info()["last_path"] == PATH_BAND, form
        assert per_cell_err(Q, ref) <= TOL_FP64, (form, per_cell_err(Q, ref))
    op.close()


@pytest.mark.skipif(not (GOLDEN / "R_hs_k11_l16_pad20.npy").exists(), reason="L = 16, K = 12 R fixture absent")
def test_band_kernel_precision_configuration_vs_oracle(cuda_available, oracle_lib):
    """Hard spheres, L = 16, K = 12 (R from the GPU quadrature), bi-Maxwellian cells: the FP64 forms of
    the precision configuration on a sample of 9 cells the oracle finishes in seconds; the exact-zero
    invariants."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(16, 12, np.load(GOLDEN / "R_hs_k11_l16_pad20.npy"))
    cells = workloads.bimaxwellian_cells(12, 16, 9, seed=20260)
    ref = _oracle(geo, R, 12, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    op.set_kernel_path("band")
    for form in ("af", "af_sym"):
        Q = _device_q(op, cells, form)
        assert per_cell_err(Q, ref) <= TOL_FP64, (form, per_cell_err(Q, ref))
        assert np.abs(Q[:, 0, 0]).max() == 0.0 and np.abs(Q[:, 1, 0]).max() == 0.0
        assert np.abs(Q[:, 0, 1:4]).max() == 0.0
    op.close()


def test_band_kernel_accumulates_and_is_deterministic(cuda_available, oracle_lib):
    """out += Q(f) from a nonzero Q, and two runs give the same bits."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(6, 12, seed=5)
    cells = workloads.maxwellian_cells(12, 6, 19, seed=2)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    op.set_kernel_path("band")
    q0 = np.random.default_rng(1).standard_normal(cells.shape)
    f = torch.from_numpy(cells).cuda()
    outs = []
    for _ in range(2):
        Q = torch.from_numpy(q0.copy()).cuda()
        op.q(f, out=Q, form="af_sym")
        torch.cuda.synchronize()
        outs.append(Q.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    ref = _oracle(geo, R, 12, cells, oracle_lib)
    assert per_cell_err(outs[0] - q0, ref) <= 1e-11
    op.close()
