"""The exact-split form CF_FORM_AF_SYM_I8 (FP64 Phi, K^3 step on the int8 tensor cores) on the GPU.

Parity bar: <= 1e-10 normwise per cell (max |dQ| / max |Q| of each cell) against the oracle's
restatement of the reference's angular-first kernel (src/mex/angular_first_collision_kernel_mex.cpp),
the bar the precision forms are held to.  The design point is ~1e-11: Phi and R_t are rounded to
47-bit fixed point, everything after that is exact integer arithmetic until the FP64 recombination.
The invariant entries of Q must stay exactly zero (R's conservation rows are exact zeros, so their
byte planes are zeros too).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import load_op, per_cell_err

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL_SPLIT = 1e-10


def _cells_cm(cells):
    return np.asfortranarray(cells.transpose(2, 1, 0))


def _operator(L, K, R=None, seed=3):
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    if R is None:
        R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed)
    return geo, np.asfortranarray(R)


def _invariant_abs_max(Q, NQ):
    # (q, k) = (1, 0), (1, 1), (2..4, 0) in 1-based q: Q[0,0], Q[0,1], Q[1:4,0] per cell
    return max(np.abs(Q[0, 0]).max(), np.abs(Q[0, 1]).max(), np.abs(Q[1:4, 0]).max())


def _check_vs_oracle(geo, R, K, B, oracle_lib, seed=7, bimax=False):
    import cf_b200
    from cf_b200 import workloads

    NQ = geo.n_q
    cells = (workloads.bimaxwellian_cells(K, geo.L, B, seed=seed) if bimax else
             workloads.maxwellian_cells(K, geo.L, B, seed=seed, amplitude=1e-2, decay=0.6))
    f = _cells_cm(cells)
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, *args)
    Qg = np.zeros_like(f, order="F")
    cf_b200.contract_batched(Qg, f, *args, form="af_sym_i8")
    err = per_cell_err(Qg.transpose(2, 1, 0), Qo.transpose(2, 1, 0))
    return err, Qg, Qo, f, args


def test_split_cpu_runnable_operator(cuda_available, oracle_lib):
    """K = 4, L = 4, Maxwell molecules (the CPU-runnable operator, R from the reference's quadrature)."""
    import cf_b200

    d = load_op("cfg1_k3_l4_g0")
    NQ, K = d["NQ"], d["K"]
    args = (d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    Q = np.zeros((NQ, K), order="F")
    cf_b200.contract_batched(Q, d["f"], *args, form="af_sym_i8")
    err = np.abs(Q - d["Q_af"]).max() / np.abs(d["Q_af"]).max()
    assert err <= TOL_SPLIT, err
    assert _invariant_abs_max(Q[:, :, None], NQ) == 0.0


@pytest.mark.parametrize("L", [8, 10])
def test_split_hard_spheres_k8_vs_oracle(L, cuda_available, oracle_lib):
    """Hard spheres, K = 8, R from the reference's quadrature (committed fixtures), 43 cells (not a
    multiple of the 4-cell groups)."""
    geo, R = _operator(L, 8, np.load(GOLDEN / f"R_hs_k7_l{L}_pad20.npy"))
    err, Qg, Qo, _, _ = _check_vs_oracle(geo, R, 8, 43, oracle_lib)
    assert err <= TOL_SPLIT, err
    assert _invariant_abs_max(Qg, geo.n_q) == 0.0


@pytest.mark.parametrize("L,K", [(6, 12), (3, 12), (6, 4)])
def test_split_synthetic_operators_vs_oracle(L, K, cuda_available, oracle_lib):
    geo, R = _operator(L, K, seed=L * 7 + K)
    err, Qg, _, _, _ = _check_vs_oracle(geo, R, K, 21, oracle_lib, seed=K)
    assert err <= TOL_SPLIT, err
    assert _invariant_abs_max(Qg, geo.n_q) == 0.0


@pytest.mark.skipif(not (GOLDEN / "R_hs_k11_l16_pad20.npy").exists(), reason="L = 16, K = 12 R fixture absent")
def test_split_precision_configuration_vs_oracle(cuda_available, oracle_lib):
    """Hard spheres, L = 16, K = 12, bi-Maxwellian cells (the precision-form configuration), on a
    sample of 9 cells that the oracle finishes in seconds."""
    geo, R = _operator(16, 12, np.load(GOLDEN / "R_hs_k11_l16_pad20.npy"))
    err, Qg, _, _, _ = _check_vs_oracle(geo, R, 12, 9, oracle_lib, bimax=True)
    assert err <= TOL_SPLIT, err
    assert _invariant_abs_max(Qg, geo.n_q) == 0.0


def test_split_accumulates_deterministic_and_host_equals_device(cuda_available, oracle_lib):
    """Q_out += Q(f) from a nonzero Q_in; two runs give the same bits; the host entry point and the
    device entry point (cf_q_device) give the same bits."""
    import torch

    import cf_b200

    geo, R = _operator(8, 8, np.load(GOLDEN / "R_hs_k7_l8_pad20.npy"))
    err, Qg, Qo, f, args = _check_vs_oracle(geo, R, 8, 30, oracle_lib, seed=11)
    rng = np.random.default_rng(4)
    Q0 = np.asfortranarray(rng.standard_normal(f.shape) * np.abs(Qo).max())
    Q1 = Q0.copy(order="F")
    cf_b200.contract_batched(Q1, f, *args, form="af_sym_i8")
    Q2 = Q0.copy(order="F")
    cf_b200.contract_batched(Q2, f, *args, form="af_sym_i8")
    assert np.array_equal(Q1, Q2)
    assert np.abs((Q1 - Q0) - Qg).max() <= 1e-13 * np.abs(Q0).max()
    op = cf_b200.CollisionOperator(*args)
    fd = torch.from_numpy(np.ascontiguousarray(f.transpose(2, 1, 0))).cuda()
    Qd = torch.from_numpy(np.ascontiguousarray(Q0.transpose(2, 1, 0))).cuda()
    op.q(fd, out=Qd, form="af_sym_i8")
    torch.cuda.synchronize()
    assert np.array_equal(Qd.cpu().numpy(), np.ascontiguousarray(Q1.transpose(2, 1, 0)))
    assert op.info()["last_path"] == 10  # PATH_SPLIT_I8
    op.close()


def test_split_full_size_properties(cuda_available, oracle_lib):
    """4096 cells at L = 10, K = 8 (the batch configuration): exact-zero invariants, the FP64 folded
    form within 1e-10 per cell, a sample of cells against the oracle, and homogeneity
    Q(2f) = 4 Q(f) (exact: powers of two scale the fixed point exactly)."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    geo, R = _operator(10, 8, np.load(GOLDEN / "R_hs_k7_l10_pad20.npy"))
    NQ, K, B = geo.n_q, 8, 4096
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    cells = workloads.maxwellian_cells(K, 10, B, seed=20260, amplitude=1e-2, decay=0.6)
    op = cf_b200.CollisionOperator(*args)
    fd = torch.from_numpy(cells).cuda()
    Qs = torch.zeros_like(fd)
    op.q(fd, out=Qs, form="af_sym_i8")
    Q64 = torch.zeros_like(fd)
    op.q(fd, out=Q64, form="af_sym")
    Q2 = torch.zeros_like(fd)
    op.q(2.0 * fd, out=Q2, form="af_sym_i8")
    torch.cuda.synchronize()
    Qs, Q64, Q2 = Qs.cpu().numpy(), Q64.cpu().numpy(), Q2.cpu().numpy()
    op.close()
    assert per_cell_err(Qs, Q64) <= TOL_SPLIT
    assert np.abs(Qs[:, 0, 0]).max() == 0.0 and np.abs(Qs[:, 1, 0]).max() == 0.0
    assert np.abs(Qs[:, 0, 1:4]).max() == 0.0
    assert np.array_equal(Q2, 4.0 * Qs)
    sample = np.arange(0, B, 257)
    f = _cells_cm(cells[sample])
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, *args)
    assert per_cell_err(Qs[sample], Qo.transpose(2, 1, 0)) <= TOL_SPLIT


def test_split_refusals(cuda_available):
    """K outside {4, 8, 12}, J.v, tiled arrays and the allocation-free entry point are refused."""
    import cf_b200
    from cf_b200 import _lib

    geo, R = _operator(4, 6)
    f = np.asfortranarray(np.ones((geo.n_q, 6, 3)))
    Q = np.zeros_like(f, order="F")
    with pytest.raises(_lib.CFError) as e:
        cf_b200.contract_batched(Q, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 6, form="af_sym_i8")
    assert e.value.status == _lib.CF_EUNSUPPORTED
