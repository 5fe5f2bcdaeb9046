"""Edge cases of the forms on the band kernels (the exact int8 split, the FP64 band kernel, the BF16
split on tcgen05) and of the radial-first dense form: empty and one-cell batches, batches that end
inside a cell group, operators that do not fold, and the no-alloc entry point's refusals.

Tolerances: 1e-10 for the split form, 1e-12 for the FP64 forms, 1e-4 for the BF16 split (the
bars of their parity files), normwise per cell against the oracle's restatement of the reference's
angular-first kernel.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

TOL = {"af_sym_i8": 1e-10, "af_sym_bf16": 1e-4, "rf_dense": 1e-12, "af_sym": 1e-12}


def _setup(L, K, seed=3):
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = np.asfortranarray(workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed))
    return geo, R


def _oracle(geo, R, K, cells, oracle_lib, labels=None, vals=None, ic_map=None):
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, geo.labels if labels is None else labels, geo.vals if vals is None else vals,
                        geo.ic_map if ic_map is None else ic_map, R, geo.n_q, K)
    return np.ascontiguousarray(Qo.transpose(2, 1, 0))


@pytest.mark.parametrize("form", ["af_sym_i8", "af_sym_bf16", "rf_dense"])
def test_empty_and_small_batches(form, cuda_available, oracle_lib):
    """B = 0 leaves Q untouched and launches nothing; B = 1, 3, 5 and 9 (cell groups of 4 cut
    anywhere) match the oracle cell by cell."""
    import torch

    import cf_b200
    from cf_b200 import _lib, workloads

    L, K = 5, 12
    geo, R = _setup(L, K, seed=21)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    cells = workloads.maxwellian_cells(K, L, 9, seed=5, amplitude=0.05)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    f0 = torch.zeros((0, K, geo.n_q), dtype=torch.float64, device="cuda")
    n0 = _lib.launch_count()
    op.q(f0, out=torch.zeros_like(f0), form=form)
    torch.cuda.synchronize()
    assert _lib.launch_count() == n0
    for B in (1, 3, 5, 9):
        f = torch.from_numpy(cells[:B].copy()).cuda()
        Q = torch.zeros_like(f)
        op.q(f, out=Q, form=form)
        torch.cuda.synchronize()
        assert per_cell_err(Q.cpu().numpy(), ref[:B]) <= TOL[form], (form, B)
    op.close()


def test_band_path_small_batches(cuda_available, oracle_lib):
    """The FP64 band kernel (path 'band') on 1, 2 and 7 cells at K = 8 (8 cells per CTA) and K = 12."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    for L, K in ((6, 8), (4, 12)):
        geo, R = _setup(L, K, seed=L * K)
        op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
        op.set_kernel_path("band")
        cells = workloads.maxwellian_cells(K, L, 7, seed=K)
        ref = _oracle(geo, R, K, cells, oracle_lib)
        for B in (1, 2, 7):
            f = torch.from_numpy(cells[:B].copy()).cuda()
            Q = torch.zeros_like(f)
            op.q(f, out=Q, form="af_sym")
            torch.cuda.synchronize()
            assert per_cell_err(Q.cpu().numpy(), ref[:B]) <= TOL["af_sym"], (L, K, B)
        op.close()


def test_operator_that_does_not_fold(cuda_available, oracle_lib):
    """A COO list that is not symmetric in (q2, q3), missing one entry of the half the folded list
    keeps: the folded forms (af_sym, the split form) are refused with CF_EUNSUPPORTED rather than
    dropping the orphaned mirror; the radial-first dense form runs on the plain operator and matches
    the oracle."""
    import torch

    import cf_b200
    from cf_b200 import CFError, workloads

    L, K = 4, 4
    geo, R = _setup(L, K, seed=8)
    keep = np.ones(len(geo.vals), dtype=bool)
    # drop one off-diagonal entry (q2 != q3) of the half that the folded list keeps (l2 < l3): its
    # mirror stays, so the list no longer folds
    lq = np.floor(np.sqrt(geo.labels - 1.0)).astype(int)
    kept = np.nonzero((geo.labels[:, 1] != geo.labels[:, 2]) & (lq[:, 1] < lq[:, 2]))[0]
    keep[kept[len(kept) // 2]] = False
    labels = np.ascontiguousarray(geo.labels[keep])
    vals = geo.vals[keep].copy()
    ic_map = geo.ic_map[keep].copy()
    op = cf_b200.CollisionOperator(labels, vals, ic_map, R, geo.n_q, K)
    cells = workloads.maxwellian_cells(K, L, 11, seed=2)
    ref = _oracle(geo, R, K, cells, oracle_lib, labels, vals, ic_map)
    f = torch.from_numpy(cells).cuda()
    for form in ("af_sym", "af_sym_i8"):
        with pytest.raises(CFError) as e:
            op.q(f, out=torch.zeros_like(f), form=form)
        assert e.value.status == 8, form
    Q = torch.zeros_like(f)
    op.q(f, out=Q, form="rf_dense")
    torch.cuda.synchronize()
    assert per_cell_err(Q.cpu().numpy(), ref) <= TOL["rf_dense"]
    op.close()


def test_noalloc_refusals_and_band_tables(cuda_available):
    """cf_q_device_noalloc refuses the radial-first dense form (it allocates scratch) with
    CF_EUNSUPPORTED, and the BF16 split at K = 12 with CF_EINVAL until a cf_q_device call in that form
    has built the band tables; after that it runs it, with the same bits as cf_q_device."""
    import torch

    import cf_b200
    from cf_b200 import _lib, workloads

    L, K, B = 4, 12, 50
    geo, R = _setup(L, K, seed=4)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    lib = _lib.load()
    f = torch.from_numpy(workloads.maxwellian_cells(K, L, B, seed=9)).cuda()
    s = torch.cuda.current_stream().cuda_stream
    out = torch.zeros_like(f)
    assert lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_RF_DENSE, s) == 8
    # builds the folded twin; on the gather kernel, so that no band table exists yet (the automatic
    # order runs the fast forms at K = 12 on the l-block kernel, whose first use builds them)
    op.set_kernel_path("gather")
    op.q(f, out=torch.zeros_like(f), form="af_sym")
    torch.cuda.synchronize()
    assert lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_AF_SYM_BF16, s) == 1
    ref = torch.zeros_like(f)
    op.q(f, out=ref, form="af_sym_bf16")  # builds the band tables
    torch.cuda.synchronize()
    st = lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_AF_SYM_BF16, s)
    assert st == 0, lib.cf_last_error().decode()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    op.close()
