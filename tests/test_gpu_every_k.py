"""GPU parity at every K the library builds (1..16): each Q form and the J.v modes, called through the
C ABI, against the oracle on a ragged batch with Q nonzero on entry (+= semantics).

Tolerances: fast FP64 forms <= 1e-12 per cell (normwise); the EXACT forms (Q and J.v) bit for bit;
FP32 forms <= 1e-5 per cell.  Forms that a K does not have (FP32 at odd K or K > 12) must be refused
with CF_EUNSUPPORTED, never computed some other way.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
TOL_FP32 = 1e-5
EUNSUPPORTED = 8
KS = list(range(1, 17))


def _case(K: int):
    """A small operator per K: L from 3 to 5, so that the K also meet different band layouts."""
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    L = 3 + K % 3
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=100 + K)
    B = 19 + 2 * K  # odd: not a multiple of any cell tile
    cells = workloads.maxwellian_cells(K, L, B, seed=K, amplitude=0.05)
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    rng = np.random.default_rng(K)
    q0 = np.asfortranarray(rng.standard_normal(f.shape))
    return geo, R, f, q0, (geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)


def _err(a, b):
    return per_cell_err(a.transpose(2, 1, 0), b.transpose(2, 1, 0))


@pytest.mark.parametrize("K", KS)
def test_q_forms_at_every_k(K, cuda_available, oracle_lib):
    import cf_b200
    from cf_b200 import CFError

    _, _, f, q0, args = _case(K)
    ref = {}
    for kind in ("af", "rf"):
        r = q0.copy(order="F")
        oracle_lib.af_batch(r, f, *args, form=kind)
        ref[kind] = r
    # the exact forms: the reference's operation order, bit for bit, from a nonzero Q
    for form, kind in (("af_exact", "af"), ("rf_exact", "rf")):
        q = q0.copy(order="F")
        cf_b200.contract_batched(q, f, *args, form=form)
        assert np.array_equal(q, ref[kind]), f"{form} K={K}: max |diff| {np.abs(q - ref[kind]).max():.3e}"
    # the fast FP64 forms (folded included)
    for form, kind in (("af", "af"), ("af_sym", "af"), ("rf", "rf"), ("rf_dense", "rf")):
        q = q0.copy(order="F")
        cf_b200.contract_batched(q, f, *args, form=form)
        err = _err(q - q0, ref[kind] - q0)
        assert err <= TOL_FP64, f"{form} K={K}: {err:.3e}"
    # the FP32 forms exist at even K <= 12 and are refused elsewhere
    for form in ("af_f32", "af_sym_f32"):
        q = q0.copy(order="F")
        if K % 2 == 0 and K <= 12:
            cf_b200.contract_batched(q, f, *args, form=form)
            err = _err(q - q0, ref["af"] - q0)
            assert err <= TOL_FP32, f"{form} K={K}: {err:.3e}"
        else:
            with pytest.raises(CFError) as e:
                cf_b200.contract_batched(q, f, *args, form=form)
            assert e.value.status == EUNSUPPORTED
            assert np.array_equal(q, q0), "a refused call must leave Q untouched"


@pytest.mark.parametrize("K", KS)
def test_jacobian_apply_at_every_k(K, cuda_available, oracle_lib):
    import cf_b200

    _, _, f, q0, args = _case(K)
    v = np.asfortranarray(np.random.default_rng(50 + K).standard_normal(f.shape))
    ref = q0.copy(order="F")
    oracle_lib.jv_batch(ref, f, v, *args)
    for mode in (0, 2):  # fast, folded
        out = q0.copy(order="F")
        cf_b200.collision_jacobian_apply_mex(out, f, v, *args, exact=mode)
        err = _err(out - q0, ref - q0)
        assert err <= TOL_FP64, f"J.v mode {mode} K={K}: {err:.3e}"
    out = q0.copy(order="F")
    cf_b200.collision_jacobian_apply_mex(out, f, v, *args, exact=1)
    assert np.array_equal(out, ref), f"exact J.v K={K} must equal the oracle's operation order bit for bit"


@pytest.mark.parametrize("L,K,B", [(6, 12, 301), (4, 16, 64)])
def test_exact_jacobian_apply_device_entry_above_k8(L, K, B, cuda_available, oracle_lib):
    """The exact J.v above K = 8 through cf_jv_device (two cells per CTA on the row kernel; an odd
    batch leaves the last CTA one cell): out += J(f) v bit for bit the oracle's, from a nonzero out."""
    import torch

    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=L + K)
    cells = workloads.maxwellian_cells(K, L, B, seed=3, amplitude=0.05)
    rng = np.random.default_rng(4)
    vc = rng.standard_normal(cells.shape)
    o0 = rng.standard_normal(cells.shape) * 1e-3
    ref = np.array(o0.transpose(2, 1, 0), order="F")
    oracle_lib.jv_batch(ref, np.asfortranarray(cells.transpose(2, 1, 0)), np.asfortranarray(vc.transpose(2, 1, 0)),
                        geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    out = torch.from_numpy(o0).cuda()
    op.jv(torch.from_numpy(cells).cuda(), torch.from_numpy(vc).cuda(), out=out, exact=True)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref.transpose(2, 1, 0))
    op.close()
