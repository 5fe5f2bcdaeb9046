"""The FP32 Jacobian apply (J.v modes 3 and 4): J(f).v = Q(v,f) + Q(f,v) with f, v, R, Phi and the
row sums in FP32, added into the FP64 out, on the plain and the q2 <-> q3 folded operator (the
pair kernel in FP32, as the FP32 Q form).

Tolerance: 1e-5 normwise per cell against the oracle's bilinear restatement of the reference's
angular-first kernel, the bar of the FP32 Q forms (FP32 carries ~6e-8 per operation, and the
cancellation in J.v near equilibrium leaves ~1e-6); the conservation rows exactly zero.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL_FP32 = 1e-5


def _cm(cells):
    return np.asfortranarray(cells.transpose(2, 1, 0))


@pytest.mark.parametrize("L,K,B", [(4, 4, 37), (8, 8, 60), (6, 12, 21)])
def test_jv_fp32_modes_vs_oracle(L, K, B, cuda_available, oracle_lib):
    import torch

    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = np.load(GOLDEN / "R_hs_k7_l8_pad20.npy") if (L, K) == (8, 8) else \
        workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=L + K)
    R = np.asfortranarray(R)
    NQ = geo.n_q
    cells = workloads.maxwellian_cells(K, L, B, seed=4, amplitude=0.05)
    v = np.random.default_rng(6).standard_normal(cells.shape)
    v /= np.linalg.norm(v.reshape(B, -1), axis=1)[:, None, None]
    ref = np.zeros((NQ, K, B), order="F")
    oracle_lib.jv_batch(ref, _cm(cells), _cm(v), geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    ref = ref.transpose(2, 1, 0)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    ft, vt = torch.from_numpy(cells).cuda(), torch.from_numpy(v).cuda()
    for folded in (False, True):
        out0 = np.full(cells.shape, 0.25)
        out = op.jv(ft, vt, out=torch.from_numpy(out0.copy()).cuda(), folded=folded, fp32=True).cpu().numpy() - 0.25
        err = per_cell_err(out, ref)
        assert 1e-12 < err <= TOL_FP32, (folded, err)
        assert np.all(out.reshape(B, -1)[:, [0, 1, 2, 3, NQ]] == 0.0), folded
    op.close()


def test_jv_fp32_host_entry_and_refusals(cuda_available, oracle_lib):
    """cf_jacobian_apply_host in mode 3 (host arrays, += out) matches the oracle; cf_jv_tiled, whose
    tiles are FP64, refuses the FP32 modes; a mode past 4 is CF_EINVAL."""
    import ctypes as C

    import torch

    import cf_b200
    from cf_b200 import _lib, geometry, workloads
    from oracle import rtensor

    L, K, B = 4, 6, 1100
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = np.asfortranarray(workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=2))
    NQ = geo.n_q
    cells = workloads.maxwellian_cells(K, L, B, seed=8, amplitude=0.05)
    v = np.random.default_rng(1).standard_normal(cells.shape)
    ref = np.zeros((NQ, K, B), order="F")
    oracle_lib.jv_batch(ref, _cm(cells), _cm(v), geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    lib = _lib.load()
    D = C.POINTER(C.c_double)
    out = np.asfortranarray(np.full((NQ, K, B), 0.5))
    f, vv = _cm(cells), _cm(v)
    lab = np.asfortranarray(geo.labels)
    st = lib.cf_jacobian_apply_host(out.ctypes.data_as(D), f.ctypes.data_as(D), vv.ctypes.data_as(D), B,
                                    lab.ctypes.data_as(D), geo.vals.ctypes.data_as(D), geo.ic_map.ctypes.data_as(D),
                                    R.ctypes.data_as(D), geo.n_g, R.size // K**3, NQ, K, 3)
    assert st == 0, lib.cf_last_error().decode()
    out -= 0.5
    assert per_cell_err(np.ascontiguousarray(out.transpose(2, 1, 0)), np.ascontiguousarray(ref.transpose(2, 1, 0))) <= TOL_FP32

    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    n = ((B + 31) // 32) * 32 * NQ * K
    t = torch.zeros(n, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    for mode, status in ((3, 8), (4, 8), (5, 1)):
        assert lib.cf_jv_tiled(op._h, t.data_ptr(), t.data_ptr(), t.data_ptr(), B, mode, s) == status, mode
    ft = torch.from_numpy(cells).cuda()
    assert lib.cf_jv_device(op._h, ft.data_ptr(), ft.data_ptr(), ft.data_ptr(), B, 5, s) == 1
    op.close()
