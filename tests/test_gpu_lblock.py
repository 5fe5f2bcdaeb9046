"""The l-block kernel (af_lblock64_kernel): the fast angular-first Q forms with one CTA per (l1 band,
8-cell group), R_t and the f rows of bands l2 and l3 staged per l-triplet by bulk copies from f packed
per 8-cell group, the band's (t, row) slices taken by the warps one at a time and summed into each
row in t order, and the K^3 step on the FP64 tensor cores; on kernel path 'lblock' (K = 8 and 12), and
in the automatic order at K = 12.  The FP32 forms run the same schedule on 16 cells per CTA.

Tolerance: 1e-12 normwise per cell against the oracle's restatement of the reference's angular-first
kernel (src/mex/angular_first_collision_kernel_mex.cpp:45-69), the FP64 bar of the parity suite.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL_FP64 = 1e-12
PATH_LBLOCK = 14


def _setup(L, K, R=None, seed=3):
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    if R is None:
        R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed)
    return geo, np.asfortranarray(R)


def _device_q(op, cells, form, q0=None):
    import torch

    f = torch.from_numpy(cells).cuda()
    Q = torch.zeros_like(f) if q0 is None else torch.from_numpy(q0.copy()).cuda()
    op.q(f, out=Q, form=form)
    torch.cuda.synchronize()
    return Q.cpu().numpy()


def _oracle(geo, R, K, cells, oracle_lib):
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    return np.ascontiguousarray(Qo.transpose(2, 1, 0))


@pytest.mark.parametrize("L,K,B", [(6, 12, 37), (3, 12, 16), (1, 12, 13), (8, 8, 37), (10, 8, 21), (0, 8, 11)])
def test_lblock_kernel_vs_oracle(L, K, B, cuda_available, oracle_lib):
    """Plain and folded fast forms on the l-block kernel; batches with a ragged last 8-cell group or
    whole groups only, and bands whose l-triplets have l2 = l3 (one staged row block) or not."""
    import cf_b200
    from cf_b200 import workloads

    R = np.load(GOLDEN / "R_hs_k7_l8_pad20.npy") if (L, K) == (8, 8) else None
    if (L, K) == (10, 8):
        R = np.load(GOLDEN / "R_hs_k7_l10_pad20.npy")
    geo, R = _setup(L, K, R, seed=L + K)
    cells = workloads.maxwellian_cells(K, L, B, seed=K + B)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    op.set_kernel_path("lblock")
    for form in ("af", "af_sym"):
        Q = _device_q(op, cells, form)
        assert op.info()["last_path"] == PATH_LBLOCK, form
        assert per_cell_err(Q, ref) <= TOL_FP64, (form, per_cell_err(Q, ref))
    op.close()


@pytest.mark.skipif(not (GOLDEN / "R_hs_k11_l16_pad20.npy").exists(), reason="L = 16, K = 12 R fixture absent")
def test_lblock_kernel_precision_configuration_vs_oracle(cuda_available, oracle_lib):
    """Hard spheres, L = 16, K = 12 (R from the GPU quadrature), bi-Maxwellian cells: the FP64 forms of
    the precision configuration on 11 cells (a whole and a ragged 8-cell group) against the oracle;
    the five invariant entries exactly zero."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(16, 12, np.load(GOLDEN / "R_hs_k11_l16_pad20.npy"))
    cells = workloads.bimaxwellian_cells(12, 16, 11, seed=20261)
    ref = _oracle(geo, R, 12, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    op.set_kernel_path("lblock")
    for form in ("af", "af_sym"):
        Q = _device_q(op, cells, form)
        assert op.info()["last_path"] == PATH_LBLOCK, form
        assert per_cell_err(Q, ref) <= TOL_FP64, (form, per_cell_err(Q, ref))
        assert np.abs(Q[:, 0, 0]).max() == 0.0 and np.abs(Q[:, 1, 0]).max() == 0.0
        assert np.abs(Q[:, 0, 1:4]).max() == 0.0
    op.close()


@pytest.mark.skipif(not (GOLDEN / "R_hs_k11_l16_pad20.npy").exists(), reason="L = 16, K = 12 R fixture absent")
def test_precision_configuration_automatic_order_vs_oracle(cuda_available, oracle_lib):
    """The automatic kernel order at L = 16, K = 12 (hard spheres, R from the GPU quadrature): the plain
    and folded FP64 forms on the l-block kernel, both within 1e-12 of the oracle on 13 bi-Maxwellian
    cells; an operator given in an unsorted COO order (several runs per (t, q1)) has no band tables
    and runs on the gather kernel, to the same tolerance."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(16, 12, np.load(GOLDEN / "R_hs_k11_l16_pad20.npy"))
    cells = workloads.bimaxwellian_cells(12, 16, 13, seed=20262)
    ref = _oracle(geo, R, 12, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    for form in ("af", "af_sym"):
        Q = _device_q(op, cells, form)
        assert cf_b200._lib.PATH_NAMES[op.info()["last_path"]] == "lblock", form
        assert per_cell_err(Q, ref) <= TOL_FP64, (form, per_cell_err(Q, ref))
    op.close()
    perm = np.random.default_rng(3).permutation(geo.n_g)
    op = cf_b200.CollisionOperator(np.asfortranarray(geo.labels[perm]), geo.vals[perm], geo.ic_map[perm], R,
                                   geo.n_q, 12)
    Q = _device_q(op, cells, "af")
    assert cf_b200._lib.PATH_NAMES[op.info()["last_path"]] == "gather"
    assert per_cell_err(Q, ref) <= TOL_FP64
    op.close()


def test_lblock_kernel_accumulates_and_is_deterministic(cuda_available, oracle_lib):
    """out += Q(f) from a nonzero Q, two runs give the same bits (whichever warp takes which slice, each
    row sums its slices in t order), and Q(2f) = 4 Q(f) bit for bit."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(6, 12, seed=5)
    cells = workloads.maxwellian_cells(12, 6, 19, seed=2)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    op.set_kernel_path("lblock")
    q0 = np.random.default_rng(1).standard_normal(cells.shape)
    outs = [_device_q(op, cells, "af_sym", q0) for _ in range(2)]
    assert np.array_equal(outs[0], outs[1])
    ref = _oracle(geo, R, 12, cells, oracle_lib)
    assert per_cell_err(outs[0] - q0, ref) <= 1e-11
    q1 = _device_q(op, cells, "af_sym")
    q2 = _device_q(op, 2.0 * cells, "af_sym")
    assert np.array_equal(q2, 4.0 * q1)
    op.close()


def test_lblock_kernel_refuses_other_k(cuda_available):
    """K outside {8, 12} on path 'lblock' is refused with CF_EUNSUPPORTED, not run on another kernel."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(4, 4, seed=1)
    cells = workloads.maxwellian_cells(4, 4, 9, seed=1)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 4)
    op.set_kernel_path("lblock")
    with pytest.raises(cf_b200.CFError) as e:
        _device_q(op, cells, "af_sym")
    assert e.value.status == cf_b200._lib.CF_EUNSUPPORTED
    op.close()


@pytest.mark.parametrize("L,K,B", [(6, 12, 37), (10, 8, 21), (16, 12, 19)])
def test_lblock_fp32_forms_vs_oracle(L, K, B, cuda_available, oracle_lib):
    """The FP32 forms on the l-block kernel (16 cells per CTA; f, Phi and the K^3 step in FP32, each
    slice's result added into FP64 Q): within 1e-5 per cell of the oracle (FP32 arithmetic), the
    invariant entries exactly zero, two runs bit for bit equal."""
    import cf_b200
    from cf_b200 import workloads

    R = None
    if (L, K) == (10, 8):
        R = np.load(GOLDEN / "R_hs_k7_l10_pad20.npy")
    if (L, K) == (16, 12):
        R = np.load(GOLDEN / "R_hs_k11_l16_pad20.npy")
    geo, R = _setup(L, K, R, seed=L * K)
    cells = workloads.bimaxwellian_cells(K, L, B, seed=5) if L == 16 else workloads.maxwellian_cells(K, L, B, seed=5)
    ref = _oracle(geo, R, K, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    op.set_kernel_path("lblock")
    for form in ("af_f32", "af_sym_f32"):
        Q = _device_q(op, cells, form)
        assert op.info()["last_path"] == PATH_LBLOCK, form
        err = per_cell_err(Q, ref)
        assert 1e-12 < err <= 1e-5, (form, err)
        inv = Q.reshape(B, -1)[:, [0, 1, 2, 3, geo.n_q]]
        assert np.all(inv == 0.0), form
        assert np.array_equal(_device_q(op, cells, form), Q), form
    op.close()


def test_lblock_wait_gives_up_and_reports(cuda_available, oracle_lib):
    """A launch whose stages never fill: every bounded wait (stage assignment, mbarrier, row ticket)
    runs out after 1 ms, the kernel returns, the call reports CF_ETIMEOUT, and the same plan then
    contracts correctly (the error word is cleared)."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(6, 12, seed=9)
    cells = workloads.maxwellian_cells(12, 6, 21, seed=4)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    op.set_kernel_path("lblock")
    assert op.lblock_selftest(1e-3) == 9
    assert "gave up" in cf_b200._lib.load().cf_last_error().decode()
    Q = _device_q(op, cells, "af")
    assert op.info()["last_path"] == PATH_LBLOCK
    assert per_cell_err(Q, _oracle(geo, R, 12, cells, oracle_lib)) <= TOL_FP64
    assert op.lblock_selftest(1e-3) == 9
    assert np.array_equal(_device_q(op, cells, "af"), Q)
    op.close()


def test_lblock_through_the_allocation_free_entry_point(cuda_available):
    """At K = 12  the automatic order runs the fast forms on the l-block kernel, whose band
    tables are built with allocations on first use: cf_q_device_noalloc refuses the form (CF_EINVAL)
    until one cf_q_device call has built them, then packs f into its fixed array and gives the bits
    of cf_q_device, on two calls in a row."""
    import torch

    import cf_b200
    from cf_b200 import _lib, workloads

    geo, R = _setup(8, 12, seed=13)
    B = 50
    f = torch.from_numpy(workloads.maxwellian_cells(12, 8, B, seed=6)).cuda()
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    lib = _lib.load()
    s = torch.cuda.current_stream().cuda_stream
    out = torch.zeros_like(f)
    assert lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_AF, s) == _lib.CF_EINVAL
    ref = op.q(f, form="af")  # cf_q_device: builds the band tables
    assert op.info()["last_path"] == PATH_LBLOCK
    for _ in range(2):
        out = torch.zeros_like(f)
        assert lib.cf_q_device_noalloc(op._h, out.data_ptr(), f.data_ptr(), B, _lib.FORM_AF, s) == 0
        torch.cuda.synchronize()
        assert op.info()["last_path"] == PATH_LBLOCK
        assert torch.equal(out, ref)
    op.close()


@pytest.mark.parametrize("L,K,B", [(6, 12, 21), (3, 16, 10), (5, 12, 3)])
def test_exact_form_above_k8_bitwise(L, K, B, cuda_available, oracle_lib):
    """The exact angular-first form above K = 8 (one CTA per (q1, pair of cells), the reference's operation
    order) gives the oracle's bits, which are the compiled reference kernel's: batches of any size and
    a handful of cells, from Q = 0 and from a nonzero Q."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(L, K, seed=L * K)
    cells = workloads.maxwellian_cells(K, L, B, seed=B)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    q0 = np.random.default_rng(2).standard_normal(cells.shape) * 1e-3
    for start in (None, q0):
        f = np.asfortranarray(cells.transpose(2, 1, 0))
        Qo = np.zeros_like(f, order="F") if start is None else np.array(start.transpose(2, 1, 0), order="F")
        oracle_lib.af_batch(Qo, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
        Q = _device_q(op, cells, "af_exact", start)
        assert np.array_equal(Q, Qo.transpose(2, 1, 0))
    op.close()


@pytest.mark.skipif(not (GOLDEN / "R_hs_k11_l16_pad20.npy").exists(), reason="L = 16, K = 12 R fixture absent")
def test_exact_form_precision_configuration_bitwise(cuda_available, oracle_lib):
    """L = 16, K = 12 (hard spheres, R from the GPU quadrature), 9 bi-Maxwellian cells: the exact form
    bit for bit the oracle's (the reference kernel's operation order)."""
    import cf_b200
    from cf_b200 import workloads

    geo, R = _setup(16, 12, np.load(GOLDEN / "R_hs_k11_l16_pad20.npy"))
    cells = workloads.bimaxwellian_cells(12, 16, 9, seed=20263)
    ref = _oracle(geo, R, 12, cells, oracle_lib)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, 12)
    assert np.array_equal(_device_q(op, cells, "af_exact"), ref)
    op.close()
