"""GPU parity: the sm_100a kernels, called through the C ABI, against the oracle and the reference.

Tolerances: FP64 forms <= 1e-12 normwise per cell; the EXACT forms are
bit-for-bit equal to the reference's own compiled kernels.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_op, normwise_err, per_cell_err

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12
OPS = ["wcu_k2_l2_g0", "cfg1_k3_l4_g0", "hs_k4_l4_g1", "bkw_k5_l1_g0"]


def _cells_cm(cells):
    """[B, K, NQ] C-order -> column-major [NQ, K, B] (same bytes)."""
    return np.asfortranarray(cells.transpose(2, 1, 0))


@pytest.mark.parametrize("name", OPS)
def test_mex_angular_first_matches_reference(name, cuda_available):
    import cf_b200

    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    Q = np.zeros((NQ, K), order="F")
    cf_b200.angular_first_collision_kernel_mex(Q, d["f"], d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"],
                                               d["R"], NQ, K)
    assert normwise_err(Q, d["Q_af"]) <= TOL_FP64
    Q2 = np.zeros((NQ, K), order="F")
    cf_b200.radial_first_collision_kernel_mex(Q2, d["f"], d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"],
                                              d["R"], NQ, K)
    assert normwise_err(Q2, d["Q_rf"]) <= TOL_FP64


@pytest.mark.parametrize("name", OPS)
def test_exact_forms_bitwise_equal_reference(name, cuda_available):
    """The EXACT forms reproduce the compiled reference kernels bit for bit (golden outputs)."""
    import cf_b200

    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    for form, key in (("af_exact", "Q_af"), ("rf_exact", "Q_rf")):
        Q = np.zeros((NQ, K), order="F")
        cf_b200.contract_batched(Q, d["f"], d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K,
                                 form=form)
        assert np.array_equal(Q, d[key]), f"{form}: max |diff| = {np.abs(Q - d[key]).max()}"


def test_exact_form_bitwise_on_batch_and_nonzero_q(cuda_available, oracle_lib, reference_lib):
    """Bitwise parity with the reference's MEX called cell by cell, Q_out nonzero on entry (+= semantics)."""
    import cf_b200
    from cf_b200 import workloads

    d = load_op("hs_k4_l4_g1")
    NQ, K = d["NQ"], d["K"]
    cells = workloads.maxwellian_cells(K, d["L"], 45, seed=21)
    f = _cells_cm(cells)
    rng = np.random.default_rng(5)
    Q0 = np.asfortranarray(rng.standard_normal(f.shape))
    args = (d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    Qr = Q0.copy(order="F")
    reference_lib.batch("af", Qr, f, *args, nthreads=4)
    Qg = Q0.copy(order="F")
    cf_b200.contract_batched(Qg, f, *args, form="af_exact")
    assert np.array_equal(Qg, Qr)
    Qr = Q0.copy(order="F")
    reference_lib.batch("rf", Qr, f, *args, nthreads=4)
    Qg = Q0.copy(order="F")
    cf_b200.contract_batched(Qg, f, *args, form="rf_exact")
    assert np.array_equal(Qg, Qr)


@pytest.mark.parametrize("L,K", [(4, 4), (6, 6), (8, 6), (10, 8), (6, 12), (4, 16), (3, 1)])
def test_fast_forms_vs_oracle(L, K, cuda_available, oracle_lib):
    """AF and RF fast forms vs the oracle on batches whose size is not a multiple of the tile."""
    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=L * 31 + K)
    B = 37 if L <= 8 else 13
    f = _cells_cm(workloads.maxwellian_cells(K, L, B, seed=L + K))
    NQ = geo.n_q
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, *args)
    for form in ("af", "rf", "af_sym"):
        Qg = np.zeros_like(f, order="F")
        cf_b200.contract_batched(Qg, f, *args, form=form)
        err = per_cell_err(Qg.transpose(2, 1, 0), Qo.transpose(2, 1, 0))
        assert err <= TOL_FP64, f"{form} L={L} K={K}: {err:.3e}"


@pytest.mark.parametrize("L,K", [(4, 4), (8, 8), (6, 12), (4, 16)])
def test_jacobian_apply_vs_oracle(L, K, cuda_available, oracle_lib):
    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=5)
    B = 35
    f = _cells_cm(workloads.maxwellian_cells(K, L, B, seed=9))
    rng = np.random.default_rng(2)
    v = np.asfortranarray(rng.standard_normal(f.shape))
    NQ = geo.n_q
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    ref = np.zeros_like(f, order="F")
    oracle_lib.jv_batch(ref, f, v, *args)
    out = np.zeros_like(f, order="F")
    cf_b200.collision_jacobian_apply_mex(out, f, v, *args)
    assert per_cell_err(out.transpose(2, 1, 0), ref.transpose(2, 1, 0)) <= TOL_FP64
    out3 = np.zeros_like(f, order="F")
    cf_b200.collision_jacobian_apply_mex(out3, f, v, *args, exact=2)  # folded operator
    assert per_cell_err(out3.transpose(2, 1, 0), ref.transpose(2, 1, 0)) <= TOL_FP64
    out2 = np.zeros_like(f, order="F")
    cf_b200.collision_jacobian_apply_mex(out2, f, v, *args, exact=True)
    assert np.array_equal(out2, ref), "exact J.v must equal the oracle's operation order bit for bit"


def test_unsorted_and_interleaved_coo(cuda_available, oracle_lib):
    """Any entry order is accepted: runs of equal (t, q1) are summed in the caller's order."""
    import cf_b200

    d = load_op("cfg1_k3_l4_g0")
    NQ, K = d["NQ"], d["K"]
    rng = np.random.default_rng(1)
    perm = rng.permutation(d["labels"].shape[0])
    lab = np.asfortranarray(d["labels"][perm])
    vals, ic = d["vals"][perm], d["ic_map"][perm]
    Qo = np.zeros((NQ, K), order="F")
    oracle_lib.af(Qo, d["f"], lab, vals, ic, d["R"], NQ, K)
    Qg = np.zeros((NQ, K), order="F")
    cf_b200.contract_batched(Qg, d["f"], lab, vals, ic, d["R"], NQ, K, form="af_exact")
    assert np.array_equal(Qg, Qo)
    Qg = np.zeros((NQ, K), order="F")
    cf_b200.angular_first_collision_kernel_mex(Qg, d["f"], lab, vals, ic, d["R"], NQ, K)
    assert normwise_err(Qg, Qo) <= TOL_FP64


def test_edge_cases(cuda_available):
    import cf_b200
    from cf_b200 import CFError

    d = load_op("wcu_k2_l2_g0")
    NQ, K = d["NQ"], d["K"]
    args = (d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    # empty COO: Q unchanged
    Q = np.full((NQ, K), 3.0, order="F")
    cf_b200.angular_first_collision_kernel_mex(Q, d["f"], np.zeros((0, 3), order="F"), np.zeros(0), np.zeros(0),
                                               d["R"], NQ, K)
    assert np.all(Q == 3.0)
    # empty batch
    Qb = np.zeros((NQ, K, 0), order="F")
    cf_b200.contract_batched(Qb, np.zeros((NQ, K, 0), order="F"), *args)
    # one entry
    lab1 = np.asfortranarray(d["labels_sorted"][5:6])
    Q1 = np.zeros((NQ, K), order="F")
    cf_b200.contract_batched(Q1, d["f"], lab1, d["vals_sorted"][5:6], d["ic_map_sorted"][5:6], d["R"], NQ, K,
                             form="af_exact")
    from oracle.reference import Oracle

    Qo = np.zeros((NQ, K), order="F")
    Oracle().af(Qo, d["f"], lab1, d["vals_sorted"][5:6], d["ic_map_sorted"][5:6], d["R"], NQ, K)
    assert np.array_equal(Q1, Qo)
    # bad indices are rejected with a status, not read out of bounds
    bad = d["labels_sorted"].copy(order="F")
    bad[3, 1] = NQ + 1
    with pytest.raises(CFError) as e:
        cf_b200.angular_first_collision_kernel_mex(np.zeros((NQ, K), order="F"), d["f"], bad, d["vals_sorted"],
                                                   d["ic_map_sorted"], d["R"], NQ, K)
    assert e.value.status == 3
    badic = d["ic_map_sorted"].copy()
    badic[0] = 999
    with pytest.raises(CFError) as e:
        cf_b200.angular_first_collision_kernel_mex(np.zeros((NQ, K), order="F"), d["f"], d["labels_sorted"],
                                                   d["vals_sorted"], badic, d["R"], NQ, K)
    assert e.value.status == 3
    badv = d["vals_sorted"].copy()
    badv[2] = np.nan
    with pytest.raises(CFError) as e:
        cf_b200.angular_first_collision_kernel_mex(np.zeros((NQ, K), order="F"), d["f"], d["labels_sorted"], badv,
                                                   d["ic_map_sorted"], d["R"], NQ, K)
    assert e.value.status == 4
    with pytest.raises(CFError):
        cf_b200.angular_first_collision_kernel_mex(np.zeros((NQ, K)), d["f"], *args)  # C-order Q_out rejected


def test_conservation_rows_give_exact_zero_invariants(cuda_available):
    """R rows of mass, momentum and energy are zero, so those Q entries are exactly 0 (src/GeneralCollisionTensor.m:184-191)."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    d = load_op("hs_k4_l4_g1")
    NQ, K = d["NQ"], d["K"]
    op = cf_b200.CollisionOperator(d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    f = torch.from_numpy(workloads.maxwellian_cells(K, d["L"], 100, seed=4, amplitude=0.1)).cuda()
    Q = op.q(f)
    inv = Q.reshape(100, -1)[:, [0, 1, 2, 3, NQ]].cpu().numpy()
    assert np.all(inv == 0.0)


def test_operator_device_api_and_determinism(cuda_available, oracle_lib):
    import torch

    import cf_b200
    from cf_b200 import workloads

    d = load_op("hs_k4_l4_g1")
    NQ, K = d["NQ"], d["K"]
    op = cf_b200.CollisionOperator(d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    assert op.n_slices > 0 and op.flops_q > 0
    cells = workloads.maxwellian_cells(K, d["L"], 70, seed=8)
    f = torch.from_numpy(cells).cuda()
    Q1 = op.q(f)
    Q2 = op.q(f)
    assert torch.equal(Q1, Q2), "the atomic-free path must be deterministic"
    ws = torch.empty(op.workspace_bytes(70) // 8 + 1, dtype=torch.float64, device="cuda")
    Q3 = op.q(f, workspace=ws)
    assert torch.equal(Q1, Q3)
    Qo = np.zeros((NQ, K, 70), order="F")
    oracle_lib.af_batch(Qo, _cells_cm(cells), d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    assert per_cell_err(Q1.cpu().numpy(), Qo.transpose(2, 1, 0)) <= TOL_FP64
    # += semantics on device
    Q4 = Q1.clone()
    op.q(f, out=Q4)
    assert per_cell_err(Q4.cpu().numpy(), 2 * Q1.cpu().numpy()) <= 1e-14
    # quadratic homogeneity Q(a f) = a^2 Q(f) and J(f) f = 2 Q(f)
    Qa = op.q(3.0 * f)
    assert per_cell_err(Qa.cpu().numpy(), 9.0 * Q1.cpu().numpy()) <= 1e-14
    J = op.jv(f, f)
    assert per_cell_err(J.cpu().numpy(), 2.0 * Q1.cpu().numpy()) <= 1e-14
    op.close()


@pytest.mark.parametrize("L,K,B", [(4, 4, 1), (4, 4, 33), (6, 6, 97), (8, 6, 300), (8, 8, 40), (10, 8, 2500)])
def test_kernel_paths_agree(L, K, B, cuda_available, oracle_lib):
    """The pair kernel, the tile-resident kernel and the gather kernel all match the oracle (fast:
    1e-12; exact: bitwise).  The batch sizes exercise whole half-tile units, quarter and sixteenth
    bins, and a last tile with padding cells."""
    import torch

    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=3 * L + K)
    NQ = geo.n_q
    cells = workloads.maxwellian_cells(K, L, B, seed=B + K)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    f = torch.from_numpy(cells).cuda()
    Qo = np.zeros((NQ, K, B), order="F")
    oracle_lib.af_batch(Qo, _cells_cm(cells), geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    ref = Qo.transpose(2, 1, 0)
    outs = {}
    for path in ("tile_mma", "pair_split", "pair", "pair_l1", "tile", "gather"):
        op.set_kernel_path(path)
        Qf = op.q(f).cpu().numpy()
        assert per_cell_err(Qf, ref) <= TOL_FP64, f"{path}: {per_cell_err(Qf, ref):.3e}"
        Qs = op.q(f, form="af_sym").cpu().numpy()
        assert per_cell_err(Qs, ref) <= TOL_FP64, f"{path} folded: {per_cell_err(Qs, ref):.3e}"
        outs[path] = op.q(f, form="af_exact").cpu().numpy()
        assert np.array_equal(outs[path], ref), f"{path}: exact form not bitwise equal to the oracle"
    op.close()


@pytest.mark.parametrize("L,K,B", [(8, 8, 70), (6, 6, 40)])
def test_tile_path_jacobian(L, K, B, cuda_available, oracle_lib):
    import torch

    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=11)
    NQ = geo.n_q
    cells = workloads.maxwellian_cells(K, L, B, seed=4)
    rng = np.random.default_rng(6)
    v = rng.standard_normal(cells.shape)
    ref = np.zeros((NQ, K, B), order="F")
    oracle_lib.jv_batch(ref, _cells_cm(cells), _cells_cm(v), geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    ref = ref.transpose(2, 1, 0)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    ft, vt = torch.from_numpy(cells).cuda(), torch.from_numpy(v).cuda()
    for path in ("pair", "pair_l1", "tile"):
        op.set_kernel_path(path)
        assert per_cell_err(op.jv(ft, vt).cpu().numpy(), ref) <= TOL_FP64
        assert np.array_equal(op.jv(ft, vt, exact=True).cpu().numpy(), ref)
    op.close()


def test_folded_form_rejects_an_asymmetric_list(cuda_available):
    """A COO list that is not symmetric in (q2, q3) cannot be folded: CF_EUNSUPPORTED, not a wrong answer."""
    import cf_b200
    from cf_b200 import CFError

    d = load_op("cfg1_k3_l4_g0")
    NQ, K = d["NQ"], d["K"]
    keep = np.ones(d["labels"].shape[0], dtype=bool)
    lab = d["labels"]
    off = np.flatnonzero(lab[:, 1] != lab[:, 2])[0]
    keep[off] = False  # drop one entry: its mirror is left without a partner
    Q = np.zeros((NQ, K), order="F")
    with pytest.raises(CFError) as e:
        cf_b200.contract_batched(Q, d["f"], np.asfortranarray(lab[keep]), d["vals"][keep], d["ic_map"][keep], d["R"],
                                 NQ, K, form="af_sym")
    assert e.value.status == 8


def test_pair_path_with_unpaired_rows(cuda_available, oracle_lib):
    """A shuffled COO list breaks the mirrored-row structure: rows fall back to single items and the
    result is unchanged (exact form bitwise, in the caller's run order)."""
    import torch

    import cf_b200
    from cf_b200 import workloads

    d = load_op("hs_k4_l4_g1")
    NQ, K = d["NQ"], d["K"]
    rng = np.random.default_rng(4)
    perm = rng.permutation(d["labels"].shape[0])
    lab = np.asfortranarray(d["labels"][perm])
    vals, ic = d["vals"][perm], d["ic_map"][perm]
    cells = workloads.maxwellian_cells(K, d["L"], 50, seed=2)
    ref = np.zeros((NQ, K, 50), order="F")
    oracle_lib.af_batch(ref, _cells_cm(cells), lab, vals, ic, d["R"], NQ, K)
    op = cf_b200.CollisionOperator(lab, vals, ic, d["R"], NQ, K)
    op.set_kernel_path("pair")
    out = op.q(torch.from_numpy(cells).cuda(), form="af_exact").cpu().numpy()
    assert np.array_equal(out, ref.transpose(2, 1, 0))
    op.set_kernel_path("pair_split")  # single rows use all 32 lanes, k3 split over the half-warps
    out = op.q(torch.from_numpy(cells).cuda()).cpu().numpy()
    assert per_cell_err(out, ref.transpose(2, 1, 0)) <= TOL_FP64
    op.close()


@pytest.mark.parametrize("L,K,B", [(8, 8, 50), (10, 8, 40), (16, 12, 13)])
def test_fp32_forms_error_and_invariants(L, K, B, cuda_available, oracle_lib):
    """FP32 forms: relative error at FP32 level (<= 1e-5 per cell), invariant rows exactly zero."""
    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=2)
    NQ = geo.n_q
    f = _cells_cm(workloads.maxwellian_cells(K, L, B, seed=6, amplitude=0.05))
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, *args)
    for form in ("af_f32", "af_sym_f32"):
        Qg = np.zeros_like(f, order="F")
        cf_b200.contract_batched(Qg, f, *args, form=form)
        err = per_cell_err(Qg.transpose(2, 1, 0), Qo.transpose(2, 1, 0))
        assert 1e-12 < err <= 1e-5, f"{form}: {err:.3e}"
        inv = Qg.transpose(2, 1, 0).reshape(B, -1)[:, [0, 1, 2, 3, NQ]]
        assert np.all(inv == 0.0)


@pytest.mark.parametrize("L,K,B", [(4, 8, 33), (8, 8, 50), (10, 8, 300)])
def test_bf16_split_forms_error_and_invariants(L, K, B, cuda_available, oracle_lib):
    """BF16-split forms (K^3 step on the BF16 tensor cores, R and Phi as hi + lo): relative error
    near FP32's (<= 1e-4 per cell), invariant rows exactly zero, other K refused."""
    import cf_b200
    from cf_b200 import CFError, geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=4)
    NQ = geo.n_q
    f = _cells_cm(workloads.maxwellian_cells(K, L, B, seed=9, amplitude=0.05))
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, *args)
    for form in ("af_bf16", "af_sym_bf16"):
        Qg = np.asfortranarray(np.full_like(f, 0.125))  # += semantics
        cf_b200.contract_batched(Qg, f, *args, form=form)
        Qg -= 0.125
        err = per_cell_err(Qg.transpose(2, 1, 0), Qo.transpose(2, 1, 0))
        assert 1e-12 < err <= 1e-4, f"{form}: {err:.3e}"
        inv = Qg.transpose(2, 1, 0).reshape(B, -1)[:, [0, 1, 2, 3, NQ]]
        assert np.all(inv == 0.0)
    geo6 = geometry.sort_for_contraction(geometry.generate_geometry(4))
    R6 = workloads.synthetic_R(rtensor.l_triplets_of(geo6), 6, seed=1)
    f6 = _cells_cm(workloads.maxwellian_cells(6, 4, 3, seed=1))
    with pytest.raises(CFError) as e:
        cf_b200.contract_batched(np.zeros_like(f6, order="F"), f6, geo6.labels, geo6.vals, geo6.ic_map, R6,
                                 geo6.n_q, 6, form="af_bf16")
    assert e.value.status == 8


def test_host_entry_chunked_matches_oracle(cuda_available, oracle_lib):
    """Batches of >= 1024 cells go through the host entry points in chunks on three streams; the
    result is the same as the oracle's (fast and folded Q, J.v), cells split at ragged chunk ends."""
    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    L, K, B = 4, 4, 1500
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=21)
    NQ = geo.n_q
    f = _cells_cm(workloads.maxwellian_cells(K, L, B, seed=8))
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, *args)
    for form in ("af", "af_sym", "af_exact"):
        Qg = np.asfortranarray(np.full_like(f, 0.5))
        cf_b200.contract_batched(Qg, f, *args, form=form)
        Qg -= 0.5
        assert per_cell_err(Qg.transpose(2, 1, 0), Qo.transpose(2, 1, 0)) <= TOL_FP64, form
    rng = np.random.default_rng(2)
    v = np.asfortranarray(rng.standard_normal(f.shape))
    Jo = np.zeros_like(f, order="F")
    oracle_lib.jv_batch(Jo, f, v, *args)
    Jg = np.zeros_like(f, order="F")
    cf_b200.collision_jacobian_apply_mex(Jg, f, v, *args)
    assert per_cell_err(Jg.transpose(2, 1, 0), Jo.transpose(2, 1, 0)) <= TOL_FP64
    Je = np.zeros_like(f, order="F")
    cf_b200.collision_jacobian_apply_mex(Je, f, v, *args, exact=1)
    assert np.array_equal(Je, Jo)


def test_two_streams_share_a_plan(cuda_available):
    """Persistent launches of one plan on two streams at once each get their own work counter."""
    import torch

    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    L, K = 8, 8
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=5)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    op.set_kernel_path("pair_split")
    f1 = torch.from_numpy(workloads.maxwellian_cells(K, L, 600, seed=1)).cuda()
    f2 = torch.from_numpy(workloads.maxwellian_cells(K, L, 700, seed=2)).cuda()
    ref1, ref2 = op.q(f1), op.q(f2)
    torch.cuda.synchronize()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    ws1 = torch.empty(op.workspace_bytes(600) // 8 + 8, dtype=torch.float64, device="cuda")
    ws2 = torch.empty(op.workspace_bytes(700) // 8 + 8, dtype=torch.float64, device="cuda")
    outs1 = [torch.zeros_like(f1) for _ in range(4)]
    outs2 = [torch.zeros_like(f2) for _ in range(4)]
    for o1, o2 in zip(outs1, outs2):
        op.q(f1, out=o1, stream=s1, workspace=ws1)
        op.q(f2, out=o2, stream=s2, workspace=ws2)
    torch.cuda.synchronize()
    assert all(torch.equal(o, ref1) for o in outs1)
    assert all(torch.equal(o, ref2) for o in outs2)
    op.close()


@pytest.mark.parametrize("L,K,B", [(10, 8, 37), (10, 8, 300), (16, 4, 45)])
def test_quarter_tile_jacobian_vs_oracle(L, K, B, cuda_available, oracle_lib):
    """Where f and v do not fit as 16-cell tiles (L = 10 at K = 8), J.v runs on the 8-cell quarter-tile
    kernel (plain and folded operator); it must match the oracle like every other family."""
    import torch

    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=L + K)
    NQ = geo.n_q
    cells = workloads.maxwellian_cells(K, L, B, seed=11)
    rng = np.random.default_rng(3)
    vc = rng.standard_normal(cells.shape)
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    ref = np.zeros((NQ, K, B), order="F")
    oracle_lib.jv_batch(ref, _cells_cm(cells), _cells_cm(vc), *args)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    f, v = torch.from_numpy(cells).cuda(), torch.from_numpy(vc).cuda()
    for folded in (False, True):
        out = op.jv(f, v, folded=folded).cpu().numpy()
        assert cf_b200._lib.PATH_NAMES[op.info()["last_path"]] == "tile_quarter", folded
        assert per_cell_err(out, ref.transpose(2, 1, 0)) <= TOL_FP64, folded
    op.close()


def test_quarter_tile_q_vs_oracle(cuda_available, oracle_lib):
    """Q where neither the 16-cell tile nor the pair kernel fits (L = 16, K = 8): the quarter-tile
    kernel, plain and folded, against the oracle."""
    import torch

    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    L, K, B = 16, 8, 21
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=4)
    NQ = geo.n_q
    cells = workloads.maxwellian_cells(K, L, B, seed=12)
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    ref = np.zeros((NQ, K, B), order="F")
    oracle_lib.af_batch(ref, _cells_cm(cells), *args)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    f = torch.from_numpy(cells).cuda()
    for form in ("af", "af_sym"):
        out = op.q(f, form=form).cpu().numpy()
        assert cf_b200._lib.PATH_NAMES[op.info()["last_path"]] == "tile_quarter", form
        assert per_cell_err(out, ref.transpose(2, 1, 0)) <= TOL_FP64, form
    op.close()
