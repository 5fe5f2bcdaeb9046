"""The few-cell kernel: batches of at most 8 cells (one f per call, as the reference's MEX is called)
contracted in one launch on the cell-major arrays, from device arrays and from host arrays.

The fast FP64 forms (angular first, plain and q2 <-> q3 folded; radial first) must agree with the
oracle to 1e-12 normwise per cell, give the same bits from the device entry point and the host call,
and take one launch.  What the kernel does not take (the exact order, J.v, radial first above K = 8,
more than 8 cells) keeps its own kernels.  An operator changed in place between host calls (the
host call guesses the plan from the array addresses) must be seen.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_op, normwise_err, per_cell_err

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def _setup(L, K, B, seed):
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = np.asfortranarray(workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed))
    cells = workloads.maxwellian_cells(K, L, B, seed=seed + 1)  # [B, K, N_Q]
    q0 = np.random.default_rng(seed + 2).standard_normal(cells.shape) * 1e-3
    return geo, R, cells, q0


def _oracle(oracle_lib, geo, R, cells, K, form):
    f_cm = np.asfortranarray(cells.transpose(2, 1, 0))
    Qo = np.zeros_like(f_cm, order="F")
    oracle_lib.af_batch(Qo, f_cm, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, form="rf" if form == "rf" else "af")
    return Qo.transpose(2, 1, 0)


# f and Q_in of the host call travel in the launch's parameter block up to 3968 doubles (2 B M); above
# that, (10, 8, 3) and (8, 8, 8), they go through the copy route
@pytest.mark.parametrize("L,K,B", [(4, 4, 1), (4, 4, 3), (2, 2, 8), (6, 6, 5), (8, 8, 1), (10, 8, 2), (6, 12, 1),
                                   (4, 16, 3), (3, 5, 2), (10, 8, 3), (8, 8, 8)])
@pytest.mark.parametrize("form", ["af", "af_sym", "rf"])
def test_few_cells_device_and_host_vs_oracle(L, K, B, form, cuda_available, oracle_lib):
    import torch

    import cf_b200

    geo, R, cells, q0 = _setup(L, K, B, seed=7 * L + K + B)
    Qo = _oracle(oracle_lib, geo, R, cells, K, form)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    f = torch.from_numpy(cells).cuda()
    Qd = torch.from_numpy(q0.copy()).cuda()
    op.q(f, out=torch.zeros_like(f), form=form)  # builds the folded operator on first use
    n0 = cf_b200.launch_count()
    op.q(f, out=Qd, form=form)
    torch.cuda.synchronize()
    few = not (form == "rf" and K > 8)
    if few:
        assert cf_b200.launch_count() - n0 == 1
        assert cf_b200._lib.PATH_NAMES[op.info()["last_path"]] == "few" or form == "rf"
    qd = Qd.cpu().numpy()
    assert per_cell_err(qd - q0, Qo) <= TOL_FP64
    # the host call: the same contraction, f and Q_in in the launch's parameter block or copied, the same bits
    f_cm = np.asfortranarray(cells.transpose(2, 1, 0))
    route = "none" if not few else ("parameter block" if 2 * B * geo.n_q * K <= 3968 else "copies")
    for _ in range(2):  # the second call guesses the plan from the array addresses
        Qh = np.array(q0.transpose(2, 1, 0), order="F")
        cf_b200.contract_batched(Qh, f_cm, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, form=form)
        assert cf_b200.few_route_last() == route
        assert np.array_equal(Qh.transpose(2, 1, 0), qd)
    op.close()


@pytest.mark.parametrize("name", ["wcu_k2_l2_g0", "cfg1_k3_l4_g0", "hs_k4_l4_g1", "bkw_k5_l1_g0"])
def test_single_f_mex_calls_take_one_launch(name, cuda_available):
    import cf_b200

    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    args = (d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    for fn, key in ((cf_b200.angular_first_collision_kernel_mex, "Q_af"), (cf_b200.radial_first_collision_kernel_mex,
                                                                          "Q_rf")):
        fn(np.zeros((NQ, K), order="F"), d["f"], *args)
        Q = np.zeros((NQ, K), order="F")
        n0 = cf_b200.launch_count()
        fn(Q, d["f"], *args)
        assert cf_b200.launch_count() - n0 == 1, key
        assert cf_b200.few_route_last() == "parameter block", key
        assert normwise_err(Q, d[key]) <= TOL_FP64, key
        # Q_out += : a second call on the same Q doubles the contraction
        fn(Q, d["f"], *args)
        assert normwise_err(Q, 2 * d[key]) <= TOL_FP64, key


def test_outside_the_few_cell_kernel(cuda_available, oracle_lib):
    """More than 8 cells and J.v keep their kernels (more than one launch here); the exact order of
    one cell runs on the few-cell exact kernel, bit for bit the oracle's operation order."""
    import torch

    import cf_b200

    L, K = 4, 4
    geo, R, cells, q0 = _setup(L, K, 9, seed=3)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    f = torch.from_numpy(cells).cuda()
    Qo = _oracle(oracle_lib, geo, R, cells, K, "af")
    Q = torch.zeros_like(f)
    op.q(f, out=Q, form="af")
    n0 = cf_b200.launch_count()
    Q.zero_()
    op.q(f, out=Q, form="af")
    torch.cuda.synchronize()
    assert cf_b200.launch_count() - n0 > 1
    assert cf_b200._lib.PATH_NAMES[op.info()["last_path"]] != "few"
    assert per_cell_err(Q.cpu().numpy(), Qo) <= TOL_FP64
    for B in (1, 3):
        Qe = torch.zeros_like(f[:B])
        n0 = cf_b200.launch_count()
        op.q(f[:B].contiguous(), out=Qe, form="af_exact")
        torch.cuda.synchronize()
        assert cf_b200.launch_count() - n0 == 1
        assert cf_b200._lib.PATH_NAMES[op.info()["last_path"]] == "few"
        assert np.array_equal(Qe.cpu().numpy(), Qo[:B])
    v = torch.from_numpy(np.random.default_rng(4).standard_normal(cells[:1].shape)).cuda()
    f1 = f[:1].contiguous()
    J = op.jv(f1, v)
    eps = 1e-6
    fd = (op.q(f1 + eps * v) - op.q(f1 - eps * v)) / (2 * eps)
    assert normwise_err(J.cpu().numpy(), fd.cpu().numpy()) <= 1e-6
    op.close()


def test_few_cell_host_call_sees_an_operator_changed_in_place(cuda_available):
    import torch

    import cf_b200

    L, K, B = 4, 4, 1
    geo, R, cells, q0 = _setup(L, K, B, seed=11)
    labels = np.asfortranarray(geo.labels)
    vals = np.array(geo.vals)
    ic = np.array(geo.ic_map)
    Rf = np.asfortranarray(R)
    f_cm = np.asfortranarray(cells.transpose(2, 1, 0))

    def host():
        Q = np.array(q0.transpose(2, 1, 0), order="F")
        cf_b200.contract_batched(Q, f_cm, labels, vals, ic, Rf, geo.n_q, K, form="af")
        return Q.transpose(2, 1, 0)

    def device():
        op = cf_b200.CollisionOperator(labels, vals, ic, Rf, geo.n_q, K)
        Qd = torch.from_numpy(q0.copy()).cuda()
        op.q(torch.from_numpy(cells).cuda(), out=Qd, form="af")
        op.close()
        return Qd.cpu().numpy()

    first = host()
    assert np.array_equal(host(), device())  # same arrays: the guess holds
    Rf *= 1.5  # same addresses, new content
    vals *= 0.75
    changed = host()
    assert np.array_equal(changed, device())
    assert not np.array_equal(changed, first)


@pytest.mark.parametrize("name", ["wcu_k2_l2_g0", "cfg1_k3_l4_g0", "hs_k4_l4_g1", "bkw_k5_l1_g0"])
def test_single_f_exact_host_call_is_the_reference_bit_for_bit(name, cuda_available):
    import cf_b200

    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    args = (d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    for _ in range(2):  # the second call guesses the plan from the array addresses
        Q = np.zeros((NQ, K), order="F")
        n0 = cf_b200.launch_count()
        cf_b200.contract_batched(Q, d["f"], *args, form="af_exact")
        assert cf_b200.launch_count() - n0 == 1
        assert cf_b200.few_route_last() == "parameter block"
        assert np.array_equal(Q, d["Q_af"])


def test_time_contract_host_runs_the_calls_it_times(cuda_available):
    """cf_time_contract_host: n back-to-back cf_contract_host calls, each adding into Q."""
    import ctypes

    import cf_b200
    from cf_b200 import _lib

    d = load_op("cfg1_k3_l4_g0")
    NQ, K = d["NQ"], d["K"]
    lab = np.asfortranarray(d["labels_sorted"])
    vals, ic = np.ascontiguousarray(d["vals_sorted"]), np.ascontiguousarray(d["ic_map_sorted"])
    R, f = np.asfortranarray(d["R"]), np.asfortranarray(d["f"])
    Q = np.zeros((NQ, K), order="F")
    Dp = ctypes.POINTER(ctypes.c_double)
    secs = ctypes.c_double(-1.0)
    st = _lib.load().cf_time_contract_host(5, ctypes.byref(secs), Q.ctypes.data_as(Dp), f.ctypes.data_as(Dp), 1,
                                           lab.ctypes.data_as(Dp), vals.ctypes.data_as(Dp), ic.ctypes.data_as(Dp),
                                           R.ctypes.data_as(Dp), lab.shape[0], R.size // K ** 3, NQ, K,
                                           _lib.FORMS["af"])
    assert st == 0 and secs.value > 0.0
    assert cf_b200.few_route_last() == "parameter block"
    assert normwise_err(Q, 5 * d["Q_af"]) <= TOL_FP64


def test_rows_without_slices_pass_through(cuda_available, oracle_lib):
    """One COO entry: every other row of Q has no slice and must come back as it went in, from the
    host call (f and Q_in in the parameter block, Q_out a separate buffer) and the device call."""
    import torch

    import cf_b200

    d = load_op("cfg1_k3_l4_g0")
    NQ, K = d["NQ"], d["K"]
    lab1 = np.asfortranarray(d["labels_sorted"][7:8])
    vals1, ic1 = d["vals_sorted"][7:8], d["ic_map_sorted"][7:8]
    q0 = np.asfortranarray(np.random.default_rng(5).standard_normal((NQ, K)))
    Qo = q0.copy(order="F")
    oracle_lib.af(Qo, d["f"], lab1, vals1, ic1, d["R"], NQ, K)
    Qh = q0.copy(order="F")
    cf_b200.angular_first_collision_kernel_mex(Qh, d["f"], lab1, vals1, ic1, d["R"], NQ, K)
    assert cf_b200.few_route_last() == "parameter block"
    q1 = int(lab1[0, 0]) - 1
    others = [q for q in range(NQ) if q != q1]
    assert np.array_equal(Qh[others], q0[others])
    assert normwise_err(Qh, Qo) <= TOL_FP64
    op = cf_b200.CollisionOperator(lab1, vals1, ic1, d["R"], NQ, K)
    Qd = torch.from_numpy(np.ascontiguousarray(q0.T).reshape(1, K, NQ).copy()).cuda()
    op.q(torch.from_numpy(np.ascontiguousarray(d["f"].T).reshape(1, K, NQ).copy()).cuda(), out=Qd, form="af")
    assert np.array_equal(Qd.cpu().numpy().reshape(K, NQ).T, Qh)
    op.close()


@pytest.mark.parametrize("name", ["cfg1_k3_l4_g0", "hs_k4_l4_g1"])
def test_single_f_exact_adds_into_nonzero_q_bit_for_bit(name, cuda_available, oracle_lib):
    """The exact few-cell kernels start from Q_in and add each slice's sum in the reference's order
    (Q[q1] += q_val, angular_first_collision_kernel_mex.cpp:68): with a nonzero, non-round Q_in the
    host call (Q_in in the parameter block) and the in-place device call both equal the oracle run
    on the same Q_in, bit for bit."""
    import torch

    import cf_b200

    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    args = (d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    q0 = np.asfortranarray(np.random.default_rng(21).standard_normal((NQ, K)) * (np.pi / 7.0))
    Qo = q0.copy(order="F")
    oracle_lib.af(Qo, d["f"], *args)
    Qh = q0.copy(order="F")
    cf_b200.contract_batched(Qh, d["f"], *args, form="af_exact")
    assert cf_b200.few_route_last() == "parameter block"
    assert np.array_equal(Qh, Qo), np.abs(Qh - Qo).max()
    op = cf_b200.CollisionOperator(*args)
    B = 3
    fb = np.stack([np.ascontiguousarray(d["f"].T)] * B)  # [B, K, NQ]
    qb = np.stack([np.ascontiguousarray(q0.T) * (1.0 + 0.25 * b) for b in range(B)])
    Qd = torch.from_numpy(qb.copy()).cuda()
    op.q(torch.from_numpy(fb.copy()).cuda(), out=Qd, form="af_exact")
    got = Qd.cpu().numpy()
    op.close()
    for b in range(B):
        ref = np.asfortranarray(qb[b].T)
        oracle_lib.af(ref, d["f"], *args)
        assert np.array_equal(got[b].T, ref), (b, np.abs(got[b].T - ref).max())
