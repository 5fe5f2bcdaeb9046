"""The streamed host path: one tile-kernel launch over a whole host batch while it is copied in and out.

cf_contract_host streams batches of >= 512 cells in the folded fast form (the tile kernel): the
result must equal the device entry point's bit for bit (same per-row operations, Q_in read at the
start of each row), for ragged batch ends, pageable and pinned host memory, and nonzero Q on entry.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-12


def _setup(L, K, B, seed):
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed)
    cells = workloads.maxwellian_cells(K, L, B, seed=seed + 1)  # [B, K, N_Q]
    rng = np.random.default_rng(seed + 2)
    q0 = rng.standard_normal(cells.shape) * 1e-3
    return geo, R, cells, q0


@pytest.mark.parametrize("L,K,B", [(4, 4, 513), (3, 2, 777), (6, 6, 2049), (8, 8, 1000), (10, 8, 4096)])
def test_streamed_host_call_equals_device_path(L, K, B, cuda_available, oracle_lib):
    import torch

    import cf_b200

    geo, R, cells, q0 = _setup(L, K, B, seed=10 * L + K)
    NQ = geo.n_q
    args = (geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    # device entry point (tiled kernel)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, NQ, K)
    Qd = torch.from_numpy(q0.copy()).cuda()
    op.q(torch.from_numpy(cells).cuda(), out=Qd, form="af_sym")
    Qd = Qd.cpu().numpy()
    # host entry point (streamed): [N_Q x K x B] column-major views of the same bytes
    f_cm = np.asfortranarray(cells.transpose(2, 1, 0))
    Qh = np.array(q0.transpose(2, 1, 0), order="F")  # a copy: the host call writes it in place
    cf_b200.contract_batched(np.zeros_like(Qh, order="F"), f_cm, *args, form="af_sym")  # builds the plans
    n0 = cf_b200.launch_count()
    cf_b200.contract_batched(Qh, f_cm, *args, form="af_sym")
    assert cf_b200.launch_count() - n0 == 1  # one launch for the whole batch
    assert np.array_equal(Qh.transpose(2, 1, 0), Qd)
    # and the oracle agrees
    Qo = np.zeros_like(f_cm, order="F")
    oracle_lib.af_batch(Qo, f_cm, *args)
    dQ = Qh - q0.transpose(2, 1, 0)
    assert per_cell_err(dQ.transpose(2, 1, 0), Qo.transpose(2, 1, 0)) <= TOL_FP64
    op.close()


def test_streamed_host_call_pinned_memory(cuda_available):
    """Pinned host buffers (asynchronous copies that overlap the kernel) give the same bits."""
    import torch

    import cf_b200

    L, K, B = 10, 8, 3000
    geo, R, cells, q0 = _setup(L, K, B, seed=3)
    args = (geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    f_p = torch.from_numpy(cells).pin_memory()
    q_p = torch.from_numpy(q0).pin_memory()
    Qa = np.array(q0.transpose(2, 1, 0), order="F")
    cf_b200.contract_batched(Qa, np.asfortranarray(cells.transpose(2, 1, 0)), *args, form="af_sym")
    for _ in range(3):  # repeated calls reuse the plan, its buffers and the chunk flags (new epoch each call)
        q_p.copy_(torch.from_numpy(q0))
        cf_b200.contract_batched(q_p.numpy().transpose(2, 1, 0), f_p.numpy().transpose(2, 1, 0), *args,
                                 form="af_sym")
        assert np.array_equal(q_p.numpy().transpose(2, 1, 0), Qa)


def test_streamed_forms_only_where_the_tile_kernel_runs(cuda_available, oracle_lib):
    """The plain fast form (pair kernel first) and the exact form keep the chunked pipeline."""
    import cf_b200

    L, K, B = 6, 6, 1200
    geo, R, cells, q0 = _setup(L, K, B, seed=4)
    args = (geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    f_cm = np.asfortranarray(cells.transpose(2, 1, 0))
    Qo = np.zeros_like(f_cm, order="F")
    oracle_lib.af_batch(Qo, f_cm, *args)
    for form in ("af", "af_exact"):
        Q = np.zeros_like(f_cm, order="F")
        cf_b200.contract_batched(np.zeros_like(Q, order="F"), f_cm, *args, form=form)
        n0 = cf_b200.launch_count()
        cf_b200.contract_batched(Q, f_cm, *args, form=form)
        assert cf_b200.launch_count() - n0 > 1, form
        assert per_cell_err(Q.transpose(2, 1, 0), Qo.transpose(2, 1, 0)) <= TOL_FP64, form


def test_stream_wait_gives_up_and_reports(cuda_available):
    """A batch whose data never arrives: every wait runs out after 1 ms, the kernel returns, the call
    reports CF_ETIMEOUT, and the same plan then contracts correctly."""
    import torch

    import cf_b200

    L, K = 4, 4
    geo, R, cells, _ = _setup(L, K, 40, seed=5)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    assert op.stream_selftest(1e-3) == 9
    assert "did not arrive" in cf_b200._lib.load().cf_last_error().decode()
    f = torch.from_numpy(cells).cuda()
    ref = op.q(f, form="af").cpu().numpy()
    assert op.stream_selftest(1e-3) == 9
    assert np.array_equal(op.q(f, form="af").cpu().numpy(), ref)
    op.close()


def test_operator_changed_in_place_between_calls(cuda_available):
    """The host call guesses the plan from the operator arrays' addresses and checks their content
    while the GPU works; arrays changed in place (same addresses) must still give the new operator's
    result, and Q is written only once the check passed."""
    import torch

    import cf_b200

    L, K, B = 8, 8, 1500
    geo, R, cells, q0 = _setup(L, K, B, seed=6)
    labels = np.asfortranarray(geo.labels)
    vals = np.array(geo.vals)
    ic = np.array(geo.ic_map)
    Rf = np.asfortranarray(R)
    f_cm = np.asfortranarray(cells.transpose(2, 1, 0))

    def host(Rx):
        Q = np.array(q0.transpose(2, 1, 0), order="F")
        cf_b200.contract_batched(Q, f_cm, labels, vals, ic, Rx, geo.n_q, K, form="af_sym")
        return Q

    def device(vx, Rx):
        op = cf_b200.CollisionOperator(labels, vx, ic, Rx, geo.n_q, K)
        Qd = torch.from_numpy(q0.copy()).cuda()
        op.q(torch.from_numpy(cells).cuda(), out=Qd, form="af_sym")
        op.close()
        return Qd.cpu().numpy()

    first = host(Rf)
    assert np.array_equal(host(Rf).transpose(2, 1, 0), device(vals, Rf))  # same arrays: the guess holds
    Rf *= 1.5  # same addresses, new content (kept symmetric in q2 <-> q3, as the folded form needs)
    vals *= 0.75
    changed = host(Rf)
    assert np.array_equal(changed.transpose(2, 1, 0), device(vals, Rf))
    assert not np.array_equal(changed, first)


@pytest.mark.parametrize("L,K,form", [(8, 12, "af_sym"), (8, 12, "af"), (6, 8, "af")])
def test_chunked_host_call_operator_changed_in_place(L, K, form, cuda_available):
    """Forms that do not run on the streamed tile kernel take the chunked pipeline; from the second call
    on it too starts from the plan of the operator arrays' addresses and checks their content while the
    GPU works, holding every download back until the check passed.  Same arrays: bit for bit the
    device entry point's result; arrays changed in place: the new operator's result."""
    import torch

    import cf_b200

    B = 700
    geo, R, cells, q0 = _setup(L, K, B, seed=7 + K)
    labels = np.asfortranarray(geo.labels)
    vals = np.array(geo.vals)
    ic = np.array(geo.ic_map)
    Rf = np.asfortranarray(R)
    f_cm = np.asfortranarray(cells.transpose(2, 1, 0))

    def host():
        Q = np.array(q0.transpose(2, 1, 0), order="F")
        cf_b200.contract_batched(Q, f_cm, labels, vals, ic, Rf, geo.n_q, K, form=form)
        return Q.transpose(2, 1, 0)

    def device():
        op = cf_b200.CollisionOperator(labels, vals, ic, Rf, geo.n_q, K)
        Qd = torch.from_numpy(q0.copy()).cuda()
        op.q(torch.from_numpy(cells).cuda(), out=Qd, form=form)
        op.close()
        return Qd.cpu().numpy()

    first = host()
    assert np.array_equal(host(), first)  # the second call starts from the address guess
    assert np.array_equal(first, device())
    Rf *= 1.5  # same addresses, new content (kept symmetric in q2 <-> q3, as the folded form needs)
    vals *= 0.75
    changed = host()
    assert np.array_equal(changed, device())
    assert not np.array_equal(changed, first)
