"""cf_ragged_q_host: a ragged batch from host arrays.

With the tile routine and every bucket fused, the buckets stream through one launch while they are
copied in and out; the result must equal the device step (cf_ragged_q) bit for bit, on repeated calls,
with nonzero Q on entry and ragged half-tile ends.  Any other handle copies up, runs the device step
and copies back.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

BUCKETS = [(4, 4), (6, 6), (8, 6), (10, 8)]


def _ops(buckets, seed=0):
    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    ops = []
    for i, (L, K) in enumerate(buckets):
        geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
        R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed + i)
        ops.append((geo, R, cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)))
    return ops


def _inputs(buckets, cells, seed):
    from cf_b200 import workloads

    rng = np.random.default_rng(seed)
    fs = [workloads.maxwellian_cells(K, L, c, seed=seed + c) for (L, K), c in zip(buckets, cells)]
    q0 = [rng.standard_normal(f.shape) * 1e-3 for f in fs]
    return fs, q0


@pytest.mark.parametrize("cells,tail_split", [([700, 530, 350, 180], 4), ([41, 30, 19, 10], 16),
                                              ([700, 530, 350, 180], 0), ([0, 530, 0, 181], 4)])
def test_streamed_ragged_host_equals_device_step(cells, tail_split, cuda_available, oracle_lib):
    import torch

    import cf_b200
    from cf_b200.ragged import RaggedBatch

    ops = _ops(BUCKETS)
    fs, q0 = _inputs(BUCKETS, cells, seed=3)
    rb = RaggedBatch([o for _, _, o in ops], cells, forms=["af_sym"] * 4, tail_split=tail_split, family="tile")
    qd = [torch.from_numpy(q.copy()).cuda() for q in q0]
    rb.q([torch.from_numpy(f).cuda() for f in fs], qd)
    qd = [q.cpu().numpy() for q in qd]
    fh = [torch.from_numpy(f).pin_memory() for f in fs]
    for call in range(2):
        qh = [torch.from_numpy(q.copy()).pin_memory() for q in q0]
        n0 = cf_b200.launch_count()
        rb.q_host(fh, qh)
        if call == 1:
            assert cf_b200.launch_count() - n0 == 1  # one launch for every bucket
        for b in range(4):
            assert np.array_equal(qh[b].numpy(), qd[b]), f"call {call}, bucket {b}"
    # and the oracle agrees on the largest bucket
    geo, R, _ = ops[3]
    L, K = BUCKETS[3]
    if cells[3]:
        Qo = np.zeros((geo.n_q, K, cells[3]), order="F")
        oracle_lib.af_batch(Qo, np.asfortranarray(fs[3].transpose(2, 1, 0)), geo.labels, geo.vals, geo.ic_map, R,
                            geo.n_q, K)
        assert per_cell_err(qh[3].numpy() - q0[3], Qo.transpose(2, 1, 0)) <= 1e-12


def test_ragged_host_other_handles_copy_and_step(cuda_available):
    """The pair routine (and pageable numpy arrays): copies up, the device step, copies back."""
    import torch

    import cf_b200
    from cf_b200.ragged import RaggedBatch

    cells = [300, 200, 120, 70]
    ops = _ops(BUCKETS, seed=5)
    fs, q0 = _inputs(BUCKETS, cells, seed=7)
    rb = RaggedBatch([o for _, _, o in ops], cells, forms=["af_sym"] * 4, tail_split=4, family="pair")
    qd = [torch.from_numpy(q.copy()).cuda() for q in q0]
    rb.q([torch.from_numpy(f).cuda() for f in fs], qd)
    qh = [q.copy() for q in q0]
    rb.q_host(fs, qh)
    n0 = cf_b200.launch_count()
    qh2 = [q.copy() for q in q0]
    rb.q_host(fs, qh2)
    assert cf_b200.launch_count() - n0 > 1
    for b in range(4):
        assert np.array_equal(qh[b], qd[b].cpu().numpy()) and np.array_equal(qh2[b], qh[b])
