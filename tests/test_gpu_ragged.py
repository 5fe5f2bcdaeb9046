"""Ragged batches: one fused persistent launch over mixed resolutions, its CUDA-graph replay and the
per-bucket autotuner."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

BUCKETS = [(4, 4), (6, 6), (8, 6), (10, 8)]
CELLS = [41, 30, 19, 10]


def _bucket_ops(buckets, seed=0):
    import cf_b200
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    ops = []
    for i, (L, K) in enumerate(buckets):
        geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
        R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=seed + i)
        ops.append((geo, R, cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)))
    return ops


def _cells(buckets, cells):
    import torch

    from cf_b200 import workloads

    return [torch.from_numpy(workloads.maxwellian_cells(K, L, c, seed=c)).cuda() for (L, K), c in zip(buckets, cells)]


def _oracle_q(oracle_lib, geo, R, K, f):
    Qo = np.zeros((geo.n_q, K, f.shape[0]), order="F")
    oracle_lib.af_batch(Qo, np.asfortranarray(f.cpu().numpy().transpose(2, 1, 0)), geo.labels, geo.vals, geo.ic_map,
                        R, geo.n_q, K)
    return Qo.transpose(2, 1, 0)


@pytest.mark.parametrize("tail_split,family", [(0, "pair"), (4, "pair"), (16, "pair"), (4, "tile"), (16, "tile")])
def test_ragged_fused_equals_per_bucket_and_oracle(tail_split, family, cuda_available, oracle_lib):
    import torch

    from cf_b200.ragged import RaggedBatch

    ops = _bucket_ops(BUCKETS)
    fs = _cells(BUCKETS, CELLS)
    rb = RaggedBatch([o for _, _, o in ops], CELLS, tail_split=tail_split, family=family)
    qs = [torch.zeros_like(f) for f in fs]
    rb.q(fs, qs)
    for (geo, R, op), f, q, (L, K) in zip(ops, fs, qs, BUCKETS):
        op.set_kernel_path(family)
        assert torch.equal(q, op.q(f)), f"the fused launch must equal the bucket's own {family} kernel bit for bit"
        assert per_cell_err(q.cpu().numpy(), _oracle_q(oracle_lib, geo, R, K, f)) <= 1e-12
    for _ in range(2):  # graph replay: same result, twice
        qg = [torch.zeros_like(f) for f in fs]
        rb.q_graph(fs, qg)
        torch.cuda.synchronize()
        assert all(torch.equal(a, b) for a, b in zip(qg, qs))
    rb.close()


def test_ragged_mixed_forms(cuda_available, oracle_lib):
    """Folded buckets run folded inside the fused launch; a radial-first bucket runs on its own."""
    import torch

    from cf_b200.ragged import RaggedBatch

    forms = ["rf", "af_sym", "af", "af_sym"]
    ops = _bucket_ops(BUCKETS, seed=7)
    fs = _cells(BUCKETS, CELLS)
    rb = RaggedBatch([o for _, _, o in ops], CELLS, forms=forms, tail_split=4, family="pair")
    qs = [torch.full_like(f, 0.25) for f in fs]  # += semantics
    rb.q_graph(fs, qs)
    torch.cuda.synchronize()
    for (geo, R, op), f, q, (L, K), form in zip(ops, fs, qs, BUCKETS, forms):
        op.set_kernel_path("pair")
        ref = op.q(f, out=torch.full_like(f, 0.25), form=form)
        assert torch.equal(q, ref), form
        assert per_cell_err(q.cpu().numpy() - 0.25, _oracle_q(oracle_lib, geo, R, K, f)) <= 1e-12
    rb.close()


def test_ragged_rejects_bad_input(cuda_available):
    import torch

    from cf_b200 import CFError
    from cf_b200.ragged import RaggedBatch

    ops = _bucket_ops(BUCKETS[:2])
    with pytest.raises(CFError):
        RaggedBatch([o for _, _, o in ops], [3, 4], tail_split=5)
    with pytest.raises(CFError):
        RaggedBatch([o for _, _, o in ops], [3, 4], forms=["af", "af_f32"])
    with pytest.raises(CFError):
        RaggedBatch([o for _, _, o in ops], [3, 4], family="gather")
    rb = RaggedBatch([o for _, _, o in ops], [3, 4])
    fs = _cells(BUCKETS[:2], [3, 4])
    with pytest.raises(CFError):
        rb.q(fs, [torch.zeros_like(fs[0]), torch.zeros((5, 6, 49), dtype=torch.float64, device="cuda")])


def test_autotune_chooses_and_caches(cuda_available, tmp_path, monkeypatch):
    from cf_b200 import ragged

    monkeypatch.setenv("CF_B200_CACHE", str(tmp_path))
    ops = [o for _, _, o in _bucket_ops(BUCKETS[:2])]
    forms, tail, family, rep = ragged.autotune(ops, [64, 48], reps=2)
    assert len(forms) == 2 and tail in (0, 4, 16) and family in ("pair", "tile") and not rep["cached"]
    for b in rep["buckets"]:
        for fam, times in b["seconds"].items():
            assert b["chosen"][fam] == min(times, key=times.get)
    assert rep["step_seconds"][f"{family}/{tail}"] == min(rep["step_seconds"].values())
    forms2, tail2, family2, rep2 = ragged.autotune(ops, [64, 48], reps=2)
    assert rep2["cached"] and forms2 == forms and tail2 == tail and family2 == family



def test_ragged_bucket_beyond_k8_with_graph(cuda_available, oracle_lib):
    """A K = 12 bucket (L = 8) runs on its own plan's kernel on the tiled buffers beside the fused launch
    (the gather kernel): eager and two graph replays give the same bits, equal to that plan's gather
    kernel and within 1e-12 of the oracle."""
    import torch

    from cf_b200.ragged import RaggedBatch

    buckets, cells = [(4, 4), (8, 12)], [41, 19]
    ops = _bucket_ops(buckets, seed=11)
    fs = _cells(buckets, cells)
    rb = RaggedBatch([o for _, _, o in ops], cells, forms=["af_sym", "af_sym"], tail_split=4, family="tile")
    qs = [torch.zeros_like(f) for f in fs]
    rb.q(fs, qs)
    torch.cuda.synchronize()
    geo, R, op = ops[1]
    op.set_kernel_path("gather")
    assert torch.equal(qs[1], op.q(fs[1], form="af_sym"))
    for (g, Rb, _), f, q, (L, K) in zip(ops, fs, qs, buckets):
        assert per_cell_err(q.cpu().numpy(), _oracle_q(oracle_lib, g, Rb, K, f)) <= 1e-12
    for _ in range(2):
        qg = [torch.zeros_like(f) for f in fs]
        rb.q_graph(fs, qg)
        torch.cuda.synchronize()
        assert all(torch.equal(a, b) for a, b in zip(qg, qs))
    rb.close()
