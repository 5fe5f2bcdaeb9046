"""The single-operator kernel autotuner (CollisionOperator.autotune): it times each kernel path for
one form and batch size, sets the fastest, and caches the choice.

Tolerance: 1e-12 normwise per cell against the oracle's restatement of the reference's angular-first
kernel (src/mex/angular_first_collision_kernel_mex.cpp:45-69), whichever path it picks.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,K,form", [(8, 12, "af_sym"), (6, 8, "af")])
def test_kernel_autotune_chooses_and_caches(L, K, form, cuda_available, oracle_lib, tmp_path, monkeypatch):
    import torch

    import cf_b200
    from cf_b200 import geometry, operator, workloads
    from oracle import rtensor

    monkeypatch.setenv("CF_B200_CACHE", str(tmp_path))
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = np.asfortranarray(workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=L))
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    B = 300
    best, rep = op.autotune(B, form=form, reps=2)
    assert best in operator.AUTOTUNE_PATHS and not rep["cached"]
    assert "auto" in rep["seconds"] and best == operator.choose_fastest(rep["seconds"])
    # every timed path gives the operator's result; the chosen one is set on the plan
    cells = workloads.maxwellian_cells(K, L, 37, seed=3)
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    Qo = np.zeros_like(f, order="F")
    oracle_lib.af_batch(Qo, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    Q = op.q(torch.from_numpy(cells).cuda(), form=form).cpu().numpy()
    assert per_cell_err(Q, Qo.transpose(2, 1, 0)) <= 1e-12
    best2, rep2 = op.autotune(B, form=form, reps=2)
    assert rep2["cached"] and best2 == best
    op.close()
