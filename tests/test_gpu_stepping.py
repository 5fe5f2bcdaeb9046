"""Batched explicit RK2 stepping with the GPU operator: the BKW transient and stress relaxation."""
from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_op
from test_kat import dense_of, project_bkw

pytestmark = pytest.mark.gpu


def _cell(c_vec, K, NQ):
    """Column-major [N_Q x K] vector -> [K, N_Q] cell."""
    return c_vec.reshape(NQ, K, order="F").T


def test_bkw_transient_batched(cuda_available):
    """40 BKW cells (alpha_0 from 0.05 to 0.3) stepped with Heun's method to t = 4/mu from a CUDA
    graph track alpha(t) = alpha_0 exp(-mu t / 2) (tutorial_collisions_bwu_solution.m:47-104) and
    keep mass, momentum and energy."""
    import torch

    import cf_b200
    from cf_b200 import basis
    from cf_b200.stepping import RK2Stepper

    d = load_op("bkw_k5_l1_g0")
    K, L, NQ = d["K"], d["L"], d["NQ"]
    op = cf_b200.CollisionOperator(d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    mu = 4.0 * math.pi / 3.0
    alphas = np.linspace(0.05, 0.3, 40)
    f0 = np.stack([_cell(project_bkw(a, K, L), K, NQ) for a in alphas])
    st = RK2Stepper(op, torch.from_numpy(f0).cuda())
    dt = 0.001 / mu
    inv = basis.invariant_indices(NQ)
    for block in range(4):
        st.step_graph(dt, 1000)
        t = (block + 1) * 1000 * dt
        cells = st.cells().cpu().numpy()
        for a0, c in zip(alphas, cells):
            ca = _cell(project_bkw(a0 * math.exp(-mu / 2 * t), K, L), K, NQ)
            assert np.max(np.abs(c - ca)) / np.max(np.abs(ca)) < 1e-7
    c_end = np.stack([c.T.ravel(order="F") for c in cells])
    c_0 = np.stack([c.T.ravel(order="F") for c in f0])
    assert np.max(np.abs(c_end[:, inv] - c_0[:, inv])) < 1e-13
    op.close()


def test_stress_relaxation_matches_dense_oracle(cuda_available):
    """Hard spheres K_max = 4, L = 4: the GPU stepper equals the dense-tensor RK2 of the oracle to
    rounding over 200 steps, eager and graph replays agree bit for bit, invariants stay put."""
    import torch

    import cf_b200
    from cf_b200 import basis, workloads
    from cf_b200.stepping import RK2Stepper

    d, Cd = dense_of("hs_k4_l4_g1")
    K, L, NQ = d["K"], d["L"], d["NQ"]
    N = K * NQ
    Cf = Cd.reshape(N, N * N, order="F")
    J = Cd[:, :, 0] + Cd[:, 0, :]
    mu = abs(J[6, 6])
    dt = 0.005 / mu
    cells = workloads.stress_cells(K, L, 8, seed=3, amplitude=0.3)
    op = cf_b200.CollisionOperator(d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    eager = RK2Stepper(op, torch.from_numpy(cells).cuda())
    graph = RK2Stepper(op, torch.from_numpy(cells).cuda())
    for _ in range(4):
        eager.step(dt, 50)
        graph.step_graph(dt, 50)
    ce, cg = eager.cells(), graph.cells()
    assert torch.equal(ce, cg)
    ref = []
    for cell in cells:
        c = cell.T.ravel(order="F").copy()
        for _ in range(200):
            q1 = Cf @ np.outer(c, c).ravel(order="F")
            ct = c + dt * q1
            q2 = Cf @ np.outer(ct, ct).ravel(order="F")
            c = c + 0.5 * dt * (q1 + q2)
        ref.append(_cell(c, K, NQ))
    ref = np.stack(ref)
    got = ce.cpu().numpy()
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12
    inv = basis.invariant_indices(NQ)
    g = np.stack([c.T.ravel(order="F") for c in got])
    c0 = np.stack([c.T.ravel(order="F") for c in cells])
    assert np.max(np.abs(g[:, inv] - c0[:, inv])) < 1e-13
    op.close()
