"""Implicit solves on the GPU: batched GMRES against a dense solve, preconditioning, conservation."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_op

pytestmark = pytest.mark.gpu


def _dense(name):
    from cf_b200.geometry import Geometry
    from oracle import rtensor

    d = load_op(name)
    geo = Geometry(d["L"], d["labels"], d["vals"], d["ic_map"], d["l_triplets"])
    return d, rtensor.assemble_dense(geo, d["R"], d["K"])


@pytest.fixture(scope="module")
def hs_op():
    import cf_b200

    d, Cd = _dense("hs_k4_l4_g1")
    op = cf_b200.CollisionOperator(d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], d["NQ"], d["K"])
    yield d, Cd, op
    op.close()


def test_gmres_matches_dense_solve(cuda_available, hs_op):
    """(I - dt J(f)) x = b per cell: GMRES(30) to 1e-12 against numpy's dense solve of the assembled operator."""
    import torch

    from cf_b200 import implicit, workloads

    d, Cd, op = hs_op
    K, NQ, L = d["K"], d["NQ"], d["L"]
    N = K * NQ
    B = 37
    cells = workloads.maxwellian_cells(K, L, B, seed=12, amplitude=0.05)
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal(cells.shape)
    dt = 0.7
    x, iters, rel = implicit.gmres_solve(op, torch.from_numpy(cells).cuda(), torch.from_numpy(rhs).cuda(), dt,
                                         restart=30, tol=1e-12, max_iters=2000)
    x = x.cpu().numpy()
    assert np.all(rel <= 1e-12)
    worst = 0.0
    for bcell in range(B):
        fv = cells[bcell].ravel()  # [K, NQ] C order = column-major [NQ x K] = global index k*NQ + q
        J = np.einsum("ijk,k->ij", Cd, fv) + np.einsum("ijk,j->ik", Cd, fv)
        A = np.eye(N) - dt * J
        xr = np.linalg.solve(A, rhs[bcell].ravel())
        worst = max(worst, np.abs(x[bcell].ravel() - xr).max() / np.abs(xr).max())
    assert worst < 1e-9, worst


def test_block_preconditioner_reduces_iterations(cuda_available, hs_op):
    import torch

    from cf_b200 import implicit, workloads

    d, Cd, op = hs_op
    K, L = d["K"], d["L"]
    B = 64
    cells = workloads.stress_cells(K, L, B, seed=5, amplitude=0.1)
    f = torch.from_numpy(cells).cuda()
    rhs = op.q(f)
    J6 = implicit.equilibrium_jacobian_blocks(op)[6]
    nu = abs(J6[0, 0])
    dt = 10.0 / nu
    P = implicit.block_preconditioner(op, dt)
    _, it_none, rel_none = implicit.gmres_solve(op, f, rhs, dt, tol=1e-10)
    _, it_blk, rel_blk = implicit.gmres_solve(op, f, rhs, dt, tol=1e-10, precond=P)
    assert np.all(rel_none <= 1e-10) and np.all(rel_blk <= 1e-10)
    assert it_blk.mean() < it_none.mean()
    # per-cell blocks (the learned preconditioner's format) reproduce the shared-block run exactly
    Pc = np.broadcast_to(P, (B,) + P.shape).copy()
    _, it_pc, rel_pc = implicit.gmres_solve(op, f, rhs, dt, tol=1e-10, precond=Pc)
    assert np.array_equal(it_pc, it_blk)


def test_equilibrium_blocks_match_dense_jacobian(cuda_available, hs_op):
    from cf_b200 import implicit

    d, Cd, op = hs_op
    K, NQ = d["K"], d["NQ"]
    J = Cd[:, :, 0] + Cd[:, 0, :]
    blocks = implicit.equilibrium_jacobian_blocks(op)
    for q in range(NQ):
        idx = np.arange(K) * NQ + q
        ref = J[np.ix_(idx, idx)]
        assert np.abs(blocks[q] - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    # the equilibrium Jacobian couples no two angular modes
    off = J.copy()
    for q in range(NQ):
        idx = np.arange(K) * NQ + q
        off[np.ix_(idx, idx)] = 0.0
    assert np.abs(off).max() < 1e-12 * np.abs(J).max()


def test_backward_euler_relaxation_conserves_invariants(cuda_available, hs_op):
    import torch

    from cf_b200 import basis, implicit, workloads

    d, Cd, op = hs_op
    K, L, NQ = d["K"], d["L"], d["NQ"]
    B = 40
    f0 = torch.from_numpy(workloads.stress_cells(K, L, B, seed=9, amplitude=0.1)).cuda()
    nu = abs(implicit.equilibrium_jacobian_blocks(op)[6][0, 0])
    dt = 1.0 / nu
    P = implicit.block_preconditioner(op, dt)
    f = f0
    inv = basis.invariant_indices(NQ)
    s0 = f0[:, 0, 4:9].abs().amax().item()
    for _ in range(3):
        f, stats = implicit.backward_euler_step(op, f, dt, precond=P)
        assert stats and stats[-1]["relres_max"] <= 1e-10
    drift = (f - f0).reshape(B, -1)[:, inv].abs().max().item()
    assert drift < 1e-13
    s1 = f[:, 0, 4:9].abs().amax().item()
    # linear backward Euler shrinks the stress by 1/(1 + dt nu) per step; three steps ~ 1/8
    assert s1 < 0.2 * s0
