"""The learned preconditioner's network: GPU forward/backward against the CPU restatement, the
probe loss and its gradient, and what the trained network gains over the Maxwellian blocks."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_op

pytestmark = pytest.mark.gpu


def test_mlp_forward_backward_match_cpu(cuda_available):
    import torch

    from cf_b200.learned import MLP
    from oracle import mlp as ref

    n_in, hid, n_out, n = 13, 40, 22, 9
    net = MLP(n_in, hid, n_out, max_batch=16, seed=3)
    rng = np.random.default_rng(0)
    flat = net.params()
    flat[:] = rng.uniform(-0.4, 0.4, flat.shape).astype(np.float32)
    net.set_params(flat)
    params = ref.unpack(flat.astype(np.float64), n_in, hid, n_out)
    x = rng.standard_normal((n, n_in)).astype(np.float32)
    dy = rng.standard_normal((n, n_out)).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty((n, n_out), dtype=torch.float32, device="cuda")
    net.forward(xt, yt, train=True)
    y_ref, cache = ref.forward(params, x.astype(np.float64))
    assert np.abs(yt.cpu().numpy() - y_ref).max() <= 1e-5 * max(1.0, np.abs(y_ref).max())
    net.backward(xt, torch.from_numpy(dy).cuda())
    torch.cuda.synchronize()
    g = net.grads().astype(np.float64)
    g_ref = ref.pack_like(ref.backward(params, x.astype(np.float64), cache, dy.astype(np.float64)), n_in, hid, n_out)
    err = np.abs(g - g_ref).max() / np.abs(g_ref).max()
    assert err <= 1e-5, err
    # a finite-difference check of one weight on the float64 restatement ties both to the calculus
    i = 5
    eps = 1e-6
    p2 = [p.copy() for p in params]
    p2[0].flat[i] += eps
    yp, _ = ref.forward(p2, x.astype(np.float64))
    p2[0].flat[i] -= 2 * eps
    ym, _ = ref.forward(p2, x.astype(np.float64))
    fd = float(np.sum(dy * (yp - ym)) / (2 * eps))
    assert abs(fd - g_ref[i]) <= 1e-6 * max(1.0, abs(fd))
    net.close()


def test_probe_loss_and_gradient_match_cpu(cuda_available):
    import torch

    from cf_b200 import _lib
    from oracle import mlp as ref

    rng = np.random.default_rng(1)
    n, npr, nq, K, scale = 6, 4, 9, 5, 0.1
    delta = rng.standard_normal((n, nq, K, K)).astype(np.float32)
    peq = rng.standard_normal((nq, K, K))
    av = rng.standard_normal((n, npr, nq * K)).astype(np.float32)
    v = rng.standard_normal((n, npr, nq * K)).astype(np.float32)
    vn2 = (v.astype(np.float64) ** 2).sum(-1).astype(np.float32)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    d_t, p_t, a_t, v_t, n_t = T(delta), T(peq), T(av), T(v), T(vn2)
    grad = torch.empty_like(d_t)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = _lib.load().cf_precond_probe_loss(int(d_t.data_ptr()), int(p_t.data_ptr()), int(a_t.data_ptr()),
                                           int(v_t.data_ptr()), int(n_t.data_ptr()), scale, n, npr, nq, K,
                                           int(grad.data_ptr()), int(loss.data_ptr()), 0)
    assert st == 0
    torch.cuda.synchronize()
    l_ref, g_ref = ref.probe_loss(delta.astype(np.float64), peq, av.astype(np.float64), v.astype(np.float64),
                                  vn2.astype(np.float64), scale)
    assert abs(loss.item() - l_ref) <= 1e-5 * l_ref
    assert np.abs(grad.cpu().numpy() - g_ref).max() <= 1e-4 * np.abs(g_ref).max()


def test_trained_network_against_maxwellian_blocks(cuda_available):
    """Trained on operator-generated probe pairs, the network lowers its training loss; the
    correction it predicts, scaled by the least-squares gain fitted on validation probes, keeps the
    held-out probe loss at or below the Maxwellian blocks', and GMRES with the learned blocks
    converges to 1e-10 in no more iterations (the block-diagonal family leaves little room: the
    exact per-state block-Jacobi inverse saves only a few per cent of the iterations here)."""
    import torch

    import cf_b200
    from cf_b200 import implicit
    from cf_b200.learned import LearnedPreconditioner

    d = load_op("hs_k4_l4_g1")
    op = cf_b200.CollisionOperator(d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], d["NQ"], d["K"])
    lp = LearnedPreconditioner(op, hidden=128, max_batch=512, scale=0.1, seed=1)
    train = lp.make_samples(3000, dt_nu_values=(10.0,), n_probes=6, seed=2, amp_range=(0.0, 0.6))
    val = lp.make_samples(400, dt_nu_values=(10.0,), n_probes=6, seed=4, amp_range=(0.0, 0.6))
    test = lp.make_samples(400, dt_nu_values=(10.0,), n_probes=6, seed=3, amp_range=(0.0, 0.6))
    lp.fit_normalisation(train)
    dt = float(train["dt"][0])
    before = lp.probe_loss(test, dt, use_net=False)
    hist = lp.train(train, epochs=25, batch=256, lr=2e-3)
    assert hist[-1] < hist[0]
    gains = lp.calibrate(val)
    assert len(gains) == 1 and all(0.0 <= g <= 2.0 for g in gains.values())
    after = lp.probe_loss(test, dt, use_net=True)
    assert after <= before * 1.01, (before, after)
    f = test["f"][:128]
    rhs = op.q(f)
    peq = implicit.block_preconditioner(op, dt)
    _, it_eq, rel_eq = implicit.gmres_solve(op, f, rhs, dt, tol=1e-10, precond=peq)
    _, it_ln, rel_ln = implicit.gmres_solve(op, f, rhs, dt, tol=1e-10, precond=lp.predict(f, dt))
    assert np.all(rel_eq <= 1e-10) and np.all(rel_ln <= 1e-10)
    assert it_ln.mean() <= it_eq.mean() + 0.5, (it_eq.mean(), it_ln.mean())
    op.close()


def test_mlp_gradients_at_the_implicit_configuration_shape(cuda_available):
    """The network of the implicit configuration (hard spheres L = 8, K = 8: 648 coefficients + log10(dt nu)
    in, two hidden layers of 512 GELU, 81 blocks of 8 x 8 out): forward and parameter gradients of the
    library's FP32 kernels against the float64 restatement."""
    import torch

    from cf_b200.learned import MLP
    from oracle import mlp as ref

    n_in, hid, n_out, n = 649, 512, 81 * 64, 16
    net = MLP(n_in, hid, n_out, max_batch=n, seed=5)
    flat = net.params()
    params = ref.unpack(flat.astype(np.float64), n_in, hid, n_out)
    rng = np.random.default_rng(9)
    x = rng.standard_normal((n, n_in)).astype(np.float32)
    dy = rng.standard_normal((n, n_out)).astype(np.float32)
    xt = torch.from_numpy(x).cuda()
    yt = torch.empty((n, n_out), dtype=torch.float32, device="cuda")
    net.forward(xt, yt, train=True)
    y_ref, cache = ref.forward(params, x.astype(np.float64))
    assert np.abs(yt.cpu().numpy() - y_ref).max() <= 1e-4 * np.abs(y_ref).max()
    net.backward(xt, torch.from_numpy(dy).cuda())
    torch.cuda.synchronize()
    g = net.grads().astype(np.float64)
    g_ref = ref.pack_like(ref.backward(params, x.astype(np.float64), cache, dy.astype(np.float64)), n_in, hid, n_out)
    assert np.abs(g - g_ref).max() <= 1e-4 * np.abs(g_ref).max()
    net.close()


def test_learned_solve_not_slower_than_block_at_the_implicit_configuration(cuda_available):
    """Hard spheres L = 8, K = 8 (R from the reference's quadrature), the implicit configuration's network
    (2 x 512 GELU): after training and calibration, GMRES(30) to 1e-10 with the learned preconditioner takes
    no more iterations than with the Maxwellian blocks, and no more time (the network is skipped where its
    calibrated gain is below the threshold); the exact per-state block-Jacobi inverse, the ceiling of the
    block-diagonal family, takes no more iterations than either."""
    import time
    from pathlib import Path

    import torch

    import cf_b200
    from cf_b200 import geometry, implicit, workloads
    from cf_b200.learned import LearnedPreconditioner

    L, K = 8, 8
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = np.asfortranarray(np.load(Path(__file__).resolve().parent / "golden" / "R_hs_k7_l8_pad20.npy"))
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    lp = LearnedPreconditioner(op, hidden=512, max_batch=1024, scale=0.1, seed=2)
    train = lp.make_samples(2048, dt_nu_values=(10.0,), n_probes=8, seed=3, amp_range=(0.0, 0.3))
    lp.fit_normalisation(train)
    hist = lp.train(train, epochs=3, batch=512, lr=1e-3)
    assert hist[-1] <= hist[0]
    del train
    val = lp.make_samples(512, dt_nu_values=(10.0,), n_probes=8, seed=4, amp_range=(0.0, 0.3))
    lp.calibrate(val)
    dt = float(val["dt"][0])
    del val
    cells = workloads.stress_cells(K, L, 256, seed=5, amplitude=0.1)
    cells[:, 0, 4:9] *= np.random.default_rng(6).uniform(0.0, 3.0, size=(256, 1))
    f = torch.from_numpy(cells).cuda()
    rhs = op.q(f)

    def timed(make_p):
        best, out = None, None
        for _ in range(3):
            torch.cuda.synchronize()
            t = time.perf_counter()
            P = make_p()
            out = implicit.gmres_solve(op, f, rhs, dt, restart=30, tol=1e-10, precond=P)
            torch.cuda.synchronize()
            dt_s = time.perf_counter() - t
            best = dt_s if best is None else min(best, dt_s)
        return best, out

    t_block, (_, it_block, rel_block) = timed(lambda: implicit.block_preconditioner(op, dt))
    t_learn, (_, it_learn, rel_learn) = timed(lambda: lp.predict(f, dt))
    assert np.all(rel_block <= 1e-10) and np.all(rel_learn <= 1e-10)
    assert it_learn.mean() <= it_block.mean() + 0.5, (it_block.mean(), it_learn.mean())
    assert t_learn <= 1.15 * t_block + 2e-3, (t_block, t_learn)
    P_exact = implicit.exact_block_jacobi(op, f, dt)
    _, it_exact, rel_exact = implicit.gmres_solve(op, f, rhs, dt, restart=30, tol=1e-10, precond=P_exact)
    assert np.all(rel_exact <= 1e-10)
    assert it_exact.mean() <= min(it_block.mean(), it_learn.mean()) + 0.5
    op.close()
