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
