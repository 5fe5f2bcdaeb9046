"""The oracle restatement against the reference's own compiled kernels and the golden fixtures."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import load_op, normwise_err

OPS = ["wcu_k2_l2_g0", "cfg1_k3_l4_g0", "hs_k4_l4_g1", "bkw_k5_l1_g0"]


@pytest.mark.parametrize("name", OPS)
def test_restatement_matches_compiled_reference_bitwise(name, oracle_lib, reference_lib):
    """oracle/contraction.c reproduces angular_first / radial_first / naive bit for bit."""
    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    for kern in ("af", "rf", "naive"):
        lab = ("labels_sorted", "vals_sorted", "ic_map_sorted") if kern != "naive" else ("labels", "vals", "ic_map")
        Qo = np.zeros((NQ, K), order="F")
        getattr(oracle_lib, kern)(Qo, d["f"], d[lab[0]], d[lab[1]], d[lab[2]], d["R"], NQ, K)
        Qr = np.zeros((NQ, K), order="F")
        reference_lib.contract(kern, Qr, d["f"], d[lab[0]], d[lab[1]], d[lab[2]], d["R"], NQ, K)
        assert np.array_equal(Qo, Qr), f"{kern}: max diff {np.abs(Qo - Qr).max()}"


@pytest.mark.parametrize("name", OPS)
def test_oracle_reproduces_golden_outputs(name, oracle_lib):
    """The committed reference outputs (compiled reference, exact build) are reproduced bit for bit."""
    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    Q = np.zeros((NQ, K), order="F")
    oracle_lib.af(Q, d["f"], d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    assert np.array_equal(Q, d["Q_af"])
    Q = np.zeros((NQ, K), order="F")
    oracle_lib.rf(Q, d["f"], d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    assert np.array_equal(Q, d["Q_rf"])
    Q = np.zeros((NQ, K), order="F")
    oracle_lib.naive(Q, d["f"], d["labels"], d["vals"], d["ic_map"], d["R"], NQ, K)
    assert np.array_equal(Q, d["Q_naive"])


@pytest.mark.parametrize("name", OPS)
def test_orderings_agree(name):
    """Angular-first, radial-first, naive and dense orderings give the same Q to rounding.

    The reference never compares its kernels with one another; this is that comparison.
    """
    from oracle import rtensor

    d = load_op(name)
    assert normwise_err(d["Q_rf"], d["Q_af"]) < 1e-13
    assert normwise_err(d["Q_naive"], d["Q_af"]) < 1e-13
    if d["NQ"] * d["K"] <= 130:
        from cf_b200.geometry import Geometry
        from oracle.reference import Oracle

        geo = Geometry(d["L"], d["labels"], d["vals"], d["ic_map"], d["l_triplets"])
        Cd = rtensor.assemble_dense(geo, d["R"], d["K"])
        N = d["NQ"] * d["K"]
        Qd = np.zeros(N)
        Oracle().dense(Qd, d["f"].ravel(order="F"), Cd, N)
        assert normwise_err(Qd.reshape(d["NQ"], d["K"], order="F"), d["Q_af"]) < 1e-13


@pytest.mark.parametrize("name", ["cfg1_k3_l4_g0", "hs_k4_l4_g1"])
def test_jacobian_oracle(name, oracle_lib):
    """J(f).v: J(f).f = 2 Q(f); linear in v; matches the dense C(:,:,f) + C(:,f,:) and a difference quotient."""
    from cf_b200.geometry import Geometry
    from oracle import rtensor

    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    args = (d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    f = d["f"]
    out = np.zeros((NQ, K), order="F")
    oracle_lib.jv(out, f, f, *args)
    assert normwise_err(out, 2.0 * d["Q_af"]) < 1e-13
    rng = np.random.default_rng(3)
    v = np.asfortranarray(rng.standard_normal((NQ, K)))
    w = np.asfortranarray(rng.standard_normal((NQ, K)))
    jv = np.zeros((NQ, K), order="F")
    oracle_lib.jv(jv, f, v, *args)
    jw = np.zeros((NQ, K), order="F")
    oracle_lib.jv(jw, f, w, *args)
    jvw = np.zeros((NQ, K), order="F")
    oracle_lib.jv(jvw, f, np.asfortranarray(2.0 * v - 3.0 * w), *args)
    assert normwise_err(jvw, 2.0 * jv - 3.0 * jw) < 1e-13
    geo = Geometry(d["L"], d["labels"], d["vals"], d["ic_map"], d["l_triplets"])
    Cd = rtensor.assemble_dense(geo, d["R"], K)
    fv = f.ravel(order="F")
    J = np.einsum("ijk,k->ij", Cd, fv) + np.einsum("ijk,j->ik", Cd, fv)
    assert normwise_err(jv.ravel(order="F"), J @ v.ravel(order="F")) < 1e-12
    # Q is quadratic: (Q(f + h v) - Q(f - h v)) / (2h) = J(f) v exactly up to rounding
    h = 1e-3
    Qp = np.zeros((NQ, K), order="F")
    oracle_lib.af(Qp, np.asfortranarray(f + h * v), *args)
    Qm = np.zeros((NQ, K), order="F")
    oracle_lib.af(Qm, np.asfortranarray(f - h * v), *args)
    assert normwise_err((Qp - Qm) / (2 * h), jv) < 1e-9


def test_unsorted_input_still_correct(oracle_lib, reference_lib):
    """The reference kernels are correct for any entry order (runs of equal (t,q1) simply get shorter)."""
    d = load_op("cfg1_k3_l4_g0")
    NQ, K = d["NQ"], d["K"]
    rng = np.random.default_rng(0)
    perm = rng.permutation(d["labels"].shape[0])
    lab = np.asfortranarray(d["labels"][perm])
    Qo = np.zeros((NQ, K), order="F")
    oracle_lib.af(Qo, d["f"], lab, d["vals"][perm], d["ic_map"][perm], d["R"], NQ, K)
    Qr = np.zeros((NQ, K), order="F")
    reference_lib.contract("af", Qr, d["f"], lab, d["vals"][perm], d["ic_map"][perm], d["R"], NQ, K)
    assert np.array_equal(Qo, Qr)
    assert normwise_err(Qo, d["Q_af"]) < 1e-13


def test_batched_oracle_equals_per_cell(oracle_lib, reference_lib):
    d = load_op("hs_k4_l4_g1")
    NQ, K = d["NQ"], d["K"]
    from cf_b200 import workloads

    cells = workloads.maxwellian_cells(K, d["L"], 7, seed=3)  # [B, K, NQ]
    fb = np.asfortranarray(cells.transpose(2, 1, 0))  # [NQ, K, B]
    args = (d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    Qb = np.zeros_like(fb, order="F")
    oracle_lib.af_batch(Qb, fb, *args, nthreads=2)
    Qr = np.zeros_like(fb, order="F")
    reference_lib.batch("af", Qr, fb, *args, nthreads=2)
    assert np.array_equal(Qb, Qr)
    for b in range(fb.shape[2]):
        Q1 = np.zeros((NQ, K), order="F")
        oracle_lib.af(Q1, np.asfortranarray(fb[:, :, b]), *args)
        assert np.array_equal(Q1, Qb[:, :, b])


@pytest.mark.parametrize("name", ["cfg1_k3_l4_g0", "hs_k4_l4_g1"])
def test_q2q3_folded_operator_is_the_same_quadratic_form(name, oracle_lib):
    """The folded list (half the entries, R_t + R_t'^T) gives the reference's Q to rounding."""
    from cf_b200 import geometry

    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    geo = geometry.sort_for_contraction(
        geometry.Geometry(d["L"], d["labels"], d["vals"], d["ic_map"], d["l_triplets"]))
    lab, vals, ic, Rs = geometry.fold_q2q3(geo, d["R"], K)
    assert lab.shape[0] < 0.6 * geo.n_g
    Q = np.zeros((NQ, K), order="F")
    oracle_lib.af(Q, d["f"], lab, vals, ic, Rs, NQ, K)
    assert normwise_err(Q, d["Q_af"]) < 1e-14


def test_fold_refuses_a_list_missing_a_kept_entry():
    """The folded list keeps one entry of each mirror pair (l2 < l3, or l2 = l3 and q2 <= q3).  A list
    that lacks a kept entry but still holds its mirror does not fold: the restatement refuses it
    (the library returns CF_EUNSUPPORTED, tests/test_gpu_band_edges.py), instead of dropping the
    orphaned mirror from Q."""
    from cf_b200 import geometry

    geo = geometry.sort_for_contraction(geometry.generate_geometry(3))
    K = 2
    R = np.zeros((K, K, K, int(geo.ic_map.max())))
    geometry.fold_q2q3(geo, R, K)  # the full list folds
    lq = np.floor(np.sqrt(geo.labels - 1.0)).astype(int)
    z = int(np.nonzero((geo.labels[:, 1] != geo.labels[:, 2]) & (lq[:, 1] < lq[:, 2]))[0][0])
    keep = np.ones(len(geo.vals), dtype=bool)
    keep[z] = False
    import dataclasses

    cut = dataclasses.replace(geo, labels=np.ascontiguousarray(geo.labels[keep]), vals=geo.vals[keep].copy(),
                              ic_map=geo.ic_map[keep].copy())
    with pytest.raises(ValueError):
        geometry.fold_q2q3(cut, R, K)


@pytest.mark.parametrize("K", list(range(1, 17)))
def test_restatement_bitwise_at_every_k(K, oracle_lib, reference_lib):
    """The oracle against the reference's compiled angular-first and radial-first kernels at every K
    the library builds, on the operators the GPU sweep uses (L = 3 + K mod 3, synthetic R), from a
    nonzero Q: the GPU's exact forms are checked against this oracle at the same K."""
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    L = 3 + K % 3
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=100 + K)
    f = np.asfortranarray(workloads.maxwellian_cells(K, L, 5, seed=K, amplitude=0.05).transpose(2, 1, 0))
    q0 = np.asfortranarray(np.random.default_rng(K).standard_normal(f.shape))
    args = (geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    for kern in ("af", "rf"):
        Qo = q0.copy(order="F")
        oracle_lib.af_batch(Qo, f, *args, nthreads=2, form=kern)
        Qr = q0.copy(order="F")
        reference_lib.batch(kern, Qr, f, *args, nthreads=2)
        assert np.array_equal(Qo, Qr), f"{kern} K={K}: max diff {np.abs(Qo - Qr).max():.3e}"


@pytest.mark.parametrize("K", list(range(1, 17)))
def test_jacobian_oracle_at_every_k(K, oracle_lib):
    """The oracle's J(f).v at every K on the GPU sweep's operators: J(f).f = 2 Q(f) against the
    angular-first oracle (itself pinned to the compiled reference), and the central difference of the
    quadratic Q, (Q(f + h v) - Q(f - h v)) / 2h = J(f).v up to rounding."""
    from cf_b200 import geometry, workloads
    from oracle import rtensor

    L = 3 + K % 3
    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    R = workloads.synthetic_R(rtensor.l_triplets_of(geo), K, seed=100 + K)
    f = np.asfortranarray(workloads.maxwellian_cells(K, L, 1, seed=K, amplitude=0.05)[0].T)
    v = np.asfortranarray(np.random.default_rng(K).standard_normal(f.shape))
    args = (geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    q = np.zeros_like(f, order="F")
    oracle_lib.af(q, f, *args)
    jf = np.zeros_like(f, order="F")
    oracle_lib.jv(jf, f, f, *args)
    assert normwise_err(jf, 2.0 * q) < 1e-13
    jv = np.zeros_like(f, order="F")
    oracle_lib.jv(jv, f, v, *args)
    h = 1e-3
    qp = np.zeros_like(f, order="F")
    oracle_lib.af(qp, np.asfortranarray(f + h * v), *args)
    qm = np.zeros_like(f, order="F")
    oracle_lib.af(qm, np.asfortranarray(f - h * v), *args)
    assert normwise_err((qp - qm) / (2 * h), jv) < 1e-9
