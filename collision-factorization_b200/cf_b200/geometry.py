"""COO Gaunt routing lists of the factorised collision operator.

Restates how the reference builds the lists that the contraction kernels walk:

* the complex Gaunt skeleton (l-triangle, parity, m3 = m1 + m2;
  src/SHL/gaunt_generate_labels.m:1-41) and its values from log-factorial Racah
  sums (src/SHL/gaunt_compute_values.m:1-90);
* the complex-to-real transform U (src/SHL/complex2real.m:1-40) applied as
  G_real(i,j,k) = sum U(i,a) U(j,b) conj(U(k,c)) G_c(a,b,c)
  (src/GeneralCollisionTensor.m:261-272);
* nonzeros |G_real| > 1e-12 in MATLAB ``find`` order, i.e. column-major over
  (q1, q2, q3) with q1 fastest (src/GeneralCollisionTensor.m:273-275);
* ``ic_map``: the 1-based index of each entry's l-triplet among the unique
  triplets sorted lexicographically (MATLAB ``unique(...,'rows')``;
  src/GeneralCollisionTensor.m:277-279);
* the stable ``sortrows([ic_map, q1])`` that the angular-first and radial-first
  kernels require (benchmark_collision_contraction_scaling.m:82-85).

Arrays are returned in the reference's representation: labels [N_G x 3] as
float64 holding 1-based integers, vals [N_G], ic_map [N_G] float64 1-based.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .basis import n_q, q_index


def gaunt_labels_complex(L: int) -> np.ndarray:
    """Complex Gaunt skeleton [n x 3] of 1-based (q1, q2, q3), in the reference's loop order.

    Loops l1, l2, l3 (from |l1-l2| stepping by 2 so that l1+l2+l3 is even, up to
    min(L, l1+l2)), m1, m2; keeps m3 = m1 + m2 when |m3| <= l3
    (src/SHL/gaunt_generate_labels.m:8-31).
    """
    rows = []
    for l1 in range(L + 1):
        for l2 in range(L + 1):
            lo, hi = abs(l1 - l2), min(L, l1 + l2)
            start = lo if (l1 + l2 + lo) % 2 == 0 else lo + 1
            for l3 in range(start, hi + 1, 2):
                m1 = np.arange(-l1, l1 + 1)
                m2 = np.arange(-l2, l2 + 1)
                M1, M2 = np.meshgrid(m1, m2, indexing="ij")  # m1 outer, m2 inner
                M3 = M1 + M2
                ok = np.abs(M3) <= l3
                q1 = l1 * l1 + l1 + M1[ok] + 1
                q2 = l2 * l2 + l2 + M2[ok] + 1
                q3 = l3 * l3 + l3 + M3[ok] + 1
                rows.append(np.stack([q1, q2, q3], axis=1))
    if not rows:
        return np.zeros((0, 3), dtype=np.int64)
    return np.concatenate(rows, axis=0).astype(np.int64)


def _log_factorials(n: int) -> np.ndarray:
    """lf[n] = log(n!) as a running sum of logs (src/SHL/gaunt_compute_values.m:3-4)."""
    return np.concatenate(([0.0], np.cumsum(np.log(np.arange(1, n + 1, dtype=np.float64)))))


def gaunt_values_complex(L: int, labels: np.ndarray) -> np.ndarray:
    """Complex Gaunt values int Y_{l1m1} Y_{l2m2} conj(Y_{l3m3}) for the skeleton.

    (-1)^m3 sqrt((2l1+1)(2l2+1)(2l3+1)/4pi) (l1 l2 l3; 0 0 0) (l1 l2 l3; m1 m2 -m3),
    with both 3j symbols from log-factorial Racah sums
    (src/SHL/gaunt_compute_values.m:21-90).
    """
    lf = _log_factorials(3 * L + 2)
    q = labels.astype(np.float64)
    l = np.floor(np.sqrt(q - 1.0)).astype(np.int64)
    m = (labels - 1) - l * l - l
    l1, l2, l3 = l[:, 0], l[:, 1], l[:, 2]
    m1, m2, m3 = m[:, 0], m[:, 1], -m[:, 2]  # the 3j is evaluated at (m1, m2, -m3)

    # 3j(l1 l2 l3; 0 0 0), zero unless l1+l2+l3 is even (parity is already enforced)
    J = l1 + l2 + l3
    g = J // 2
    log_w0 = 0.5 * (lf[2 * g - 2 * l1] + lf[2 * g - 2 * l2] + lf[2 * g - 2 * l3] - lf[2 * g + 1]) + lf[g] - (
        lf[g - l1] + lf[g - l2] + lf[g - l3]
    )
    w0 = np.where(J % 2 == 0, np.where(g % 2 == 0, 1.0, -1.0) * np.exp(log_w0), 0.0)

    # 3j(l1 l2 l3; m1 m2 m3) by the Racah sum over t, summed sequentially in t
    log_delta = 0.5 * (lf[l1 + l2 - l3] + lf[l1 - l2 + l3] + lf[-l1 + l2 + l3] - lf[l1 + l2 + l3 + 1])
    t_min = np.maximum.reduce([np.zeros_like(l1), l2 - l3 - m1, l1 - l3 + m2])
    t_max = np.minimum.reduce([l1 - m1, l2 + m2, l1 + l2 - l3])
    log_mag = 0.5 * (lf[l1 + m1] + lf[l1 - m1] + lf[l2 + m2] + lf[l2 - m2] + lf[l3 + m3] + lf[l3 - m3])
    total = np.zeros(labels.shape[0])
    span = int(np.max(t_max - t_min)) + 1 if labels.shape[0] else 0
    for dt in range(max(span, 0)):
        t = t_min + dt
        live = t <= t_max
        tc = np.where(live, t, t_min)
        idx = [tc, l1 + l2 - l3 - tc, l1 - m1 - tc, l2 + m2 - tc, l3 - l2 + m1 + tc, l3 - l1 - m2 + tc]
        term_log = sum(lf[np.clip(i, 0, None)] for i in idx)
        term = np.where(tc % 2 == 0, 1.0, -1.0) * np.exp(-term_log)
        total = total + np.where(live, term, 0.0)
    phase = np.where((l1 - l2 - m3) % 2 == 0, 1.0, -1.0)
    w_m = phase * np.exp(log_delta + log_mag) * total

    pref = np.where(m[:, 2] % 2 == 0, 1.0, -1.0) * np.sqrt((2 * l1 + 1) * (2 * l2 + 1) * (2 * l3 + 1) / (4.0 * math.pi)) * w0
    return pref * w_m


def complex_to_real_block(l: int) -> np.ndarray:
    """(2l+1) x (2l+1) block of U for degree l (src/SHL/complex2real.m:17-39).

    Rows are real harmonics m = -l..l, columns complex harmonics m = -l..l:
      Y_real(-m) = i/sqrt2 (Y_{-m} - (-1)^m Y_m),  Y_real(0) = Y_0,
      Y_real(+m) = 1/sqrt2 (Y_{-m} + (-1)^m Y_m)         for m = 1..l.
    """
    d = 2 * l + 1
    U = np.zeros((d, d), dtype=np.complex128)
    if l == 0:
        U[0, 0] = 1.0
        return U
    s = 1.0 / math.sqrt(2.0)
    for mm in range(1, l + 1):
        neg, pos = l - mm, l + mm  # row/col positions of -mm and +mm
        sign = -1.0 if mm % 2 else 1.0
        U[neg, neg] = 1j * s
        U[neg, pos] = -1j * sign * s
        U[pos, pos] = sign * s
        U[pos, neg] = s
    U[l, l] = 1.0
    return U


@dataclass
class Geometry:
    L: int
    labels: np.ndarray  # [N_G x 3] float64, 1-based (q1, q2, q3)
    vals: np.ndarray  # [N_G] float64
    ic_map: np.ndarray  # [N_G] float64, 1-based l-triplet index
    l_triplets: np.ndarray  # [N_L x 3] int64 unique sorted (l1, l2, l3)

    @property
    def n_g(self) -> int:
        return int(self.vals.shape[0])

    @property
    def n_l(self) -> int:
        return int(self.l_triplets.shape[0])

    @property
    def n_q(self) -> int:
        return n_q(self.L)


def generate_geometry(L: int, threshold: float = 1e-12) -> Geometry:
    """Real Gaunt COO lists in the reference's order (src/GeneralCollisionTensor.m:251-281).

    The complex Gaunt tensor is block-sparse in l-triplets and U is block-diagonal
    in l, so the three mode products are applied per complex l-triplet block.
    The surviving entries are then ordered column-major over (q1, q2, q3), which
    is the order MATLAB's ``find`` returns.
    """
    cl = gaunt_labels_complex(L)
    cv = gaunt_values_complex(L, cl)
    NQ = n_q(L)
    lq = np.floor(np.sqrt(cl.astype(np.float64) - 1.0)).astype(np.int64)
    Ub = [complex_to_real_block(l) for l in range(L + 1)]
    Q1, Q2, Q3, V = [], [], [], []
    # group complex entries by their l-triplet
    key = (lq[:, 0] * (L + 1) + lq[:, 1]) * (L + 1) + lq[:, 2]
    order = np.argsort(key, kind="stable")
    key_s = key[order]
    bounds = np.flatnonzero(np.diff(key_s)) + 1
    starts = np.concatenate(([0], bounds))
    ends = np.concatenate((bounds, [key_s.size]))
    for s, e in zip(starts, ends):
        idx = order[s:e]
        l1, l2, l3 = lq[idx[0]]
        d1, d2, d3 = 2 * l1 + 1, 2 * l2 + 1, 2 * l3 + 1
        blk = np.zeros((d1, d2, d3), dtype=np.complex128)
        a = cl[idx, 0] - 1 - l1 * l1
        b = cl[idx, 1] - 1 - l2 * l2
        c = cl[idx, 2] - 1 - l3 * l3
        blk[a, b, c] = cv[idx]
        blk = np.tensordot(Ub[l1], blk, axes=(1, 0))  # mode 1: U
        blk = np.tensordot(Ub[l2], blk, axes=(1, 1)).transpose(1, 0, 2)  # mode 2: U
        blk = np.tensordot(np.conj(Ub[l3]), blk, axes=(1, 2)).transpose(1, 2, 0)  # mode 3: conj(U)
        re = blk.real
        i, j, k = np.nonzero(np.abs(re) > threshold)
        Q1.append(i + l1 * l1 + 1)
        Q2.append(j + l2 * l2 + 1)
        Q3.append(k + l3 * l3 + 1)
        V.append(re[i, j, k])
    q1 = np.concatenate(Q1) if Q1 else np.zeros(0, np.int64)
    q2 = np.concatenate(Q2) if Q2 else np.zeros(0, np.int64)
    q3 = np.concatenate(Q3) if Q3 else np.zeros(0, np.int64)
    vals = np.concatenate(V) if V else np.zeros(0)
    # MATLAB find() order: linear index q1 + NQ*q2 + NQ^2*q3 ascending
    lin = (q1 - 1) + NQ * ((q2 - 1) + NQ * (q3 - 1))
    o = np.argsort(lin, kind="stable")
    q1, q2, q3, vals = q1[o], q2[o], q3[o], vals[o]
    labels = np.stack([q1, q2, q3], axis=1)
    ltrip = np.floor(np.sqrt(labels.astype(np.float64) - 1.0)).astype(np.int64)
    uniq, inv = np.unique(ltrip, axis=0, return_inverse=True)
    return Geometry(
        L=L,
        labels=labels.astype(np.float64),
        vals=vals.astype(np.float64),
        ic_map=(inv.reshape(-1) + 1).astype(np.float64),
        l_triplets=uniq.astype(np.int64),
    )


def sort_for_contraction(geo: Geometry) -> Geometry:
    """Stable sortrows([ic_map, q1]) (benchmark_collision_contraction_scaling.m:82-85)."""
    o = np.lexsort((geo.labels[:, 0], geo.ic_map))
    return Geometry(L=geo.L, labels=np.ascontiguousarray(geo.labels[o]), vals=geo.vals[o].copy(),
                    ic_map=geo.ic_map[o].copy(), l_triplets=geo.l_triplets)


def labels_colmajor(labels: np.ndarray) -> np.ndarray:
    """The [N_G x 3] labels as a column-major buffer (the layout MATLAB passes to MEX)."""
    return np.asfortranarray(labels, dtype=np.float64)


def slice_count(geo: Geometry) -> int:
    """Number of (t, q1) runs in a sorted list: the S of the K^3 step."""
    if geo.n_g == 0:
        return 0
    t = geo.ic_map
    q1 = geo.labels[:, 0]
    change = (np.diff(t) != 0) | (np.diff(q1) != 0)
    return int(1 + np.count_nonzero(change))


def fold_q2q3(geo: Geometry, R: np.ndarray, K: int):
    """The q2 <-> q3 folded operator (labels, vals, ic_map, R_sym), the same quadratic form as (geo, R).

    Entries (q1,q2,q3) with l-triplet t = (l1,l2,l3) and their mirrors (q1,q3,q2) with
    t' = (l1,l3,l2) contribute G R_t.(f2 (x) f3) + G' R_t'.(f3 (x) f2); with G = G' (real Gaunt
    symmetry) this is G (R_t + R_t'^T23).(f2 (x) f3).  The folded list keeps entries with l2 < l3, or
    l2 = l3 and q2 <= q3 (q2 = q3 at G/2), against R^S_t = R_t + R_t'^T23, renumbering the kept
    triplets in order.  Inside each run of equal (triplet, q1) the entries are then ordered by
    (q2, q3).  This is the host-side statement of what the library builds for CF_FORM_AF_SYM
    (csrc/plan.cu, build_folded).
    """
    lab = geo.labels.astype(np.int64)
    ic = geo.ic_map.astype(np.int64) - 1
    l = np.floor(np.sqrt(lab - 1.0)).astype(np.int64)
    n_l = int(ic.max()) + 1
    trip = np.zeros((n_l, 3), dtype=np.int64)
    trip[ic] = l
    tindex = {tuple(t): i for i, t in enumerate(trip)}
    keep_t = trip[:, 1] <= trip[:, 2]
    tnew = np.cumsum(keep_t) - 1
    R = np.asarray(R).reshape(K, K, K, -1, order="F")
    Rs = []
    for t in np.flatnonzero(keep_t):
        tp = tindex[(trip[t, 0], trip[t, 2], trip[t, 1])]
        Rs.append(R[:, :, :, t] + R[:, :, :, tp].transpose(0, 2, 1))
    Rs = np.asfortranarray(np.stack(Rs, axis=3))
    where = {tuple(r): i for i, r in enumerate(lab)}
    rows, vals, ics = [], [], []
    for z in range(lab.shape[0]):
        q1, q2, q3 = lab[z]
        l2, l3 = l[z, 1], l[z, 2]
        if (q1, q3, q2) not in where:  # every entry needs its mirror, kept or dropped
            raise ValueError(f"entry {z + 1} has no (q1, q3, q2) mirror: the list does not fold")
        if not (l2 < l3 or (l2 == l3 and q2 <= q3)):
            continue
        zp = where[(q1, q3, q2)]
        g = 0.5 * geo.vals[z] if q2 == q3 else 0.5 * (geo.vals[z] + geo.vals[zp])
        rows.append((q1, q2, q3))
        vals.append(g)
        ics.append(tnew[ic[z]] + 1)
    rows = np.array(rows, dtype=np.float64).reshape(-1, 3)
    vals = np.array(vals)
    ics = np.array(ics, dtype=np.float64)
    # order by (q2, q3) inside each run of equal (triplet, q1)
    run = np.cumsum(np.r_[True, (np.diff(ics) != 0) | (np.diff(rows[:, 0]) != 0)]) if len(ics) else np.zeros(0)
    o = np.lexsort((rows[:, 2], rows[:, 1], run))
    return np.asfortranarray(rows[o]), vals[o], ics[o], Rs
