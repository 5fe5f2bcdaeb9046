"""COO routing lists: the reference's selection-rule tests and pins of the restated geometry."""
from __future__ import annotations

import json
import math

import numpy as np
import pytest

from conftest import GOLDEN


def q2lm(q):
    q = np.asarray(q, dtype=np.int64)
    l = np.floor(np.sqrt(q - 1)).astype(np.int64)
    return l, (q - 1) - l * l - l


@pytest.fixture(scope="module")
def skeleton():
    from cf_b200 import geometry

    return geometry.gaunt_labels_complex(5)  # tests/TestSphericalHarmonics.m:3 (L_max = 5)


def test_triangle_inequality(skeleton):
    """tests/TestSphericalHarmonics.m:15-29"""
    l1, _ = q2lm(skeleton[:, 0])
    l2, _ = q2lm(skeleton[:, 1])
    l3, _ = q2lm(skeleton[:, 2])
    assert np.all((l3 >= np.abs(l1 - l2)) & (l3 <= l1 + l2))


def test_parity(skeleton):
    """tests/TestSphericalHarmonics.m:31-43"""
    l = [q2lm(skeleton[:, i])[0] for i in range(3)]
    assert np.all((l[0] + l[1] + l[2]) % 2 == 0)


def test_magnetic_projection(skeleton):
    """tests/TestSphericalHarmonics.m:45-57"""
    m = [q2lm(skeleton[:, i])[1] for i in range(3)]
    assert np.all(m[0] + m[1] == m[2])


def test_index_bounds(skeleton):
    """tests/TestSphericalHarmonics.m:59-64"""
    assert skeleton.min() >= 1 and skeleton.max() <= 36


def test_counts_and_digests_pinned():
    """N_G, N_L, S and the (labels, ic_map) digest for L = 0..12 equal the committed pins."""
    import hashlib

    from cf_b200 import geometry

    pins = json.loads((GOLDEN / "geometry_counts.json").read_text())
    for L in range(0, 13):
        g = geometry.sort_for_contraction(geometry.generate_geometry(L))
        h = hashlib.sha256()
        for a in (g.labels, g.ic_map):
            h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        got = dict(n_g=g.n_g, n_l=g.n_l, n_slices=geometry.slice_count(g), digest=h.hexdigest()[:16])
        assert got == pins[str(L)], f"L={L}: {got} != {pins[str(L)]}"
    # the sizes the contraction is benchmarked on
    assert pins["10"]["n_g"] == 65913 and pins["10"]["n_l"] == 381 and pins["10"]["n_slices"] == 4741
    assert pins["16"]["n_g"] == 601569 and pins["16"]["n_l"] == 1341 and pins["16"]["n_slices"] == 26061


@pytest.mark.parametrize("L", [3, 5])
def test_real_gaunt_values_against_quadrature(L):
    """G_real(q1,q2,q3) = int Y_q1 Y_q2 Y_q3 dOmega of real harmonics; the nonzero set is exactly |G| > 1e-12."""
    from cf_b200 import basis, geometry, quadrature

    g = geometry.generate_geometry(L)
    n = 3 * L + 2
    pol = quadrature.legendre(n, -1.0, 1.0)
    phi = 2 * math.pi * np.arange(2 * n) / (2 * n)
    CT, PH = np.meshgrid(pol.x, phi, indexing="ij")
    W = (pol.w[:, None] * np.full_like(PH, 2 * math.pi / (2 * n))).ravel()
    Y = basis.real_sh(L, np.arccos(CT.ravel()), PH.ravel())
    NQ = basis.n_q(L)
    G = np.einsum("p,pi,pj,pk->ijk", W, Y, Y, Y)
    q = g.labels.astype(np.int64) - 1
    vals_quad = G[q[:, 0], q[:, 1], q[:, 2]]
    assert np.max(np.abs(vals_quad - g.vals)) < 1e-13
    mask = np.abs(G) > 1e-10
    assert mask.sum() == g.n_g
    assert np.all(mask[q[:, 0], q[:, 1], q[:, 2]])


def test_find_order_unique_rows_and_stable_sort():
    from cf_b200 import geometry

    g = geometry.generate_geometry(6)
    NQ = g.n_q
    lin = (g.labels[:, 0] - 1) + NQ * ((g.labels[:, 1] - 1) + NQ * (g.labels[:, 2] - 1))
    assert np.all(np.diff(lin) > 0), "MATLAB find() order: column-major, q1 fastest"
    l = np.floor(np.sqrt(g.labels - 1)).astype(np.int64)
    trip = g.l_triplets[g.ic_map.astype(np.int64) - 1]
    assert np.array_equal(trip, l)
    keys = g.l_triplets[:, 0] * 10000 + g.l_triplets[:, 1] * 100 + g.l_triplets[:, 2]
    assert np.all(np.diff(keys) > 0), "unique(...,'rows') is sorted lexicographically"
    s = geometry.sort_for_contraction(g)
    key = s.ic_map * 1e6 + s.labels[:, 0]
    assert np.all(np.diff(key) >= 0)
    # stability: inside equal (ic, q1) the original order is kept
    o = np.lexsort((g.labels[:, 0], g.ic_map))
    assert np.array_equal(s.labels, g.labels[o])


def test_gaunt_symmetric_in_q2_q3():
    """Real Gaunt coefficients are symmetric in their last two indices.

    The reference's log-factorial Racah sums (src/SHL/gaunt_compute_values.m:49-90) carry a few
    1e-13 of relative rounding at L = 8, so the computed lists are symmetric to 1e-12, not bitwise."""
    from cf_b200 import geometry

    g = geometry.generate_geometry(8)
    NQ = g.n_q
    d = {}
    for (a, b, c), v in zip(g.labels.astype(np.int64), g.vals):
        d[(a, b, c)] = v
    worst = 0.0
    for (a, b, c), v in d.items():
        w = d.get((a, c, b))
        assert w is not None
        worst = max(worst, abs(v - w) / abs(v))
    assert worst < 1e-12
