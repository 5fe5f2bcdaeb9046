"""The GPU quadrature of the reduced radial tensor R against the reference's own sumfac MEX."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import load_op

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("K_max,L,gamma,pad", [(2, 2, 0.0, 16), (3, 4, 0.0, 20), (4, 4, 1.0, 20), (5, 1, 0.0, 16)])
def test_sumfac_matches_compiled_reference(K_max, L, gamma, pad, cuda_available, reference_lib):
    """Raw quadrature (before the conservation rule) equals compute_rtensor_sumfac_mex, compiled
    unmodified, to rounding: normwise over R and per channel."""
    from cf_b200 import geometry, rtensor

    geo = geometry.generate_geometry(L)  # the reference's find order decides each triplet's lists
    args = rtensor.sumfac_inputs(geo, K_max, gamma, pad, pad)
    R_gpu = rtensor.compute_R(args, zero_conservation=False)
    (R_ref,) = reference_lib.call("ref_sumfac_mexFunction", args, nlhs=1)
    N_K = K_max + 1
    R_ref = R_ref.reshape(N_K, N_K, N_K, -1, order="F")
    assert R_gpu.shape == R_ref.shape
    assert _rel(R_gpu, R_ref) < 1e-12
    for t in range(R_ref.shape[3]):
        if np.max(np.abs(R_ref[..., t])) > 1e-8 * np.max(np.abs(R_ref)):
            assert _rel(R_gpu[..., t], R_ref[..., t]) < 1e-10, t
    # deterministic: the same inputs give the same bits
    assert np.array_equal(R_gpu, rtensor.compute_R(args, zero_conservation=False))


@pytest.mark.parametrize("name", ["cfg1_k3_l4_g0", "hs_k4_l4_g1"])
def test_sumfac_reproduces_fixture_operators(name, cuda_available):
    """With the conservation rule applied, the GPU R equals the fixtures' R (reference pipeline)."""
    from cf_b200 import geometry, rtensor

    d = load_op(name)
    geo = geometry.generate_geometry(d["L"])
    args = rtensor.sumfac_inputs(geo, d["K_max"], d["gamma"], d["pad"], d["pad"])
    R = rtensor.compute_R(args)
    assert _rel(R, d["R"]) < 1e-12


@pytest.mark.parametrize("L", [8, 10])
def test_sumfac_full_size_hard_spheres(L, cuda_available):
    """Hard spheres, K_max = 7, pad 20 at L = 8 and 10: the committed R (18 and 39 minutes of the
    reference's quadrature on 8 CPU cores) from the GPU in about a second."""
    from cf_b200 import geometry, rtensor

    R_fix = np.load(GOLDEN / f"R_hs_k7_l{L}_pad20.npy")
    geo = geometry.generate_geometry(L)
    args = rtensor.sumfac_inputs(geo, 7, 1.0, 20, 20)
    R = rtensor.compute_R(args)
    assert _rel(R, R_fix) < 1e-12


@pytest.mark.parametrize("K_max,L,gamma,pad", [(3, 4, 0.0, 20), (4, 4, 1.0, 20), (7, 8, 1.0, 20)])
def test_sumfac_packed_equals_dense(K_max, L, gamma, pad, cuda_available):
    """cf_rtensor_sumfac_packed on the compressed gain tables gives cf_rtensor_sumfac's R bit for bit."""
    from cf_b200 import geometry, rtensor

    geo = geometry.generate_geometry(L)
    args = rtensor.sumfac_inputs(geo, K_max, gamma, pad, pad)
    pargs, pg1, pg2 = rtensor.sumfac_inputs(geo, K_max, gamma, pad, pad, packed=True)
    R_dense = rtensor.compute_R(args, zero_conservation=False)
    R_packed = rtensor.compute_R(pargs, zero_conservation=False, packed=(pg1, pg2))
    assert np.array_equal(R_dense, R_packed)
