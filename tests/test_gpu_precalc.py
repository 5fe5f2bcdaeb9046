"""The GPU quadrature and the GPU operator against the reference's MATLAB-saved operators.

``tests/golden/precalc_k4_pins.npz`` holds, for the nine files of src/precalc (K_max = 4, pad 20), the
saved R projected on four seeded vectors per channel, and three full R tensors.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import per_cell_err

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
TAGS = ["l2_g0", "l4_g0", "l6_g0", "l2_g1", "l4_g1", "l6_g1", "l8_g1", "l10_g1", "l12_g1"]


@pytest.fixture(scope="module")
def pins():
    with np.load(GOLDEN / "precalc_k4_pins.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("tag", TAGS)
def test_gpu_quadrature_reproduces_matlab_R(tag, pins, cuda_available):
    """R from the GPU quadrature (restated driver, conservation rule applied) equals MATLAB's saved R."""
    from cf_b200 import geometry, rtensor

    K_max, L, alpha, n_g, n_l = pins[f"{tag}__meta"]
    geo = geometry.generate_geometry(int(L))
    R = rtensor.compute_R(rtensor.sumfac_inputs(geo, int(K_max), float(alpha), 20, 20))
    assert R.shape == (5, 5, 5, int(n_l))
    P = (pins["W"] @ R.reshape(125, -1, order="F")).T
    ref = pins[f"{tag}__R_proj"]
    assert np.max(np.abs(P - ref)) <= 1e-12 * np.max(np.abs(ref)), tag
    if f"{tag}__R" in pins:
        full = pins[f"{tag}__R"]
        assert np.max(np.abs(R - full)) <= 1e-12 * np.max(np.abs(full)), tag


def test_operator_from_saved_arrays(pins, cuda_available, oracle_lib):
    """A CollisionTensorFile (MATLAB's R, L = 4, hard spheres) drives the GPU operator; Q matches the oracle."""
    import torch

    from cf_b200 import geometry, workloads
    from cf_b200.matfile import CollisionTensorFile

    geo = geometry.generate_geometry(4)
    c = CollisionTensorFile(K_max=4, L_max=4, R=pins["l4_g1__R"], labels=geo.labels, vals=geo.vals,
                            ic_map=geo.ic_map, alpha=1.0)
    op = c.operator()
    cells = workloads.maxwellian_cells(c.K, 4, 53, seed=3)  # [B, K, N_Q]
    f = torch.from_numpy(cells).cuda()
    lab, vals, ic = c.sorted_for_contraction()
    Qo = np.zeros((c.N_Q, c.K, cells.shape[0]), order="F")
    oracle_lib.af_batch(Qo, np.asfortranarray(cells.transpose(2, 1, 0)), lab, vals, ic, c.R, c.N_Q, c.K)
    for form in ("af", "rf", "af_sym"):
        Q = op.q(f, form=form).cpu().numpy()
        assert per_cell_err(Q, Qo.transpose(2, 1, 0)) <= 1e-12, form
    op.close()
