"""Reduced radial tensor R from the reference's own quadrature (TEST INFRASTRUCTURE).

Calls the reference's compiled ``compute_rtensor_sumfac_mex`` (oracle/_ref) on the 26 inputs that
``cf_b200.rtensor.sumfac_inputs`` prepares (the restated MATLAB driver,
src/GeneralCollisionTensor.m:43-181), applies the conservation rule (:183-191), and assembles the
dense tensor of src/GeneralCollisionTensor.m:283-311 for the small-L comparators.

The reference computes R on its own CPU path; this module only feeds it.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parents[1] / "collision-factorization_b200"
if str(_PKG) not in sys.path:
    sys.path.insert(0, str(_PKG))

from cf_b200 import basis, quadrature  # noqa: E402,F401
from cf_b200.geometry import Geometry  # noqa: E402
# the restated MATLAB driver lives in the package (the GPU quadrature needs the same inputs)
from cf_b200.rtensor import conservation_zero, grid_sizes, l_triplets_of, sumfac_inputs  # noqa: E402,F401

from .reference import Reference  # noqa: E402


def generate_R(geo: Geometry, K_max: int, gamma: float, radial_pad: int = 40, angular_pad: int = 0,
               flavour: str = "fast") -> np.ndarray:
    """R [K x K x K x N_L] (Fortran order) from the reference's sum-factorised quadrature."""
    args = sumfac_inputs(geo, K_max, gamma, radial_pad, angular_pad)
    ref = Reference(flavour)
    (R,) = ref.call("ref_sumfac_mexFunction", args, nlhs=1)
    N_K = K_max + 1
    R = np.asfortranarray(R.reshape(N_K, N_K, N_K, -1, order="F"))
    return conservation_zero(R, args[20])


def assemble_dense(geo: Geometry, R: np.ndarray, K: int) -> np.ndarray:
    """Dense C[N x N x N] (column-major) with C(k1 N_Q + q1, k2 N_Q + q2, k3 N_Q + q3) = R_t[k1,k2,k3] G.

    Follows src/GeneralCollisionTensor.m:283-311 (later entries overwrite earlier
    ones, as the MATLAB assignment does).
    """
    NQ = geo.n_q
    N = K * NQ
    Cd = np.zeros((N, N, N), order="F")
    k = np.arange(K)
    for z in range(geo.n_g):
        q1, q2, q3 = (int(v) - 1 for v in geo.labels[z])
        t = int(geo.ic_map[z]) - 1
        i1 = k * NQ + q1
        i2 = k * NQ + q2
        i3 = k * NQ + q3
        Cd[np.ix_(i1, i2, i3)] = R[:, :, :, t] * geo.vals[z]
    return Cd
