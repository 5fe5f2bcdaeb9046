"""B200-native Wigner-Eckart-factorised collision contraction (host side).

* ``mex``      -- the reference's MEX contraction functions with their exact calling convention
                  (in-place Q_out, eight double arguments), running on the GPU.
* ``operator`` -- ``CollisionOperator``: a device-resident operator for batches of cells.
* ``geometry`` -- the COO Gaunt routing lists (labels, vals, ic_map) in the reference's order.
* ``basis``, ``quadrature`` -- basis conventions, Gauss rules and projections of distributions.
* ``matfile``  -- the reference's precomputed operators (MATLAB v7.3 ``.mat``) read into ``CollisionOperator``.

The contraction itself is hand-written CUDA for sm_100a in ``libcf_b200.so`` (C ABI in
``include/cf_b200.h``); there is no CPU fallback.
"""
from . import _lib, basis, geometry, quadrature  # noqa: F401
from ._lib import CFError, few_route_last, launch_count  # noqa: F401
from .mex import (  # noqa: F401
    angular_first_collision_kernel_mex,
    collision_jacobian_apply_mex,
    contract_batched,
    radial_first_collision_kernel_mex,
)
from .operator import CollisionOperator  # noqa: F401

__all__ = [
    "CFError", "CollisionOperator", "angular_first_collision_kernel_mex", "radial_first_collision_kernel_mex",
    "collision_jacobian_apply_mex", "contract_batched", "geometry", "basis", "quadrature", "launch_count", "few_route_last",
]
