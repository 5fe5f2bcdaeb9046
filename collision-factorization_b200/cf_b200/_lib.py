"""ctypes binding of libcf_b200.so (the C ABI declared in include/cf_b200.h).

The library is built in-tree by ``collision-factorization_b200/build.py``.  There is no CPU
fallback: if the library is missing, or a call is made without a CUDA device, the call raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libcf_b200.so"

_D = C.POINTER(C.c_double)
_I64 = C.c_int64
_I32 = C.c_int32

CF_OK, CF_EINVAL, CF_ESHAPE, CF_EBADIDX, CF_ENONFINITE, CF_ECUDA, CF_ENOMEM, CF_ENODEVICE, CF_EUNSUPPORTED, \
    CF_ETIMEOUT = range(10)
STATUS_NAMES = {
    0: "CF_OK", 1: "CF_EINVAL", 2: "CF_ESHAPE", 3: "CF_EBADIDX", 4: "CF_ENONFINITE", 5: "CF_ECUDA",
    6: "CF_ENOMEM", 7: "CF_ENODEVICE", 8: "CF_EUNSUPPORTED", 9: "CF_ETIMEOUT",
}

FORM_AF, FORM_RF, FORM_AF_EXACT, FORM_RF_EXACT, FORM_AF_SYM, FORM_AF_F32, FORM_AF_SYM_F32 = 0, 1, 2, 3, 4, 5, 6
FORM_AF_BF16, FORM_AF_SYM_BF16, FORM_AF_SYM_I8, FORM_RF_DENSE = 7, 8, 9, 10
FORMS = {"af": FORM_AF, "rf": FORM_RF, "af_exact": FORM_AF_EXACT, "rf_exact": FORM_RF_EXACT, "af_sym": FORM_AF_SYM,
         "af_f32": FORM_AF_F32, "af_sym_f32": FORM_AF_SYM_F32, "af_bf16": FORM_AF_BF16,
         "af_sym_bf16": FORM_AF_SYM_BF16, "af_sym_i8": FORM_AF_SYM_I8, "rf_dense": FORM_RF_DENSE}

# Every symbol the header declares; the tests check that the library exports all of them.
EXPORTS = [
    "cf_angular_first", "cf_radial_first", "cf_contract_host", "cf_time_contract_host", "cf_jacobian_apply_host",
    "cf_plan_create", "cf_plan_destroy", "cf_plan_get_info", "cf_plan_workspace_size",
    "cf_q_device", "cf_q_device_ws", "cf_jv_device", "cf_q_device_noalloc", "cf_plan_stream_selftest",
    "cf_plan_lblock_selftest",
    "cf_ragged_create", "cf_ragged_destroy", "cf_ragged_q", "cf_ragged_graph_launch", "cf_ragged_q_resident",
    "cf_ragged_q_host",
    "cf_ragged_info", "cf_rk2_workspace_size", "cf_rk2_steps_tiled", "cf_rtensor_sumfac", "cf_rtensor_sumfac_packed",
    "cf_gmres_workspace_size", "cf_gmres_solve_tiled",
    "cf_mlp_create", "cf_mlp_destroy", "cf_mlp_num_params", "cf_mlp_copy", "cf_mlp_forward", "cf_mlp_backward",
    "cf_mlp_adam_step", "cf_precond_probe_loss", "cf_precond_assemble",
    "cf_pack_cells", "cf_unpack_cells", "cf_q_tiled", "cf_jv_tiled", "cf_plan_set_kernel_path", "cf_fp64_fma_peak",
    "cf_status_string", "cf_last_error", "cf_launch_count", "cf_few_route_last", "cf_version",
]


class CFError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


class PlanInfo(C.Structure):
    _fields_ = [
        ("n_g", C.c_int64), ("n_slices", C.c_int64), ("n_l", C.c_int32), ("n_q", C.c_int32),
        ("k", C.c_int32), ("device", C.c_int32), ("flops_q", C.c_double), ("flops_jv", C.c_double),
        ("device_bytes", C.c_int64), ("last_path", C.c_int32), ("reserved", C.c_int32),
    ]

PATH_NAMES = {0: "none", 1: "gather", 2: "tile", 3: "pair", 4: "pair_l1", 5: "pair_split", 6: "tile_mma", 7: "bf16_mma", 8: "tile_quarter",
              9: "few", 10: "split_i8", 11: "band", 12: "band_bf16", 13: "rf_dense",
              14: "lblock"}

_DP = C.POINTER(C.c_double)


class SumfacInputs(C.Structure):
    """cf_sumfac_inputs: the 26 inputs of compute_rtensor_sumfac_mex."""
    _fields_ = [
        ("k_max", C.c_int32), ("n_l", C.c_int32), ("n_q", C.c_int32), ("alpha", C.c_double),
        ("x_nodes", _DP), ("w_x", _DP), ("n_x", C.c_int32),
        ("u1_nodes", _DP), ("w_u1", _DP), ("n_u1", C.c_int32),
        ("t1_nodes", _DP), ("w_t1", _DP), ("n_t1", C.c_int32),
        ("y2_nodes", _DP), ("w_y2", _DP), ("n_y2", C.c_int32),
        ("t2_nodes", _DP), ("w_t2", _DP), ("n_t2", C.c_int32),
        ("mu_chi", _DP), ("w_chi", _DP), ("n_chi", C.c_int32),
        ("eps", _DP), ("w_eps", _DP), ("n_eps", C.c_int32),
        ("radial_norm", _DP), ("sh_norm", _DP), ("l_triplets", _DP), ("qi_valid", _DP),
        ("p_loss_p1", _DP), ("p_gain_p1", _DP), ("p_loss_p2", _DP), ("p_gain_p2", _DP),
    ]


_lib = None


def load(path: str | Path | None = None) -> C.CDLL:
    """Load libcf_b200.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise CFError(7, f"{p} is missing: build it with `python collision-factorization_b200/build.py`")
    lib = C.CDLL(str(p))
    op = [_D, _D, _D, _D, _D, _I64, _I32, _I32, _I32]
    lib.cf_angular_first.argtypes = [_D] + op
    lib.cf_radial_first.argtypes = [_D] + op
    lib.cf_contract_host.argtypes = [_D, _D, _I64, _D, _D, _D, _D, _I64, _I32, _I32, _I32, _I32]
    lib.cf_time_contract_host.argtypes = [_I64, _D, _D, _D, _I64, _D, _D, _D, _D, _I64, _I32, _I32, _I32, _I32]
    lib.cf_jacobian_apply_host.argtypes = [_D, _D, _D, _I64, _D, _D, _D, _D, _I64, _I32, _I32, _I32, _I32]
    lib.cf_plan_create.argtypes = [C.POINTER(C.c_void_p), _D, _D, _D, _D, _I64, _I32, _I32, _I32, _I32]
    lib.cf_plan_destroy.argtypes = [C.c_void_p]
    lib.cf_plan_get_info.argtypes = [C.c_void_p, C.POINTER(PlanInfo)]
    lib.cf_plan_workspace_size.argtypes = [C.c_void_p, _I64, _I32, C.POINTER(C.c_size_t)]
    lib.cf_q_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _I64, _I32, C.c_void_p]
    lib.cf_q_device_ws.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _I64, _I32, C.c_void_p, C.c_size_t,
                                   C.c_void_p]
    lib.cf_jv_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _I64, _I32, C.c_void_p]
    lib.cf_q_device_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _I64, _I32, C.c_void_p]
    lib.cf_pack_cells.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _I64, C.c_void_p]
    lib.cf_unpack_cells.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _I64, C.c_void_p]
    lib.cf_q_tiled.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _I64, _I32, C.c_void_p]
    lib.cf_jv_tiled.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, _I64, _I32, C.c_void_p]
    lib.cf_fp64_fma_peak.argtypes = [_I32, C.POINTER(C.c_double)]
    lib.cf_plan_set_kernel_path.argtypes = [C.c_void_p, _I32]
    lib.cf_plan_stream_selftest.argtypes = [C.c_void_p, C.c_double]
    lib.cf_plan_lblock_selftest.argtypes = [C.c_void_p, C.c_double]
    V = C.c_void_p
    lib.cf_ragged_create.argtypes = [C.POINTER(V), V, V, V, _I32, _I32, _I32]
    lib.cf_ragged_destroy.argtypes = [V]
    lib.cf_ragged_q.argtypes = [V, V, V, V]
    lib.cf_ragged_graph_launch.argtypes = [V, V, V, V]
    lib.cf_ragged_q_resident.argtypes = [V, V]
    lib.cf_ragged_q_host.argtypes = [V, V, V]
    lib.cf_rk2_workspace_size.argtypes = [V, _I64, C.POINTER(C.c_size_t)]
    lib.cf_rtensor_sumfac.argtypes = [_D, C.POINTER(SumfacInputs), _I32, C.POINTER(C.c_double)]
    lib.cf_rtensor_sumfac_packed.argtypes = [_D, C.POINTER(SumfacInputs), _D, _D, _I32, C.POINTER(C.c_double)]
    lib.cf_rk2_steps_tiled.argtypes = [V, V, _I64, C.c_double, _I32, _I32, V, C.c_size_t, V]
    lib.cf_ragged_info.argtypes = [V, C.POINTER(_I32), C.POINTER(_I32), C.POINTER(C.c_int64), C.POINTER(_I32)]
    lib.cf_mlp_create.argtypes = [C.POINTER(V), _I32, _I32, _I32, _I32, C.c_uint64, _I32]
    lib.cf_mlp_destroy.argtypes = [V]
    lib.cf_mlp_num_params.argtypes = [V, C.POINTER(C.c_int64)]
    lib.cf_mlp_copy.argtypes = [V, V, _I32]
    lib.cf_mlp_forward.argtypes = [V, V, V, _I64, _I32, V]
    lib.cf_mlp_backward.argtypes = [V, V, V, _I64, V]
    lib.cf_mlp_adam_step.argtypes = [V, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, V]
    lib.cf_precond_probe_loss.argtypes = [V, V, V, V, V, C.c_float, _I64, _I32, _I32, _I32, V, V, V]
    lib.cf_precond_assemble.argtypes = [V, V, V, C.c_float, _I64, _I32, _I32, V]
    lib.cf_gmres_workspace_size.argtypes = [C.c_void_p, _I64, _I32, C.POINTER(C.c_size_t)]
    lib.cf_gmres_solve_tiled.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, _I64, _I32,
                                         _I32, C.c_double, C.c_void_p, _I32, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_size_t, C.c_void_p]
    lib.cf_status_string.restype = C.c_char_p
    lib.cf_status_string.argtypes = [C.c_int]
    lib.cf_last_error.restype = C.c_char_p
    lib.cf_launch_count.restype = C.c_int64
    lib.cf_few_route_last.restype = C.c_int
    lib.cf_version.restype = C.c_char_p
    if path is None:
        _lib = lib
    return lib


def check(status: int) -> None:
    if status != CF_OK:
        lib = load()
        raise CFError(status, lib.cf_last_error().decode(errors="replace"))


def launch_count() -> int:
    return int(load().cf_launch_count())


def few_route_last() -> str:
    """How the calling thread's last host call of at most 8 cells moved its data."""
    return {0: "none", 1: "parameter block", 2: "copies"}[int(load().cf_few_route_last())]


def version() -> str:
    return load().cf_version().decode()
