"""The MEX shim's compute path on the GPU.

The shim (collision-factorization_b200/mex/*.cpp) is what a MATLAB user compiles with `mex` in
place of the reference's angular_first_collision_kernel_mex / radial_first_collision_kernel_mex.
MATLAB is not on either machine, so the shim is built here against the stub MEX host
(oracle/mexhost) and called through its mexFunction exactly as
benchmark_collision_contraction_scaling.m:96-108 calls the reference (eight real double arrays,
Q_out updated in place, nothing returned; call_mex_out at :242-244 reads Q_out back).

Checked against the golden outputs of the reference's own compiled kernels and against the oracle:
single f on the four golden operators, Q_out nonzero on entry (the += of
angular_first_collision_kernel_mex.cpp:68), one N_Q x K x B batch, and the J(f).v shim.
Tolerance: 1e-12 normwise (max |dQ| / max |Q|), the FP64 bar of the parity suite.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import ROOT, load_op, normwise_err, per_cell_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
OPS = ["wcu_k2_l2_g0", "cfg1_k3_l4_g0", "hs_k4_l4_g1", "bkw_k5_l1_g0"]


class Shim:
    def __init__(self, tmp_path_factory):
        import sys

        sys.path.insert(0, str(ROOT / "collision-factorization_b200"))
        import build

        so = build.build_mex_shim(ROOT / "oracle" / "mexhost", tmp_path_factory.mktemp("mexshim"))
        lib = C.CDLL(str(so))
        lib.mxh_wrap.restype = C.c_void_p
        lib.mxh_wrap.argtypes = [C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_size_t)]
        lib.mxh_call.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
        lib.mxh_last_error.restype = C.c_char_p
        self.lib = lib

    def call(self, symbol: str, *args) -> None:
        """mexFunction(0, NULL, nargs, prhs); array arguments are borrowed, so in-place writes land in them."""
        keep = []
        handles = []
        for a in args:
            if np.isscalar(a):
                a = np.array([[float(a)]])
            assert a.dtype == np.float64 and a.flags.f_contiguous
            keep.append(a)
            dims = (C.c_size_t * a.ndim)(*a.shape)
            handles.append(self.lib.mxh_wrap(a.ctypes.data_as(C.POINTER(C.c_double)), a.ndim, dims))
        prhs = (C.c_void_p * len(handles))(*handles)
        fn = C.cast(getattr(self.lib, symbol), C.c_void_p)
        rc = self.lib.mxh_call(fn, 0, None, len(handles), prhs)
        assert rc == 0, self.lib.mxh_last_error().decode()


@pytest.fixture(scope="module")
def shim(tmp_path_factory, cuda_available):
    return Shim(tmp_path_factory)


def _op_args(d):
    return (np.asfortranarray(d["labels_sorted"]), np.asfortranarray(d["vals_sorted"].reshape(-1, 1)),
            np.asfortranarray(d["ic_map_sorted"].reshape(-1, 1)), np.asfortranarray(d["R"]), float(d["NQ"]),
            float(d["K"]))


@pytest.mark.parametrize("name", OPS)
def test_shim_single_f_matches_reference(shim, name):
    """One f per call, the reference's own calling pattern; Q_out starts at zero."""
    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    for sym, key in (("cfmex_angular_first", "Q_af"), ("cfmex_radial_first", "Q_rf")):
        Q = np.zeros((NQ, K), order="F")
        shim.call(sym, Q, np.asfortranarray(d["f"]), *_op_args(d))
        assert normwise_err(Q, d[key]) <= TOL, (sym, normwise_err(Q, d[key]))


@pytest.mark.parametrize("name", OPS)
def test_shim_accumulates_into_nonzero_q_out(shim, name):
    """Q_out += Q(f): a nonzero, non-round Q_out on entry keeps its value under the added result."""
    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    rng = np.random.default_rng(7)
    Q0 = np.asfortranarray(rng.standard_normal((NQ, K)) * np.abs(d["Q_af"]).max())
    for sym, key in (("cfmex_angular_first", "Q_af"), ("cfmex_radial_first", "Q_rf")):
        Q = Q0.copy(order="F")
        shim.call(sym, Q, np.asfortranarray(d["f"]), *_op_args(d))
        err = np.abs(Q - (Q0 + d[key])).max() / max(np.abs(d[key]).max(), np.abs(Q0).max())
        assert err <= TOL, (sym, err)


def test_shim_batch_matches_oracle(shim, oracle_lib):
    """An N_Q x K x B batch in one call: every cell equals the oracle's single-f result."""
    from cf_b200 import workloads

    d = load_op("hs_k4_l4_g1")
    NQ, K = d["NQ"], d["K"]
    B = 37
    cells = workloads.maxwellian_cells(K, d["L"], B, seed=11)  # [B, K, NQ]
    f = np.asfortranarray(cells.transpose(2, 1, 0))  # [NQ, K, B]
    args = _op_args(d)
    ref = np.zeros((B, K, NQ))
    for b in range(B):
        Qb = np.zeros((NQ, K), order="F")
        oracle_lib.af(Qb, np.asfortranarray(f[:, :, b]), d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"],
                      d["R"], NQ, K)
        ref[b] = Qb.T
    for sym in ("cfmex_angular_first", "cfmex_radial_first"):
        Q = np.zeros((NQ, K, B), order="F")
        shim.call(sym, Q, f, *args)
        got = np.ascontiguousarray(Q.transpose(2, 1, 0))
        assert per_cell_err(got, ref) <= TOL, (sym, per_cell_err(got, ref))


@pytest.mark.parametrize("name", ["cfg1_k3_l4_g0", "hs_k4_l4_g1"])
def test_shim_jacobian_apply_matches_oracle(shim, oracle_lib, name):
    """collision_jacobian_apply_mex(out, f, v, ...): out += J(f).v, against the oracle's bilinear form."""
    d = load_op(name)
    NQ, K = d["NQ"], d["K"]
    rng = np.random.default_rng(3)
    v = np.asfortranarray(rng.standard_normal((NQ, K)))
    ref = np.zeros((NQ, K), order="F")
    oracle_lib.jv(ref, d["f"], v, d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"], NQ, K)
    out0 = np.asfortranarray(rng.standard_normal((NQ, K)))
    out = out0.copy(order="F")
    shim.call("cfmex_jacobian_apply", out, np.asfortranarray(d["f"]), v, *_op_args(d))
    err = np.abs(out - (out0 + ref)).max() / max(np.abs(ref).max(), np.abs(out0).max())
    assert err <= TOL, err
