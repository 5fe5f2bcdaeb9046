"""ctypes bindings for the oracle libraries (TEST INFRASTRUCTURE).

``Oracle`` wraps liboracle.so (this project's C restatement, oracle/contraction.c).
``Reference`` wraps oracle/_ref/libref_{exact,fast}.so: the reference's own MEX
sources compiled unmodified, driven through the stub MEX host.

All arrays follow the MEX conventions: column-major float64, labels [N_G x 3]
holding 1-based (q1, q2, q3), ic_map 1-based, R [K x K x K x N_L], f and Q
[N_Q x K] per cell (or [N_Q x K x B] batched), Q accumulated in place.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_D = C.POINTER(C.c_double)
_I64 = C.c_int64


def _p(a: np.ndarray) -> _D:
    return a.ctypes.data_as(_D)


def _f64(a) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    return np.asfortranarray(a)


def _check_inputs(labels, vals, ic_map, R, NQ, K):
    labels = _f64(labels)
    vals = _f64(vals).ravel(order="F")
    ic_map = _f64(ic_map).ravel(order="F")
    R = _f64(R)
    NG = labels.shape[0]
    NL = int(R.size // (K * K * K)) if K > 0 else 0
    return labels, vals, ic_map, R, NG, NL


class Oracle:
    """This project's C restatement of the reference kernels."""

    def __init__(self, path: str | os.PathLike | None = None):
        path = Path(path) if path else HERE / "liboracle.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        self.lib = C.CDLL(str(path))
        single = [_D, _D, _D, _D, _D, _D, _I64, C.c_int, C.c_int]
        for name in ("orc_af", "orc_rf", "orc_naive"):
            getattr(self.lib, name).argtypes = single
            getattr(self.lib, name).restype = C.c_int
        self.lib.orc_jv.argtypes = [_D, _D, _D, _D, _D, _D, _D, _I64, C.c_int, C.c_int]
        self.lib.orc_dense.argtypes = [_D, _D, _D, _I64]
        batched = [_D, _D, _I64, _D, _D, _D, _D, _I64, C.c_int, C.c_int, C.c_int]
        for name in ("orc_af_batch", "orc_rf_batch"):
            getattr(self.lib, name).argtypes = batched
            getattr(self.lib, name).restype = C.c_int
        self.lib.orc_jv_batch.argtypes = [_D, _D, _D, _I64, _D, _D, _D, _D, _I64, C.c_int, C.c_int, C.c_int]
        self.lib.orc_num_threads.restype = C.c_int

    def _single(self, name, Q, f, labels, vals, ic_map, R, NQ, K):
        labels, vals, ic_map, R, NG, _ = _check_inputs(labels, vals, ic_map, R, NQ, K)
        f = _f64(f)
        assert Q.dtype == np.float64 and (Q.flags.f_contiguous or Q.ndim == 1)
        rc = getattr(self.lib, name)(_p(Q), _p(f), _p(labels), _p(vals), _p(ic_map), _p(R), NG, NQ, K)
        if rc:
            raise RuntimeError(f"{name} failed ({rc})")
        return Q

    def af(self, Q, f, labels, vals, ic_map, R, NQ, K):
        return self._single("orc_af", Q, f, labels, vals, ic_map, R, NQ, K)

    def rf(self, Q, f, labels, vals, ic_map, R, NQ, K):
        return self._single("orc_rf", Q, f, labels, vals, ic_map, R, NQ, K)

    def naive(self, Q, f, labels, vals, ic_map, R, NQ, K):
        return self._single("orc_naive", Q, f, labels, vals, ic_map, R, NQ, K)

    def jv(self, out, f, v, labels, vals, ic_map, R, NQ, K):
        labels, vals, ic_map, R, NG, _ = _check_inputs(labels, vals, ic_map, R, NQ, K)
        rc = self.lib.orc_jv(_p(out), _p(_f64(f)), _p(_f64(v)), _p(labels), _p(vals), _p(ic_map), _p(R), NG, NQ, K)
        if rc:
            raise RuntimeError("orc_jv failed")
        return out

    def dense(self, Q, f, C_dense, N):
        self.lib.orc_dense(_p(Q), _p(_f64(f)), _p(_f64(C_dense)), int(N))
        return Q

    def af_batch(self, Q, f, labels, vals, ic_map, R, NQ, K, nthreads=0, form="af"):
        labels, vals, ic_map, R, NG, _ = _check_inputs(labels, vals, ic_map, R, NQ, K)
        f = _f64(f)
        B = f.size // (NQ * K)
        fn = self.lib.orc_af_batch if form == "af" else self.lib.orc_rf_batch
        rc = fn(_p(Q), _p(f), B, _p(labels), _p(vals), _p(ic_map), _p(R), NG, NQ, K, int(nthreads))
        if rc:
            raise RuntimeError("orc batch failed")
        return Q

    def jv_batch(self, out, f, v, labels, vals, ic_map, R, NQ, K, nthreads=0):
        labels, vals, ic_map, R, NG, _ = _check_inputs(labels, vals, ic_map, R, NQ, K)
        f = _f64(f)
        B = f.size // (NQ * K)
        rc = self.lib.orc_jv_batch(_p(out), _p(f), _p(_f64(v)), B, _p(labels), _p(vals), _p(ic_map), _p(R), NG,
                                   NQ, K, int(nthreads))
        if rc:
            raise RuntimeError("orc_jv_batch failed")
        return out

    def num_threads(self) -> int:
        return int(self.lib.orc_num_threads())


class Reference:
    """The reference's MEX sources compiled unmodified (oracle/_ref)."""

    KERNELS = {"af": 0, "rf": 1, "naive": 2}

    def __init__(self, flavour: str = "exact", path: str | os.PathLike | None = None):
        path = Path(path) if path else HERE / "_ref" / f"libref_{flavour}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the reference tree exists")
        self.lib = C.CDLL(str(path))
        self.lib.mxh_wrap.argtypes = [_D, C.c_int, C.POINTER(C.c_size_t)]
        self.lib.mxh_wrap.restype = C.c_void_p
        self.lib.mxh_call.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]
        self.lib.mxh_call.restype = C.c_int
        self.lib.mxh_last_error.restype = C.c_char_p
        self.lib.mxh_data.argtypes = [C.c_void_p]
        self.lib.mxh_data.restype = _D
        self.lib.mxh_numel.argtypes = [C.c_void_p]
        self.lib.mxh_numel.restype = C.c_size_t
        self.lib.mxh_ndim.argtypes = [C.c_void_p]
        self.lib.mxh_dim.argtypes = [C.c_void_p, C.c_int]
        self.lib.mxh_dim.restype = C.c_size_t
        self.lib.mxDestroyArray.argtypes = [C.c_void_p]
        self.lib.refh_batch.argtypes = [C.c_int, _D, _D, _I64, _D, _D, _D, _D, _I64, C.c_int, C.c_int, C.c_int,
                                        C.c_int]
        self.lib.refh_batch.restype = C.c_int
        self.lib.refh_num_threads.restype = C.c_int

    # ---- generic MEX call through the stub host ----
    def _wrap(self, a: np.ndarray):
        a = np.asfortranarray(a, dtype=np.float64)
        dims = (C.c_size_t * max(a.ndim, 2))(*(list(a.shape) + [1] * (2 - a.ndim)))
        h = self.lib.mxh_wrap(_p(a), max(a.ndim, 2), dims)
        return h, a

    def call(self, symbol: str, args, nlhs: int = 0):
        """Call a reference mexFunction by symbol; returns a list of numpy outputs."""
        keep = []
        handles = []
        for a in args:
            h, arr = self._wrap(np.atleast_1d(np.asarray(a, dtype=np.float64)) if np.ndim(a) == 0 else a)
            keep.append(arr)
            handles.append(h)
        prhs = (C.c_void_p * len(handles))(*handles)
        plhs = (C.c_void_p * max(nlhs, 1))()
        fn = C.cast(getattr(self.lib, symbol), C.c_void_p)
        rc = self.lib.mxh_call(fn, nlhs, plhs, len(handles), prhs)
        for h in handles:
            self.lib.mxDestroyArray(h)
        if rc:
            raise RuntimeError(f"{symbol}: {self.lib.mxh_last_error().decode()}")
        outs = []
        for i in range(nlhs):
            h = plhs[i]
            nd = self.lib.mxh_ndim(h)
            shape = tuple(self.lib.mxh_dim(h, d) for d in range(nd))
            n = self.lib.mxh_numel(h)
            buf = np.ctypeslib.as_array(self.lib.mxh_data(h), shape=(n,)).copy()
            outs.append(buf.reshape(shape, order="F"))
            self.lib.mxDestroyArray(h)
        return outs

    # ---- the contraction kernels, MEX calling convention (Q modified in place) ----
    def contract(self, kernel: str, Q: np.ndarray, f, labels, vals, ic_map, R, NQ: int, K: int):
        """Run angular_first / radial_first / naive exactly as MATLAB would call it for one f."""
        assert Q.dtype == np.float64 and Q.flags.f_contiguous
        sym = {"af": "ref_af_mexFunction", "rf": "ref_rf_mexFunction", "naive": "ref_naive_mexFunction"}[kernel]
        args = [Q, _f64(f), _f64(labels), _f64(vals).reshape(-1, 1), _f64(ic_map).reshape(-1, 1), _f64(R),
                np.array([float(NQ)]), np.array([float(K)])]
        # wrap Q without copying so the in-place write lands in the caller's array
        handles = []
        keep = []
        for a in args:
            h, arr = self._wrap(a)
            handles.append(h)
            keep.append(arr)
        assert keep[0] is Q or np.shares_memory(keep[0], Q)
        prhs = (C.c_void_p * len(handles))(*handles)
        rc = self.lib.mxh_call(C.cast(getattr(self.lib, sym), C.c_void_p), 0, None, len(handles), prhs)
        for h in handles:
            self.lib.mxDestroyArray(h)
        if rc:
            raise RuntimeError(self.lib.mxh_last_error().decode())
        return Q

    def dense(self, Q: np.ndarray, f, C_dense, N: int):
        handles, keep = [], []
        for a in (Q, _f64(f), _f64(C_dense).reshape(-1, 1), np.array([float(N)])):
            h, arr = self._wrap(a)
            handles.append(h)
            keep.append(arr)
        prhs = (C.c_void_p * 4)(*handles)
        rc = self.lib.mxh_call(C.cast(self.lib.ref_dense_mexFunction, C.c_void_p), 0, None, 4, prhs)
        for h in handles:
            self.lib.mxDestroyArray(h)
        if rc:
            raise RuntimeError(self.lib.mxh_last_error().decode())
        return Q

    def batch(self, kernel: str, Q: np.ndarray, f: np.ndarray, labels, vals, ic_map, R, NQ: int, K: int,
              nthreads: int = 0):
        """Call the reference kernel once per cell of [N_Q x K x B] f under an OpenMP loop over cells."""
        labels, vals, ic_map, R, NG, NL = _check_inputs(labels, vals, ic_map, R, NQ, K)
        assert Q.dtype == np.float64 and Q.flags.f_contiguous
        f = _f64(f)
        B = f.size // (NQ * K)
        rc = self.lib.refh_batch(self.KERNELS[kernel], _p(Q), _p(f), B, _p(labels), _p(vals), _p(ic_map), _p(R),
                                 NG, NL, NQ, K, int(nthreads))
        if rc:
            raise RuntimeError("refh_batch failed")
        return Q

    def num_threads(self) -> int:
        return int(self.lib.refh_num_threads())


def reference_available(flavour: str = "exact") -> bool:
    return (HERE / "_ref" / f"libref_{flavour}.so").exists()
