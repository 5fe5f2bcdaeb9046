"""The C ABI library loads, exports every declared symbol and refuses to run without a GPU.

No compute call is made here: without a device, every entry point must return CF_ENODEVICE
(there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT


def declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(cf_[A-Za-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    from cf_b200 import _lib

    lib = _lib.load()
    declared = declared_functions()
    assert len(declared) >= 15
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (cf_[A-Za-z0-9_]+)", out))
    assert set(declared) <= exported
    assert set(_lib.EXPORTS) == set(declared)


def test_status_strings_and_version():
    from cf_b200 import _lib

    lib = _lib.load()
    assert lib.cf_status_string(0) == b"ok"
    assert lib.cf_status_string(3) == b"index out of range"
    assert b"sm_100a" in lib.cf_version()


def test_library_is_built_for_sm100a_only():
    from cf_b200 import _lib

    out = subprocess.run(["cuobjdump", "--list-elf", str(_lib.LIB_PATH)], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    archs = set(re.findall(r"sm_(\d+a?)", out.stdout))
    assert archs == {"100a"}, archs


def test_no_cpu_fallback_without_device():
    """Without a CUDA device the entry points return CF_ENODEVICE instead of computing on the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cf_b200 import _lib
    from cf_b200.mex import angular_first_collision_kernel_mex

    Q = np.zeros((4, 1), order="F")
    with pytest.raises(_lib.CFError) as e:
        angular_first_collision_kernel_mex(Q, np.ones((4, 1), order="F"), np.array([[1.0, 1.0, 1.0]]),
                                           np.array([0.5]), np.array([1.0]), np.ones(1), 4, 1)
    assert e.value.status == 7
    lib = _lib.load()
    h = C.c_void_p()
    D = C.POINTER(C.c_double)
    lab = np.array([1.0, 1.0, 1.0])
    st = lib.cf_plan_create(C.byref(h), lab.ctypes.data_as(D), lab.ctypes.data_as(D), lab.ctypes.data_as(D),
                            lab.ctypes.data_as(D), 1, 1, 4, 1, -1)
    assert st == 7


def test_mex_shim_argument_checks(tmp_path):
    """The MEX shim keeps the 8-argument convention and raises MATLAB errors on bad arguments."""
    import sys

    sys.path.insert(0, str(ROOT / "collision-factorization_b200"))
    import build

    so = build.build_mex_shim(ROOT / "oracle" / "mexhost", tmp_path)
    lib = C.CDLL(str(so))
    lib.mxh_wrap.restype = C.c_void_p
    lib.mxh_wrap.argtypes = [C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_size_t)]
    lib.mxh_call.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
    lib.mxh_last_error.restype = C.c_char_p
    lib.mxh_last_error_id.restype = C.c_char_p
    keep = []

    def wrap(a):
        a = np.asfortranarray(np.atleast_2d(np.asarray(a, dtype=np.float64)))
        keep.append(a)
        dims = (C.c_size_t * a.ndim)(*a.shape)
        return lib.mxh_wrap(a.ctypes.data_as(C.POINTER(C.c_double)), a.ndim, dims)

    fn = C.cast(lib.cfmex_angular_first, C.c_void_p)
    # wrong number of inputs
    prhs = (C.c_void_p * 3)(wrap(np.zeros((4, 1))), wrap(np.zeros((4, 1))), wrap(np.zeros((1, 3))))
    assert lib.mxh_call(fn, 0, None, 3, prhs) == 1
    assert b"expected 8 inputs" in lib.mxh_last_error()
    assert lib.mxh_last_error_id() == b"cf_b200:angular_first"
    # labels not N_G x 3
    args = [np.zeros((4, 1)), np.ones((4, 1)), np.ones((2, 2)), np.ones(2), np.ones(2), np.ones(1), 4.0, 1.0]
    prhs = (C.c_void_p * 8)(*[wrap(a) for a in args])
    assert lib.mxh_call(fn, 0, None, 8, prhs) == 1
    assert b"N_G x 3" in lib.mxh_last_error()
    # R not a multiple of K^3
    args = [np.zeros((4, 2)), np.ones((4, 2)), np.ones((1, 3)), np.ones(1), np.ones(1), np.ones(7), 4.0, 2.0]
    prhs = (C.c_void_p * 8)(*[wrap(a) for a in args])
    assert lib.mxh_call(fn, 0, None, 8, prhs) == 1
    assert b"multiple of K_len^3" in lib.mxh_last_error()
