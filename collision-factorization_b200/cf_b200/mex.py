"""The reference's MEX contraction functions, with their exact calling convention.

These mirror ``angular_first_collision_kernel_mex`` / ``radial_first_collision_kernel_mex``
(src/mex/angular_first_collision_kernel_mex.cpp:5-16, src/mex/radial_first_collision_kernel_mex.cpp:4-17):
eight arguments ``(Q_out, f, labels_sorted, vals_sorted, ic_map_sorted, R_tensor, N_Q, K_len)``, all
double, column-major, Q_out written IN PLACE with ``+=`` and nothing returned -- the reference's
benchmark relies on exactly that (benchmark_collision_contraction_scaling.m:242-244).

Here the work runs on the GPU through libcf_b200.so.  Unlike the reference, bad input raises
``CFError`` (with the C ABI's status) instead of reading out of bounds.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

_D = C.POINTER(C.c_double)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _in(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _operator_args(labels, vals, ic_map, R, N_Q, K_len):
    labels = _in(labels)
    if labels.ndim != 2 or labels.shape[1] != 3:
        raise _lib.CFError(2, f"labels must be N_G x 3, got {labels.shape}")
    n_g = labels.shape[0]  # N_G = mxGetM(labels) (angular_first...:14)
    vals = _in(vals).ravel(order="F")
    ic_map = _in(ic_map).ravel(order="F")
    if vals.size != n_g or ic_map.size != n_g:
        raise _lib.CFError(2, f"vals ({vals.size}) and ic_map ({ic_map.size}) must have N_G = {n_g} entries")
    K = int(N_K := float(np.asarray(K_len).ravel()[0]))
    NQ = int(float(np.asarray(N_Q).ravel()[0]))
    if K != N_K or K < 1:
        raise _lib.CFError(2, f"K_len = {K_len} is not a positive integer")
    R = _in(R)
    if R.size % (K * K * K) != 0:
        raise _lib.CFError(2, f"R has {R.size} elements, not a multiple of K^3 = {K ** 3}")
    n_l = R.size // (K * K * K)
    return labels, vals, ic_map, R, n_g, n_l, NQ, K


def _check_q(Q_out, f, NQ, K):
    if not isinstance(Q_out, np.ndarray) or Q_out.dtype != np.float64 or not Q_out.flags.f_contiguous:
        raise _lib.CFError(1, "Q_out must be a column-major float64 numpy array (it is written in place)")
    if not Q_out.flags.writeable:
        raise _lib.CFError(1, "Q_out is read-only")
    f = _in(f)
    if f.size != NQ * K or Q_out.size != NQ * K:
        raise _lib.CFError(2, f"f and Q_out must hold N_Q*K = {NQ * K} values")
    return f


def angular_first_collision_kernel_mex(Q_out, f, labels_sorted, vals_sorted, ic_map_sorted, R_tensor, N_Q, K_len):
    """Q_out += angular-first contraction of f (in place; returns None like the MEX)."""
    labels, vals, ic, R, n_g, n_l, NQ, K = _operator_args(labels_sorted, vals_sorted, ic_map_sorted, R_tensor, N_Q,
                                                          K_len)
    f = _check_q(Q_out, f, NQ, K)
    lib = _lib.load()
    _lib.check(lib.cf_angular_first(_ptr(Q_out), _ptr(f), _ptr(labels), _ptr(vals), _ptr(ic), _ptr(R), n_g, n_l,
                                    NQ, K))


def radial_first_collision_kernel_mex(Q_out, f, labels_sorted, vals_sorted, ic_map_sorted, R_tensor, N_Q, K_len):
    """Q_out += radial-first contraction of f (in place; returns None like the MEX)."""
    labels, vals, ic, R, n_g, n_l, NQ, K = _operator_args(labels_sorted, vals_sorted, ic_map_sorted, R_tensor, N_Q,
                                                          K_len)
    f = _check_q(Q_out, f, NQ, K)
    lib = _lib.load()
    _lib.check(lib.cf_radial_first(_ptr(Q_out), _ptr(f), _ptr(labels), _ptr(vals), _ptr(ic), _ptr(R), n_g, n_l,
                                   NQ, K))


def contract_batched(Q_out, f, labels, vals, ic_map, R, N_Q, K_len, form: str = "af"):
    """Q_out[N_Q x K x B] += contraction of each cell of f[N_Q x K x B] (host arrays, in place)."""
    lab, v, ic, Rr, n_g, n_l, NQ, K = _operator_args(labels, vals, ic_map, R, N_Q, K_len)
    if not isinstance(Q_out, np.ndarray) or Q_out.dtype != np.float64 or not Q_out.flags.f_contiguous:
        raise _lib.CFError(1, "Q_out must be a column-major float64 numpy array")
    f = _in(f)
    if f.size % (NQ * K) or f.size != Q_out.size:
        raise _lib.CFError(2, "f and Q_out must both be N_Q x K x B")
    B = f.size // (NQ * K)
    lib = _lib.load()
    _lib.check(lib.cf_contract_host(_ptr(Q_out), _ptr(f), B, _ptr(lab), _ptr(v), _ptr(ic), _ptr(Rr), n_g, n_l, NQ,
                                    K, _lib.FORMS[form]))


def collision_jacobian_apply_mex(out, f, v, labels, vals, ic_map, R, N_Q, K_len, exact: int = 0):
    """out += J(f).v = Q(v,f) + Q(f,v) for each cell (host arrays [N_Q x K] or [N_Q x K x B], in place).

    exact: 0 fast, 1 the exact operation order, 2 the q2 <-> q3 folded operator."""
    lab, g, ic, Rr, n_g, n_l, NQ, K = _operator_args(labels, vals, ic_map, R, N_Q, K_len)
    if not isinstance(out, np.ndarray) or out.dtype != np.float64 or not out.flags.f_contiguous:
        raise _lib.CFError(1, "out must be a column-major float64 numpy array")
    f = _in(f)
    v = _in(v)
    if f.size % (NQ * K) or f.size != out.size or v.size != out.size:
        raise _lib.CFError(2, "f, v and out must all be N_Q x K x B")
    B = f.size // (NQ * K)
    lib = _lib.load()
    _lib.check(lib.cf_jacobian_apply_host(_ptr(out), _ptr(f), _ptr(v), B, _ptr(lab), _ptr(g), _ptr(ic), _ptr(Rr),
                                          n_g, n_l, NQ, K, int(exact)))
