"""Ragged batches: cells of several resolutions contracted in one persistent launch.

Each bucket is a CollisionOperator (one (L, K) operator) with its own cells and its own FP64 form.
``RaggedBatch.q`` computes Q for every bucket in one step of the library (cf_ragged_q): the
angular-first buckets with K <= 8 share one fused persistent launch, any other bucket (radial-first,
the exact forms, K > 8) runs its own kernels in the same step.  ``RaggedBatch.q_graph`` replays the
step from a CUDA graph recorded on first use (cf_ragged_graph_launch), which is how a time stepper
calls it once per step.

``autotune`` picks each bucket's form (radial-first against angular-first, plain or q2 <-> q3
folded), the fused launch's routine (pair or tile) and its tail split by timing them on the device,
and keeps the choice in a small JSON cache keyed by the device and the buckets' operators.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
from pathlib import Path

import numpy as np

from . import _lib

FAMILIES = {"pair": 0, "tile": 1}  # routine of the fused launch: mirrored row pairs, or split Phi rows


class RaggedBatch:
    def __init__(self, operators, cells_per_bucket, forms=None, tail_split: int = 4, family: str = "pair"):
        self.ops = list(operators)
        self.cells = [int(c) for c in cells_per_bucket]
        n = len(self.ops)
        if len(self.cells) != n:
            raise _lib.CFError(_lib.CF_EINVAL, "one cell count per bucket")
        self.forms = list(forms) if forms is not None else ["af"] * n
        codes = [_lib.FORMS[f] for f in self.forms]
        self.tail_split = int(tail_split)
        if family not in FAMILIES:
            raise _lib.CFError(_lib.CF_EINVAL, f"family must be one of {sorted(FAMILIES)}")
        self.family = family
        plans = (C.c_void_p * n)(*[op._h.value for op in self.ops])
        counts = (C.c_int64 * n)(*self.cells)
        fc = (C.c_int32 * n)(*codes)
        h = C.c_void_p()
        _lib.check(_lib.load().cf_ragged_create(C.byref(h), plans, counts, fc, n, self.tail_split,
                                                FAMILIES[family]))
        self._h = h
        nu, ct, sm, nf = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int32()
        _lib.check(_lib.load().cf_ragged_info(h, C.byref(nu), C.byref(ct), C.byref(sm), C.byref(nf)))
        self.n_units, self.ctas, self.smem_bytes, self.n_fused = nu.value, ct.value, sm.value, nf.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().cf_ragged_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def flops_q(self) -> float:
        """Algorithmic FLOPs of one step (every bucket's cells through its operator)."""
        return float(sum(op.flops_q * c for op, c in zip(self.ops, self.cells)))

    def _ptrs(self, fs, qs):
        n = len(self.ops)
        if len(fs) != n or len(qs) != n:
            raise _lib.CFError(_lib.CF_EINVAL, "one f and one q array per bucket")
        for op, f, q, c in zip(self.ops, fs, qs, self.cells):
            shape = (c, op.K, op.N_Q)
            if tuple(f.shape) != shape or tuple(q.shape) != shape or not f.is_contiguous() or not q.is_contiguous():
                raise _lib.CFError(_lib.CF_ESHAPE, f"bucket arrays must be contiguous {shape} float64 CUDA tensors")
        fp = (C.c_void_p * n)(*[int(f.data_ptr()) for f in fs])
        qp = (C.c_void_p * n)(*[int(q.data_ptr()) for q in qs])
        return fp, qp

    def q(self, fs, qs, stream=None):
        """qs[b] += Q(fs[b]) for every bucket in one step."""
        import torch

        fp, qp = self._ptrs(fs, qs)
        s = int((stream or torch.cuda.current_stream()).cuda_stream)
        _lib.check(_lib.load().cf_ragged_q(self._h, qp, fp, s))
        return qs

    def launches_per_step(self) -> int:
        """Kernels one step launches: with the tile routine and every non-empty bucket fused, the one
        launch on the cell-major arrays; otherwise two layout passes in and one out per non-empty bucket,
        the fused launch, and one contraction kernel per bucket outside it."""
        if self.family == "tile" and self.n_fused and all(
                self._fused(op, f) for op, c, f in zip(self.ops, self.cells, self.forms) if c > 0):
            return 1
        nb = sum(1 for c in self.cells if c > 0)
        sep = sum(1 for op, c, f in zip(self.ops, self.cells, self.forms)
                  if c > 0 and not self._fused(op, f))
        return 3 * nb + (1 if self.n_fused else 0) + sep

    def _fused(self, op, form) -> bool:
        return form in ("af", "af_sym") and op.K <= 8 and (self.family == "pair" or op.K % 2 == 0)

    def q_resident(self, stream=None):
        """The contraction alone on the resident tiled buffers left by the last step."""
        import torch

        s = int((stream or torch.cuda.current_stream()).cuda_stream)
        _lib.check(_lib.load().cf_ragged_q_resident(self._h, s))

    def q_host(self, fs, qs):
        """qs[b] += Q(fs[b]) for every bucket, with host arrays (numpy arrays or CPU tensors of shape
        (cells, K, N_Q), C-contiguous float64; pinned memory makes the copies asynchronous).  With the
        tile routine and every bucket fused, one launch runs while the buckets are copied in and out
        (cf_ragged_q_host)."""
        import numpy as np

        n = len(self.ops)
        if len(fs) != n or len(qs) != n:
            raise _lib.CFError(_lib.CF_EINVAL, "one f and one q array per bucket")
        fps, qps = [], []
        for op, f, q, c in zip(self.ops, fs, qs, self.cells):
            shape = (c, op.K, op.N_Q)
            for a in (f, q):
                arr = a.numpy() if hasattr(a, "numpy") else a
                if not isinstance(arr, np.ndarray) or arr.dtype != np.float64 or tuple(arr.shape) != shape \
                        or not arr.flags.c_contiguous:
                    raise _lib.CFError(_lib.CF_ESHAPE, f"bucket arrays must be C-contiguous {shape} float64 host arrays")
            fps.append((f.numpy() if hasattr(f, "numpy") else f).ctypes.data)
            qps.append((q.numpy() if hasattr(q, "numpy") else q).ctypes.data)
        fp = (C.c_void_p * n)(*fps)
        qp = (C.c_void_p * n)(*qps)
        _lib.check(_lib.load().cf_ragged_q_host(self._h, qp, fp))
        return qs

    def q_graph(self, fs, qs, stream=None):
        """The same step replayed from a CUDA graph (recorded on first use for these buffers)."""
        import torch

        fp, qp = self._ptrs(fs, qs)
        s = int((stream or torch.cuda.current_stream()).cuda_stream)
        _lib.check(_lib.load().cf_ragged_graph_launch(self._h, qp, fp, s))
        return qs


# ------------------------------------------------------------------------------------- autotuning
def _cache_path() -> Path:
    root = os.environ.get("CF_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "cf_b200")
    return Path(root) / "ragged_autotune.json"


def _key(ops, cells, candidates, tail_splits) -> str:
    import torch

    dev = torch.cuda.get_device_name(ops[0].device) if torch.cuda.is_available() else "none"
    sig = [dev, _lib.version(), list(candidates), list(tail_splits)]
    for op, c in zip(ops, cells):
        sig.append([op.N_Q, op.K, op.n_g, op.n_l, int(c), op.content_digest()])
    return hashlib.sha256(json.dumps(sig).encode()).hexdigest()[:32]


def _time_step(rb: RaggedBatch, fs, qs, reps: int) -> float:
    import torch

    rb.q(fs, qs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        e0.record()
        rb.q(fs, qs)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    return best


def autotune(ops, cells, candidates=("af_sym", "af", "rf"), tail_splits=(0, 4, 16), families=("pair", "tile"),
             reps: int = 5, use_cache: bool = True, seed: int = 0):
    """Choose each bucket's form, the fused launch's routine and its tail split by timing them.

    Returns (forms, tail_split, family, report).  For each routine family, each bucket's candidate
    forms are timed alone (a one-bucket ragged step on that bucket's cells) and the fastest kept; a
    candidate the operator does not support (an unfoldable Gaunt list for af_sym) is skipped.  Then
    the whole step is timed for every (family, tail split) with those forms, and the fastest wins.
    """
    import torch

    cells = [int(c) for c in cells]
    key = _key(ops, cells, list(candidates) + list(families), tail_splits)
    path = _cache_path()
    if use_cache and path.exists():
        try:
            hit = json.loads(path.read_text()).get(key)
            if hit:
                return hit["forms"], hit["tail_split"], hit["family"], dict(hit["report"], cached=True)
        except (OSError, ValueError):
            pass
    rng = np.random.default_rng(seed)
    fs = [torch.from_numpy(1e-2 * rng.standard_normal((c, op.K, op.N_Q))).cuda(op.device) for op, c in zip(ops, cells)]
    qs = [torch.zeros_like(f) for f in fs]
    per_bucket = []
    forms_by_family = {fam: [] for fam in families}
    for op, c, f, q in zip(ops, cells, fs, qs):
        entry = {"N_Q": op.N_Q, "K": op.K, "cells": c, "seconds": {}, "chosen": {}}
        for fam in families:
            times = {}
            for form in candidates:
                try:
                    rb = RaggedBatch([op], [c], [form], tail_split=4, family=fam)
                except _lib.CFError:
                    continue
                times[form] = _time_step(rb, [f], [q], reps)
                rb.close()
            if not times:
                raise _lib.CFError(_lib.CF_EUNSUPPORTED, f"no candidate form runs for bucket N_Q={op.N_Q} K={op.K}")
            best = min(times, key=times.get)
            forms_by_family[fam].append(best)
            entry["seconds"][fam] = times
            entry["chosen"][fam] = best
        per_bucket.append(entry)
    step_times = {}
    for fam in families:
        for ts in tail_splits:
            rb = RaggedBatch(ops, cells, forms_by_family[fam], tail_split=ts, family=fam)
            step_times[f"{fam}/{int(ts)}"] = _time_step(rb, fs, qs, reps)
            rb.close()
    best = min(step_times, key=step_times.get)
    family, tail = best.split("/")[0], int(best.split("/")[1])
    forms = forms_by_family[family]
    report = {"buckets": per_bucket, "step_seconds": step_times, "cached": False}
    if use_cache:
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            data = json.loads(path.read_text()) if path.exists() else {}
            data[key] = {"forms": forms, "tail_split": tail, "family": family, "report": report}
            path.write_text(json.dumps(data, indent=1))
        except (OSError, ValueError):
            pass
    return forms, tail, family, report
