"""Device-resident collision operator for batched cells on one GPU.

``CollisionOperator`` uploads the COO lists and R once (``cf_plan_create``) and then applies
Q(f) or J(f).v to batches of cells held in device memory.  Cell data is a torch CUDA tensor of
shape ``[B, K, N_Q]`` (C-contiguous), which is the same memory as the reference's column-major
``[N_Q x K x B]``.  torch only provides device memory and streams here; the contraction is the
library's own sm_100a kernels.
"""
from __future__ import annotations

import ctypes as C
import hashlib

import numpy as np

from . import _lib


def _np_operator(labels, vals, ic_map, R, K):
    labels = np.asfortranarray(np.asarray(labels, dtype=np.float64))
    vals = np.ascontiguousarray(np.asarray(vals, dtype=np.float64).ravel())
    ic_map = np.ascontiguousarray(np.asarray(ic_map, dtype=np.float64).ravel())
    R = np.asfortranarray(np.asarray(R, dtype=np.float64))
    n_l = R.size // (K * K * K)
    return labels, vals, ic_map, R, n_l


def _dptr(t) -> int:
    return int(t.data_ptr())


def _stream_handle(stream) -> int | None:
    if stream is None:
        import torch

        return int(torch.cuda.current_stream().cuda_stream)
    return int(getattr(stream, "cuda_stream", stream))


# Kernel paths the single-operator autotuner times by default ('auto': the library's measured order).
AUTOTUNE_PATHS = ("auto", "tile", "pair", "gather", "band", "lblock")


def choose_fastest(times: dict) -> str:
    """The candidate with the smallest time; ties go to the earlier candidate (dicts keep order)."""
    return min(times, key=lambda k: (times[k], list(times).index(k)))


def _autotune_cache_path():
    import os
    from pathlib import Path

    root = os.environ.get("CF_B200_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "cf_b200")
    return Path(root) / "kernel_autotune.json"


def _autotune_key(op, B: int, form: str, candidates) -> str:
    import json

    import torch

    dev = torch.cuda.get_device_name(op.device) if torch.cuda.is_available() else "none"
    sig = [dev, _lib.version(), op.N_Q, op.K, op.n_g, op.n_l, op.content_digest(), int(B), form, list(candidates)]
    return hashlib.sha256(json.dumps(sig).encode()).hexdigest()[:32]


def _time_device(fn, reps: int) -> float:
    """Best of `reps` CUDA-event timings of fn() on the current stream, in seconds."""
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(max(1, int(reps))):
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) * 1e-3)
    return best


class CollisionOperator:
    """Q(f) and J(f).v for batches of cells, on the GPU.

    Parameters mirror what the reference's ``GeneralCollisionTensor`` holds
    (src/GeneralCollisionTensor.m:9-12): ``labels [N_G x 3]`` (1-based), ``vals [N_G]``,
    ``ic_map [N_G]`` (1-based), ``R [K x K x K x N_L]``, plus ``N_Q`` and ``K``.
    """

    def __init__(self, labels, vals, ic_map, R, N_Q: int, K: int, device: int = 0):
        self.N_Q, self.K = int(N_Q), int(K)
        lab, v, ic, Rr, n_l = _np_operator(labels, vals, ic_map, R, self.K)
        self.n_g = lab.shape[0]
        self.n_l = n_l
        lib = _lib.load()
        h = C.c_void_p()
        D = C.POINTER(C.c_double)
        _lib.check(lib.cf_plan_create(C.byref(h), lab.ctypes.data_as(D), v.ctypes.data_as(D), ic.ctypes.data_as(D),
                                      Rr.ctypes.data_as(D), self.n_g, n_l, self.N_Q, self.K, int(device)))
        self._h = h
        self.device = int(device)
        self._host_operator = (lab, v, ic, Rr)
        info = _lib.PlanInfo()
        _lib.check(lib.cf_plan_get_info(h, C.byref(info)))
        self.n_slices = int(info.n_slices)
        self.flops_q = float(info.flops_q)
        self.flops_jv = float(info.flops_jv)

    # ------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            _lib.load().cf_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        inf = _lib.PlanInfo()
        _lib.check(_lib.load().cf_plan_get_info(self._h, C.byref(inf)))
        return {f: getattr(inf, f) for f, _ in inf._fields_}

    def content_digest(self) -> str:
        """SHA-256 (hex, 16 chars) of the operator's arrays: names the operator in caches."""
        if not hasattr(self, "_digest"):
            h = hashlib.sha256()
            for a in self._host_operator:
                h.update(np.ascontiguousarray(a).tobytes())
            h.update(f"{self.N_Q},{self.K}".encode())
            self._digest = h.hexdigest()[:16]
        return self._digest

    def sym_info(self) -> dict:
        """Sizes and FLOP counts of the q2 <-> q3 folded operator (built on first use)."""
        import torch

        f = torch.zeros((1, self.K, self.N_Q), dtype=torch.float64, device=f"cuda:{self.device}")
        self.q(f, form="af_sym")  # builds the folded plan
        from . import geometry  # noqa: F401

        return dict(self._sym_counts) if hasattr(self, "_sym_counts") else self._fold_counts()

    def _fold_counts(self) -> dict:
        import numpy as np

        from . import geometry

        lab, vals, ic, R = self._host_operator
        geo = geometry.Geometry(int(round(self.N_Q ** 0.5)) - 1, lab, vals, ic, None)
        flab, fv, fic, _ = geometry.fold_q2q3(geo, np.zeros((self.K, self.K, self.K, self.n_l), order="F"), self.K)
        fgeo = geometry.Geometry(geo.L, flab, fv, fic, None)
        S = geometry.slice_count(fgeo)
        K = self.K
        self._sym_counts = {"n_g": int(flab.shape[0]), "n_slices": S,
                            "flops_q": float(flab.shape[0] * (2 * K * K + K) + S * 2 * K ** 3)}
        return dict(self._sym_counts)

    def set_kernel_path(self, path: str) -> None:
        """'auto' (default), 'gather', 'tile', 'pair', 'pair_l1', 'pair_split', 'tile_mma', 'band' or 'lblock':
        the kernel family of the AF and J.v forms ('band': the FP64 band kernel of the fast Q forms, K = 4, 8,
        12; 'lblock': one CTA per band and 8 cells, f staged per l-triplet, the band's slices shared out
        one at a time, K = 8 and 12)."""
        code = {"auto": 0, "gather": 1, "tile": 2, "pair": 3, "pair_l1": 4, "pair_split": 5, "tile_mma": 6,
                "band": 11, "lblock": 14}[path]
        _lib.check(_lib.load().cf_plan_set_kernel_path(self._h, code))

    def autotune(self, B: int, form: str = "af_sym", candidates=AUTOTUNE_PATHS, reps: int = 5,
                 use_cache: bool = True, seed: int = 0):
        """Pick this operator's kernel family for batches of B cells in `form` by timing every candidate.

        Each candidate path ('auto' is the library's own measured order) runs `form` on B seeded cells
        on the device; a path that does not fit this operator (CF_EUNSUPPORTED) is skipped; the fastest
        is set with set_kernel_path and returned with the timings.  The choice applies to every form
        of the operator (the plan has one kernel path), so tune for the form that dominates.  Choices
        are cached in a JSON file (CF_B200_CACHE, else ~/.cache/cf_b200) keyed by the device, the
        library version, the operator's content digest, B, the form and the candidates.
        """
        import json

        import torch

        key = _autotune_key(self, int(B), form, candidates)
        path = _autotune_cache_path()
        if use_cache and path.exists():
            try:
                hit = json.loads(path.read_text()).get(key)
                if hit:
                    self.set_kernel_path(hit["path"])
                    return hit["path"], dict(hit["report"], cached=True)
            except (OSError, ValueError):
                pass
        rng = np.random.default_rng(seed)
        f = torch.from_numpy(1e-2 * rng.standard_normal((int(B), self.K, self.N_Q))).cuda(self.device)
        out = torch.zeros_like(f)
        times = {}
        for cand in candidates:
            try:
                self.set_kernel_path(cand)
                self.q(f, out=out, form=form)  # builds what the path needs, outside the timing
                torch.cuda.synchronize(self.device)
            except _lib.CFError as e:
                if e.status != _lib.CF_EUNSUPPORTED:
                    raise
                continue
            times[cand] = _time_device(lambda: self.q(f, out=out, form=form), reps)
        if not times:
            raise _lib.CFError(_lib.CF_EUNSUPPORTED, f"no kernel path runs form {form!r} for this operator")
        best = choose_fastest(times)
        self.set_kernel_path(best)
        report = {"seconds": times, "B": int(B), "form": form, "cached": False}
        if use_cache:
            try:
                path.parent.mkdir(parents=True, exist_ok=True)
                data = json.loads(path.read_text()) if path.exists() else {}
                data[key] = {"path": best, "report": report}
                path.write_text(json.dumps(data, indent=1))
            except (OSError, ValueError):
                pass
        return best, report

    def lblock_selftest(self, wait_seconds: float = 1e-3) -> int:
        """Run the l-block kernel's bounded-wait self-test (K = 8 or 12); returns the status (CF_ETIMEOUT
        = 9 when every wait ran out and the kernel returned, which is the expected outcome)."""
        return int(_lib.load().cf_plan_lblock_selftest(self._h, float(wait_seconds)))

    def stream_selftest(self, wait_seconds: float = 1e-3) -> int:
        """Run the streamed host path's bounded-wait self-test; returns the status (CF_ETIMEOUT = 9
        when the kernel's waits ran out and it returned, which is the expected outcome)."""
        return int(_lib.load().cf_plan_stream_selftest(self._h, float(wait_seconds)))

    def workspace_bytes(self, B: int, jacobian: bool = False) -> int:
        n = C.c_size_t()
        _lib.check(_lib.load().cf_plan_workspace_size(self._h, int(B), int(jacobian), C.byref(n)))
        return int(n.value)

    def _check_cells(self, *ts):
        import torch

        B = None
        for t in ts:
            if not isinstance(t, torch.Tensor) or t.dtype != torch.float64 or not t.is_cuda:
                raise _lib.CFError(1, "cell arrays must be float64 CUDA tensors")
            if not t.is_contiguous() or t.dim() != 3 or t.shape[1] != self.K or t.shape[2] != self.N_Q:
                raise _lib.CFError(2, f"cell arrays must be contiguous [B, K={self.K}, N_Q={self.N_Q}]")
            if B is None:
                B = t.shape[0]
            elif t.shape[0] != B:
                raise _lib.CFError(2, "batch sizes differ")
        return B

    def q(self, f, out=None, form: str = "af", stream=None, workspace=None):
        """out += Q(f) for every cell; returns out (zeros if not given)."""
        import torch

        if out is None:
            out = torch.zeros_like(f)
        B = self._check_cells(f, out)
        lib = _lib.load()
        if workspace is None:
            st = lib.cf_q_device(self._h, _dptr(out), _dptr(f), B, _lib.FORMS[form], _stream_handle(stream))
        else:
            st = lib.cf_q_device_ws(self._h, _dptr(out), _dptr(f), B, _lib.FORMS[form], _dptr(workspace),
                                    workspace.numel() * workspace.element_size(), _stream_handle(stream))
        _lib.check(st)
        return out

    def jv(self, f, v, out=None, exact: bool = False, stream=None, folded: bool = False, fp32: bool = False):
        """out += J(f).v = Q(v,f) + Q(f,v) for every cell; returns out.

        exact: the reference-style operation order; folded: the q2 <-> q3 folded operator; fp32: the
        contraction in FP32 (added into the FP64 out; with folded, on the folded operator)."""
        import torch

        if out is None:
            out = torch.zeros_like(f)
        B = self._check_cells(f, v, out)
        if fp32 and exact:
            raise ValueError("the FP32 J.v has no exact-order mode")
        mode = (4 if folded else 3) if fp32 else (2 if folded else int(bool(exact)))
        _lib.check(_lib.load().cf_jv_device(self._h, _dptr(out), _dptr(f), _dptr(v), B, mode, _stream_handle(stream)))
        return out
