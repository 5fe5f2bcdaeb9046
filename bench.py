#!/usr/bin/env python
"""Benchmark: Q(f) cell-evals/s of the collision contraction on B200.

Workload (default): hard spheres (gamma = 1), L = 10, K = 8 radial functions (M = 968 coefficients
per cell), a batch of B = 4096 cells per GPU, FP64.  Each cell is a seeded Maxwellian plus a
perturbation N(0,1) exp(-0.6 (k+l)) at amplitude 1e-2 (synthetic data).  One step = Q(f) for the
whole batch through the library's public device API (zero Q, layout pass, contraction, layout
pass back).  The batch (f, Q and their tiled copies, ~127 MB) is about the size of L2, so L2 is
flushed with a 256 MB write before every timed step (outside the timed interval).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank takes its own 4096 cells (weak scaling, no collective on the data path);
the reported time is the max over ranks.  ``--impl reference`` times the reference's own
angular_first_collision_kernel_mex, compiled unmodified from its sources (oracle/_ref), once per
cell on all host cores, on the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "collision-factorization_b200"
for _p in (str(PKG), str(ROOT)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "Q(f) cell-evals/s at <=1e-10 rel err vs FP64: plain vs chosen form; % roofline"
WORKLOADS = {
    # name: (L, K, B, gamma)
    "hs_l10_k8_b4096": (10, 8, 4096, 1.0),
    "hs_l8_k8_b2048": (8, 8, 2048, 1.0),
    "hs_l16_k12_b1024": (16, 12, 1024, 1.0),
    "implicit_hs_l8_k8_b2048": (8, 8, 2048, 1.0),
    "ragged_hs_b16384": (10, 8, 16384, 1.0),  # largest bucket's (L, K); buckets in RAGGED_BUCKETS
    "rtensor_hs_k7_l10": (10, 8, 0, 1.0),  # the R-tensor quadrature itself (pad 20)
    "single_g0_l4_k4": (4, 4, 1, 0.0),  # one f per call, Maxwell molecules; latency in us per call
}
# operator of the single-f workload: R from the reference's own quadrature (K_max = 3, pad 20)
SINGLE_OPERATOR = "op_cfg1_k3_l4_g0.npz"
RAGGED_BUCKETS = [(4, 4), (6, 6), (8, 6), (10, 8)]  # (L, K), drawn with RAGGED_WEIGHTS per cell
# hard-sphere R (pad 20) per (L, K): from the reference's own quadrature (compute_rtensor_sumfac_mex,
# compiled unmodified) up to L = 10; at L = 16, K = 12 from this library's GPU quadrature
# (cf_rtensor_sumfac_packed), which equals the reference's to 1e-12 where both can be run
R_FILES = {(10, 8): "R_hs_k7_l10_pad20.npy", (8, 8): "R_hs_k7_l8_pad20.npy", (4, 4): "R_hs_k3_l4_pad20.npy",
           (6, 6): "R_hs_k5_l6_pad20.npy", (8, 6): "R_hs_k5_l8_pad20.npy", (16, 12): "R_hs_k11_l16_pad20.npy"}
R_SOURCES = {(16, 12): "this library's GPU quadrature (cf_rtensor_sumfac_packed, parity-tested against "
                       "compute_rtensor_sumfac_mex), K_max = 11, pad 20"}
# DRAM bytes (read + write) of one contraction launch, from the ncu captures summarised in profiles/
NCU_TRAFFIC = {
    ("hs_l10_k8_b4096", "tile", "af_sym"): (64.769024e6 + 1.074688e6,
                                            "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                                            "profiles/af_tile_kernel_folded_hs_l10_k8_b4096.md"),
    ("hs_l10_k8_b4096", "pair", "af"): (65.9e6 + 1.8e6, "ncu, profiles/af_pair_kernel_hs_l10_k8_b4096.md"),
    ("ragged_hs_b16384", "ragged_cm_0", "af_sym"): (86.157056e6 + 4.121856e6,
                                                   "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                                                   "profiles/af_ragged_stream_kernel_resident_hs_b16384.md"),
    ("ragged_hs_b16384", "ragged_tile_0", "af_sym"): (86.450176e6 + 4.645632e6,
                                                     "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                                                     "profiles/af_ragged_kernel_tile_hs_b16384.md"),
    ("hs_l10_k8_b4096", "tile_cell_major", "af_sym"): (64.777728e6 + 2.003456e6,
                                                       "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                                                       "profiles/af_tile_stream_kernel_folded_hs_l10_k8_b4096.md"),
    ("hs_l16_k12_b1024", "lblock", "af_sym"): (74.657024e6 + 9.41312e6,
                                               "ncu dram__bytes_read.sum + dram__bytes_write.sum of the l-block kernel "
                                               "launch (the pack pass before it not counted), "
                                               "profiles/af_lblock64_kernel_folded_hs_l16_k12_b1024.md"),
}


PROFILE_FORMS = ("af", "af_sym", "af_exact", "rf", "af_sym_i8", "af_f32", "af_sym_f32", "af_bf16", "af_sym_bf16", "rf_dense")


def _profile_forms(text):
    forms = text.split(",")
    for form in forms:
        if form not in PROFILE_FORMS:
            raise argparse.ArgumentTypeError(f"unknown form {form!r}; choose from {', '.join(PROFILE_FORMS)}")
    return text


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="hs_l10_k8_b4096")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=20260)
    ap.add_argument("--train-states", type=int, default=100000)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--form", default="af", type=_profile_forms,
                    help="form(s) launched by --profile, comma-separated (af, af_sym, af_exact, rf, af_sym_i8, "
                         "af_f32, af_sym_f32, af_bf16, af_sym_bf16)")
    ap.add_argument("--path", default="auto", choices=["auto", "gather", "tile", "pair", "pair_l1", "pair_split", "tile_mma",
                                                       "band", "lblock"],
                    help="kernel family of the angular-first contraction")
    ap.add_argument("--entry", choices=("tiled", "device"), default="tiled",
                    help="--profile: launch the tiled kernel (cf_q_tiled) or the device entry point (cf_q_device)")
    ap.add_argument("--profile", action="store_true",
                    help="only build the workload and launch the contraction (steps+1 times); for ncu captures")
    return ap.parse_args(argv)


# --------------------------------------------------------------------------------------------
# workload
# --------------------------------------------------------------------------------------------
def make_operator(L: int, K: int, gamma: float, seed: int):
    from cf_b200 import geometry, workloads

    geo = geometry.sort_for_contraction(geometry.generate_geometry(L))
    rfile = ROOT / "tests" / "golden" / R_FILES.get((L, K), "__none__")
    if rfile.exists() and gamma == 1.0:
        R = np.asfortranarray(np.load(rfile))
        r_source = (f"{R_SOURCES[(L, K)]}: {rfile.name}" if (L, K) in R_SOURCES else
                    f"reference quadrature (compute_rtensor_sumfac_mex, pad 20): {rfile.name}")
    else:
        from cf_b200.geometry import Geometry  # noqa: F401

        lt = np.floor(np.sqrt(geo.labels - 1.0)).astype(np.int64)
        trip = np.zeros((geo.n_l, 3), dtype=np.int64)
        trip[geo.ic_map.astype(np.int64) - 1] = lt
        R = workloads.synthetic_R(trip, K, seed=seed)
        r_source = "seeded synthetic R with the conservation rows zeroed"
    return geo, R, r_source


# workloads whose cells are anisotropic bi-Maxwellians (T_par / T_perp ~ U[0.5, 2]) rather than
# perturbed Maxwellians
BIMAXWELLIAN = {"hs_l16_k12_b1024"}


def make_cells(L: int, K: int, B: int, seed: int, workload: str | None = None):
    from cf_b200 import workloads

    if workload in BIMAXWELLIAN:
        return workloads.bimaxwellian_cells(K, L, B, seed=seed)
    return workloads.maxwellian_cells(K, L, B, seed=seed, amplitude=1e-2, decay=0.6)


def cells_description(workload: str) -> str:
    if workload in BIMAXWELLIAN:
        return "synthetic (seeded bi-Maxwellians, T_par / T_perp ~ U[0.5, 2], unit density and temperature)"
    return "synthetic (seeded Maxwellians + N(0,1) exp(-0.6(k+l)) perturbation, amplitude 1e-2)"


# --------------------------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
            "power_w_max": max(power) if power else None,
        }


# --------------------------------------------------------------------------------------------
# distributed plumbing (timing only; the data path has no collective)
# --------------------------------------------------------------------------------------------
def dist_setup(args):
    """Rank, world size and local device from the launcher's environment; a process group when
    world > 1 (NCCL on GPUs; gloo where no GPU is visible, which the multi-rank host tests use)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if not dist.is_initialized():
            if torch.cuda.is_available():
                torch.cuda.set_device(local)
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                        device_id=torch.device("cuda", local))
            else:
                dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    """Max of x over the ranks (the timed interval of a weak-scaling run is the slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def weak_rate(world: int, cells_per_rank: int, steps: int, local_seconds: float) -> tuple[float, float]:
    """Whole-job cells per second of a weak-scaling run: every rank contracts its own cells, the job
    takes as long as its slowest rank.  Returns (rate, max seconds)."""
    t = dist_max(local_seconds, world)
    return world * cells_per_rank * steps / t, t


def rank_seed(seed: int, rank: int) -> int:
    """Each rank draws its own cells (its shard of the job)."""
    return seed + rank


# --------------------------------------------------------------------------------------------
# CPU baseline: the reference's own kernel, compiled unmodified, once per cell on host cores
# --------------------------------------------------------------------------------------------
def cpu_reference_rate(geo, R, cells, K, target_seconds: float, nthreads: int = 0, kernel: str = "af",
                       reps: int = 5):
    """Cells per second of the reference's kernel, called once per cell under an OpenMP loop over
    cells: the median of `reps` repetitions, each about target_seconds / reps long.  Returns
    (median rate, cells per rep, total seconds, threads)."""
    from oracle.reference import Reference

    ref = Reference("fast")
    nthreads = nthreads or ref.num_threads()
    NQ = geo.n_q
    # calibrate: grow a batch (a multiple of the thread count) until it takes 50 ms or more
    n0 = max(nthreads, 1)
    while True:
        idx = np.arange(n0) % cells.shape[0]
        f0 = np.asfortranarray(cells[idx].transpose(2, 1, 0))
        Q0 = np.zeros_like(f0, order="F")
        t = time.perf_counter()
        ref.batch(kernel, Q0, f0, geo.labels, geo.vals, geo.ic_map, R, NQ, K, nthreads=nthreads)
        dt0 = time.perf_counter() - t
        if dt0 >= 0.05 or n0 >= (1 << 20):
            break
        n0 *= 4
    per_cell = max(dt0, 1e-6) / n0
    n = max(nthreads, int(target_seconds / reps / per_cell) // max(nthreads, 1) * max(nthreads, 1))
    idx = np.arange(n) % cells.shape[0]
    f = np.asfortranarray(cells[idx].transpose(2, 1, 0))
    rates, total = [], 0.0
    for _ in range(reps):
        Q = np.zeros_like(f, order="F")
        t = time.perf_counter()
        ref.batch(kernel, Q, f, geo.labels, geo.vals, geo.ic_map, R, NQ, K, nthreads=nthreads)
        dt = time.perf_counter() - t
        total += dt
        rates.append(n / dt)
    return statistics.median(rates), n, total, nthreads


def cpu_reference_outputs(geo, R, cells, K) -> np.ndarray:
    """Q of each given cell ([n, K, N_Q]) from the reference's angular_first kernel, compiled unmodified,
    on all host cores: the error reference of the forms where the GPU has no exact-order form (K > 8)."""
    from oracle.reference import Reference

    ref = Reference("fast")
    f = np.asfortranarray(cells.transpose(2, 1, 0))
    Qr = np.zeros_like(f, order="F")
    ref.batch("af", Qr, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, nthreads=ref.num_threads())
    return np.ascontiguousarray(Qr.transpose(2, 1, 0))


def cpu_baseline_block(geo, R, cells, K, target_seconds: float) -> dict:
    """The reference's angular_first on all host cores (the baseline), on one core, and its
    radial_first and naive kernels on all cores, each the median of 5 repetitions."""
    rate, n, dt, thr = cpu_reference_rate(geo, R, cells, K, target_seconds)
    one, n1, dt1, _ = cpu_reference_rate(geo, R, cells, K, max(target_seconds / 3, 1.0), nthreads=1)
    out = {"value": rate, "unit": "cell-evals/s", "cores": thr, "kind": "reference",
           "sample": f"5 x {n} cells of this workload through angular_first_collision_kernel_mex compiled unmodified "
                     f"(-O3 -mavx2 -mfma), one call per cell under an OpenMP loop over cells, {dt:.1f} s; median",
           "one_thread": {"value": one, "sample": f"5 x {n1} cells on one thread, {dt1:.1f} s; median"}}
    for kernel in ("rf", "naive"):
        r, nk, dk, _ = cpu_reference_rate(geo, R, cells, K, max(target_seconds / 4, 1.0), kernel=kernel)
        name = {"rf": "radial_first_collision_kernel_mex", "naive": "naive_collision_kernel_mex"}[kernel]
        out[kernel] = {"value": r, "sample": f"5 x {nk} cells through {name} on {thr} threads, {dk:.1f} s; median"}
    return out


# --------------------------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------------------------
def run_ours(args):
    import torch

    import cf_b200
    from cf_b200 import _lib

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L, K, B, gamma = WORKLOADS[args.workload]
    geo, R, r_source = make_operator(L, K, gamma, args.seed)
    NQ = geo.n_q
    M = NQ * K
    cells = make_cells(L, K, B, seed=rank_seed(args.seed, rank), workload=args.workload)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, NQ, K, device=local)
    op.set_kernel_path(args.path)
    lib = _lib.load()

    f = torch.from_numpy(cells).to(dev)
    Q = torch.zeros_like(f)
    ws = torch.empty(op.workspace_bytes(B) // 8 + 64, dtype=torch.float64, device=dev)
    n_tiles = (B + 31) // 32
    fT = torch.zeros(n_tiles * 32 * M, dtype=torch.float64, device=dev)
    QT = torch.zeros_like(fT)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = int(stream.cuda_stream)

    def step(form="af"):
        Q.zero_()
        op.q(f, out=Q, form=form, workspace=ws)

    def kernel_only(form="af"):
        _lib.check(lib.cf_q_tiled(op._h, int(QT.data_ptr()), int(fT.data_ptr()), B, _lib.FORMS[form], sh))

    _lib.check(lib.cf_pack_cells(op._h, int(fT.data_ptr()), int(f.data_ptr()), B, sh))

    # accuracy of every form against the reference's exact operation order: for K <= 8 the GPU's
    # af_exact form on every cell (bitwise equal to the reference MEX); above that the reference's
    # own compiled kernel on a sample of cells, from the CPU-baseline leg (cpu_reference_outputs)
    if K <= 8:
        ref_form, ref_idx = "af_exact", None
        step(ref_form)
        Q_exact = Q.clone()
        den = Q_exact.abs().reshape(B, -1).amax(dim=1).clamp_min(1e-300)
    else:
        ref_form, ref_idx = "reference_sample", np.unique(np.linspace(0, B - 1, 24).astype(np.int64))
        Q_ref = torch.from_numpy(cpu_reference_outputs(geo, R, cells[ref_idx], K)).to(dev)
        den = Q_ref.abs().reshape(len(ref_idx), -1).amax(dim=1).clamp_min(1e-300)

    def form_err() -> float:
        # max over the reference cells of max|Q - Q_ref| / max|Q_ref| (Q: the last step's output)
        if ref_idx is None:
            num = (Q - Q_exact).abs().reshape(B, -1).amax(dim=1)
        else:
            num = (Q[torch.from_numpy(ref_idx).to(dev)] - Q_ref).abs().reshape(len(ref_idx), -1).amax(dim=1)
        return float((num / den).max())

    step("af")
    err_af = form_err()
    inv = Q.reshape(B, -1)[:, [0, 1, 2, 3, NQ]].abs().max().item()

    # FP64 peak of this GPU (DFMA probe, cuBLAS DGEMM)
    probe = ctypes_double()
    _lib.check(lib.cf_fp64_fma_peak(local, probe))
    dfma_tf = probe.value
    dgemm_tf = dgemm_peak(dev)
    peak_tf = max(dfma_tf, dgemm_tf)

    for _ in range(max(args.warmup, 3)):
        step()
        kernel_only()
    torch.cuda.synchronize(dev)

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            fn()
            evs[i][1].record(stream)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in evs]

    clocks = ClockSampler(local)
    dist_barrier(world)
    torch.cuda.synchronize(dev)
    launches0 = _lib.launch_count()
    clocks.start()
    t_wall = time.perf_counter()
    step_ms = timed(step, args.steps)
    t_wall = time.perf_counter() - t_wall
    launches = _lib.launch_count() - launches0
    kern_ms = timed(kernel_only, args.steps)
    rf_ms = timed(lambda: step("rf"), max(2, args.steps // 4))
    # the q2 <-> q3 folded form: accuracy against the exact form, then timing (step and kernel)
    step("af_sym")
    err_sym = form_err()
    sym_ms = timed(lambda: step("af_sym"), args.steps)
    sym_kern_ms = timed(lambda: kernel_only("af_sym"), max(2, args.steps // 2))
    # the folded form's device step is one launch of the tile kernel on the cell-major arrays (no
    # layout passes) when it runs on the tile kernel: then that launch is the roofline kernel
    n0 = _lib.launch_count()
    op.q(f, out=Q, form="af_sym", workspace=ws)
    torch.cuda.synchronize(dev)
    sym_single = _lib.launch_count() - n0 == 1 and _lib.PATH_NAMES[op.info()["last_path"]] == "tile"
    if sym_single:
        sym_kern_ms = timed(lambda: op.q(f, out=Q, form="af_sym", workspace=ws), max(2, args.steps // 2))
    path_ms, sym_path_ms = {}, {}
    for path in ("tile_mma", "pair_split", "pair", "pair_l1", "tile", "gather", "band", "lblock"):
        try:
            op.set_kernel_path(path)
            path_ms[path] = timed(step, max(2, args.steps // 4))
            sym_path_ms[path] = timed(lambda: step("af_sym"), max(2, args.steps // 4))
        except Exception:
            path_ms[path] = None
            sym_path_ms[path] = None
    op.set_kernel_path(args.path)
    # the exact order: the batch kernels up to K = 8, one CTA per (row, cell) above (slow; two steps)
    if K > 8:
        step("af_exact")
        err_exact = form_err()
    else:
        err_exact = 0.0
    exact_ms = timed(lambda: step("af_exact"), max(2, args.steps // 4) if K <= 8 else 2)
    # J(f).v (the Jacobian apply of the implicit solves) on the same cells: fast, folded, exact order
    v_np = np.random.default_rng(args.seed + 5).standard_normal(cells.shape)
    v_np /= np.linalg.norm(v_np.reshape(B, -1), axis=1)[:, None, None]  # unit norm per cell
    v_dev = torch.from_numpy(v_np).to(dev)
    Jout = torch.zeros_like(f)
    jv_ms = {}
    for name, kw in (("jv", {}), ("jv_folded", {"folded": True}), ("jv_exact", {"exact": True}),
                     ("jv_f32", {"fp32": True}), ("jv_folded_f32", {"folded": True, "fp32": True})):
        def jstep(kw=kw):
            Jout.zero_()
            op.jv(f, v_dev, out=Jout, **kw)

        try:
            # the exact order above K = 8 runs on the row kernel (about 0.15 s a step at L = 16): 2 steps
            jv_ms[name] = timed(jstep, 2 if (name == "jv_exact" and K > 8) else max(2, args.steps // 4))
        except Exception:
            jv_ms[name] = None  # a mode this K does not have (the FP32 pair kernel takes even K <= 12)
    # reduced-precision forms (FP32 contraction, FP64 accumulation of Q; BF16 split; the exact int8
    # split on the tensor cores) and the radial-first dense form (FP64): error and throughput
    f32 = {}
    split_ms = None
    rfd_ms = None
    for form in ("af_f32", "af_sym_f32", "af_bf16", "af_sym_bf16", "af_sym_i8", "rf_dense"):
        try:
            step(form)
            err = form_err()
            inv_f = Q.reshape(B, -1)[:, [0, 1, 2, 3, NQ]].abs().max().item()
            ms = timed(lambda: step(form), max(2, args.steps // 4) if form not in ("af_sym_i8", "rf_dense") else args.steps)
            f32[form] = {"cells_per_s": B * len(ms) / (sum(ms) / 1e3), "max_rel_err_vs_fp64": err,
                         "meets_1e-10": bool(err <= 1e-10), "invariants_abs_max": inv_f}
            if form == "af_sym_i8":
                split_ms, err_split = ms, err
            if form == "rf_dense":
                rfd_ms, err_rfd = ms, err
        except Exception as e:
            f32[form] = {"unavailable": str(e)[:160]}
    clk = clocks.stop()
    torch.cuda.synchronize(dev)
    dist_barrier(world)

    # the headline form: the fastest form within 1e-10 of the FP64 (exact-order) result
    cand = {"af": (sum(step_ms) / len(step_ms), err_af, step_ms), "af_sym": (sum(sym_ms) / len(sym_ms), err_sym, sym_ms)}
    if split_ms:
        cand["af_sym_i8"] = (sum(split_ms) / len(split_ms), err_split, split_ms)
    if rfd_ms:
        cand["rf_dense"] = (sum(rfd_ms) / len(rfd_ms), err_rfd, rfd_ms)
    chosen = min((k for k, v in cand.items() if v[1] <= 1e-10), key=lambda k: cand[k][0], default="af")
    chosen_ms = cand[chosen][2]
    value, total_s = weak_rate(world, B, args.steps, sum(chosen_ms) / 1e3 * args.steps / len(chosen_ms))
    ms_per_step = 1e3 * total_s / args.steps
    # the kernel of the device step: one launch on the cell-major arrays for the split form and for the
    # forms on the band kernel (the step's own events time it); else the tiled launch (cf_q_tiled)
    n0 = _lib.launch_count()
    step(chosen)
    torch.cuda.synchronize(dev)
    step_path = _lib.PATH_NAMES[op.info()["last_path"]]
    step_launches = _lib.launch_count() - n0
    if ((step_path in ("split_i8", "band") and step_launches == 1) or step_path == "rf_dense"
            or (step_path == "lblock" and step_launches == 2)):
        kern_list = chosen_ms
        last_path = step_path
    else:
        kern_list = sym_kern_ms if chosen == "af_sym" else kern_ms
        kernel_only(chosen)
        torch.cuda.synchronize(dev)
        last_path = _lib.PATH_NAMES[op.info()["last_path"]]
        if chosen == "af_sym" and sym_single:
            last_path = "tile_cell_major"
    traffic = NCU_TRAFFIC.get((args.workload, last_path, chosen))
    kern_name = {"pair": "af_pair_kernel (persistent, tile-resident, mirrored row pairs)",
                 "pair_split": "af_pair_kernel, split variant (both mirrored rows per lane, k3 halves)",
                 "pair_l1": "af_pair_kernel (R_t through L1)", "tile": "af_tile_kernel (persistent, tile-resident)",
                 "tile_cell_major": "af_tile_stream_kernel, resident (the tile kernel on the cell-major arrays, "
                                    "no layout passes; the whole device step)",
                 "gather": "af_kernel (gathers through L1/L2)",
                 "tile_mma": "af_mma_kernel (tile-resident, K^3 step on the FP64 MMA)",
                 "split_i8": "af_split_kernel (Phi in FP64 on the folded operator, K^3 step on the int8 tensor cores "
                             "(tcgen05.mma kind::i8, exact 6x6-byte split); the whole device step)",
                 "band": "af_band64_kernel (l1-band units, 4 cells' f resident, R_t staged per t by cp.async.bulk, "
                         "FP64; the whole device step)",
                 "lblock": "af_lblock64_kernel (one CTA per l1 band and 8 cells, R_t and the f rows of bands l2 and "
                           "l3 staged per l-triplet by cp.async.bulk into a ring of stages, the band's slices taken "
                           "by the warps one at a time, Phi on the FP64 CUDA cores, K^3 step on the FP64 tensor cores "
                           "(mma.sync m8n8k4); timed with the pack pass before it, the whole device step)",
                 "rf_dense": "rf_dense_kernel (radial step as a dense GEMM over cells per (t, q2), FP64; the device step "
                             "with its f packing and partial-sum reduction)"}.get(last_path, "?")
    kern_s = sum(kern_list) / len(kern_list) / 1e3
    flops_launch = op.flops_q * B
    achieved_tf = flops_launch / kern_s / 1e12
    sym_info = op.sym_info() if chosen in ("af_sym", "af_sym_i8") else None
    exec_flops = (sym_info["flops_q"] if sym_info else op.flops_q) * B
    if chosen == "af_sym_i8":  # the K^3 step runs on the tensor cores: the FP64 pipe executes the Phi step
        exec_flops -= sym_info["n_slices"] * 2.0 * K**3 * B
    exec_tf = exec_flops / kern_s / 1e12

    # end to end through the host C-ABI entry point, pinned host buffers, in the headline form
    e2e = run_e2e(op, geo, R, cells, K, args, world, form=chosen)

    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline_block(geo, R, cells, K, args.cpu_seconds)
            except Exception as e:  # the baseline is reported, not required
                cpu = {"value": None, "unit": "cell-evals/s", "cores": None, "kind": "reference",
                       "sample": f"unavailable: {e}"}
        rf_rate = B / (sum(rf_ms) / len(rf_ms) / 1e3)
        sym_rate = B * len(sym_ms) / (sum(sym_ms) / 1e3)
        plain_rate = B * args.steps / (sum(step_ms) / 1e3)
        exact_rate = B / (sum(exact_ms) / len(exact_ms) / 1e3)
        out = {
            "metric": METRIC,
            "value": value,
            "unit": "cell-evals/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": cells_description(args.workload),
            "config": {
                "workload": args.workload, "L": L, "K": K, "M": M, "cells_per_gpu": B, "gamma": gamma,
                "n_g": op.n_g, "n_l": op.n_l, "n_slices": op.n_slices,
                "form": {"af_sym": "af_sym (FP64, q2<->q3 folded operator)", "af": "af (plain FP64)",
                         "af_sym_i8": "af_sym_i8 (folded operator; Phi in FP64, K^3 step on the int8 tensor cores, "
                                      "exact byte split, FP64 recombination)"}[chosen],
                "R": r_source, "l2": "flushed (256 MB write) before every timed step",
                "parallelism": f"cells sharded, {B} per GPU, no collective",
            },
            "forms": {
                "af": {"cells_per_s": plain_rate, "max_rel_err_vs_fp64": err_af},
                "af_sym": {"cells_per_s": sym_rate, "max_rel_err_vs_fp64": err_sym},
                "af_exact": {"cells_per_s": exact_rate, "max_rel_err_vs_fp64": err_exact},
                "error_reference": {"af_exact": "the reference's exact operation order on every cell (the GPU's "
                                                "af_exact form, bitwise equal to its MEX)",
                                    "reference_sample": f"the reference's angular_first_collision_kernel_mex, compiled "
                                                        f"unmodified, on a sample of {0 if ref_idx is None else len(ref_idx)} "
                                                        f"of the cells (CPU)"}[ref_form],
                "rf": {"cells_per_s": rf_rate},
                "af_by_kernel": {p: (B / (sum(v) / len(v) / 1e3) if v else None) for p, v in path_ms.items()},
                "af_sym_by_kernel": {p: (B / (sum(v) / len(v) / 1e3) if v else None) for p, v in sym_path_ms.items()},
                "jacobian_apply_cells_per_s": {k: (B / (sum(v) / len(v) / 1e3) if v else None) for k, v in jv_ms.items()},
                **f32,
                "chosen": chosen,
                "plain_cells_per_s": plain_rate,
                "chosen_vs_plain": (B * args.steps / total_s) / plain_rate,
            },
            "invariants_abs_max": inv,
            "roofline": {
                "bound": "fp64", "kernel": f"{kern_name}, K={K}" + (" on the folded operator" if chosen == "af_sym" else ""),
                "note": ("FP64-pipe roofline of the reference operator's FLOP; the form runs its K^3 step on the int8 "
                         "tensor cores, so executed_frac counts the folded Phi step only") if chosen == "af_sym_i8" else None,
                "achieved": achieved_tf, "peak": peak_tf,
                "unit": "TFLOP/s", "frac": achieved_tf / peak_tf, "traffic": traffic[0] if traffic else None,
                "traffic_source": traffic[1] if traffic else "no ncu capture of this kernel and form on this workload",
                "algorithmic_flop_per_launch": flops_launch, "kernel_ms": kern_s * 1e3,
                "executed_flop_per_launch": exec_flops, "executed_tflops": exec_tf, "executed_frac": exec_tf / peak_tf,
                "peak_source": f"measured on this GPU in this run: DFMA probe {dfma_tf:.2f}, cuBLAS DGEMM "
                               f"{dgemm_tf:.2f} TFLOP/s (max); MEASURED_PEAKS.json has no FP64 entry",
                "hbm_gbs_algorithmic": 16.0 * M * B / kern_s / 1e9,
            },
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "wall_s_timed_loop": t_wall,
        }
        print(json.dumps(out), flush=True)
    op.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return out


def ctypes_double():
    import ctypes

    return ctypes.c_double()


def dgemm_peak(dev, n: int = 8192, reps: int = 3) -> float:
    import torch

    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 1e30
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n**3 / (best * 1e-3) / 1e12


def run_e2e(op, geo, R, cells, K, args, world, form="af"):
    """Same metric through the host-pointer C-ABI call (cf_contract_host): H2D f and Q, contract, D2H Q."""
    import ctypes

    import torch

    from cf_b200 import _lib

    lib = _lib.load()
    B = cells.shape[0]
    NQ = geo.n_q
    f_h = torch.from_numpy(cells).pin_memory()
    Q_h = torch.zeros_like(f_h).pin_memory()
    D = ctypes.POINTER(ctypes.c_double)
    # the C ABI takes the MEX layouts: labels column-major [N_G x 3]
    lab = np.asfortranarray(geo.labels)
    vals = np.ascontiguousarray(geo.vals)
    ic = np.ascontiguousarray(geo.ic_map)
    Rr = np.asfortranarray(R)
    n_l = Rr.size // K**3

    def call():
        _lib.check(lib.cf_contract_host(ctypes.cast(Q_h.data_ptr(), D), ctypes.cast(f_h.data_ptr(), D), B,
                                        lab.ctypes.data_as(D), vals.ctypes.data_as(D), ic.ctypes.data_as(D),
                                        Rr.ctypes.data_as(D), geo.n_g, n_l, NQ, K, _lib.FORMS[form]))

    # Q_out is zeroed by one host thread before each call, as a caller's own buffer would be
    # (torch's multithreaded fill leaves its worker threads spinning into the timed call)
    Q_np = Q_h.numpy()
    for _ in range(2):
        Q_np.fill(0.0)
        call()
    times = []
    steps = max(3, args.steps // 2)
    for _ in range(steps):
        Q_np.fill(0.0)
        t = time.perf_counter()
        call()
        times.append(time.perf_counter() - t)
    tot = dist_max(sum(times), world)
    nbytes = B * NQ * K * 8
    return {"value": world * B * steps / tot, "unit": "cell-evals/s", "h2d_bytes_per_step": 2 * nbytes,
            "d2h_bytes_per_step": nbytes,
            "form": form,
            "path": "cf_contract_host (the MEX-compatible host entry point: content-keyed plan cache, checked while "
                    "the GPU works from the second call on; the folded fast form at K <= 8 streams the batch through one "
                    "tile-kernel launch while chunks are copied in and out, other forms run the chunked pipeline on "
                    "three streams), pinned host buffers, Q_out zeroed by one host thread before each call (outside "
                    "the timing)"}


# --------------------------------------------------------------------------------------------
# reference arm
# --------------------------------------------------------------------------------------------
def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    from oracle.reference import Reference, reference_available

    L, K, B, gamma = WORKLOADS[args.workload]
    if not reference_available("fast"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_fast.so not built"}), flush=True)
        return None
    if args.workload == "ragged_hs_b16384":
        return run_reference_ragged(args, world)
    geo, R, r_source = make_operator(L, K, gamma, args.seed)
    ref = Reference("fast")
    nthreads = ref.num_threads()
    # size one step so that warmup + steps fit in about two minutes
    budget = 120.0 / max(args.steps + args.warmup, 1)
    cells_all = make_cells(L, K, min(B, 8 * nthreads), seed=args.seed, workload=args.workload)
    f0 = np.asfortranarray(cells_all[:nthreads].transpose(2, 1, 0))
    Q0 = np.zeros_like(f0, order="F")
    t = time.perf_counter()
    ref.batch("af", Q0, f0, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, nthreads=nthreads)
    per_round = time.perf_counter() - t
    rounds = max(1, min(8, int(budget / max(per_round, 1e-6))))
    n = min(cells_all.shape[0], nthreads * rounds)
    f = np.asfortranarray(cells_all[:n].transpose(2, 1, 0))

    def one():
        Q = np.zeros_like(f, order="F")
        ref.batch("af", Q, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, nthreads=nthreads)

    for _ in range(args.warmup):
        one()
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        one()
        times.append(time.perf_counter() - t)
    value = n * args.steps / sum(times)
    sample = (f"{n} cells per step of the {args.workload} workload through angular_first_collision_kernel_mex "
              f"compiled unmodified (-O3 -mavx2 -mfma), one call per cell, OpenMP over cells")
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (same seeded cells as the GPU arm)",
        "config": {"workload": args.workload, "L": L, "K": K, "M": geo.n_q * K, "gamma": gamma, "R": r_source,
                   "cells_per_step": n},
        "cpu_baseline": {"value": value, "unit": "cell-evals/s", "cores": nthreads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return out


def run_reference_ragged(args, world):
    """Reference arm of the ragged workload: every step contracts a sample of each bucket's cells, in
    the batch's bucket proportions, with the reference kernel on all host cores."""
    from cf_b200 import workloads
    from oracle.reference import Reference

    ref = Reference("fast")
    nthreads = ref.num_threads()
    B = WORKLOADS[args.workload][2]
    assign = workloads.ragged_assignment(B, seed=rank_seed(args.seed, 0))
    counts = [int(np.sum(assign == b)) for b in range(len(RAGGED_BUCKETS))]
    frac = 1024.0 / B  # about 1024 cells per step, mixed as in the batch
    per = [max(1, int(round(c * frac))) for c in counts]
    ops = []
    for b, (L, K) in enumerate(RAGGED_BUCKETS):
        geo, R, _ = make_operator(L, K, 1.0, args.seed + 17 * b)
        cells = make_cells(L, K, per[b], seed=args.seed + 101 * b)
        ops.append((geo, R, K, np.asfortranarray(cells.transpose(2, 1, 0))))

    def one():
        for geo, R, K, f in ops:
            Q = np.zeros_like(f, order="F")
            ref.batch("af", Q, f, geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, nthreads=nthreads)

    for _ in range(args.warmup):
        one()
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        one()
        times.append(time.perf_counter() - t)
    n = sum(per)
    value = n * args.steps / sum(times)
    sample = (f"{n} cells per step ({', '.join(f'{p} of L={L} K={K}' for p, (L, K) in zip(per, RAGGED_BUCKETS))}) "
              f"through angular_first_collision_kernel_mex compiled unmodified, one call per cell, OpenMP over cells")
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded cells in the batch's bucket proportions)",
        "config": {"workload": args.workload, "buckets": RAGGED_BUCKETS, "cells_per_step": n},
        "cpu_baseline": {"value": value, "unit": "cell-evals/s", "cores": nthreads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "cell-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return out


def run_profile_ragged(args):
    """Minimal launch sequence for ncu on the ragged mix: the tile routine, no tail split, the folded
    form in every bucket (the autotuner's choice on B200), then steps+1 device steps."""
    import torch

    import cf_b200
    from cf_b200 import workloads
    from cf_b200.ragged import RaggedBatch

    B = WORKLOADS[args.workload][2]
    assign = workloads.ragged_assignment(B, seed=rank_seed(args.seed, 0))
    counts = [int(np.sum(assign == b)) for b in range(len(RAGGED_BUCKETS))]
    ops, fs = [], []
    for b, (L, K) in enumerate(RAGGED_BUCKETS):
        geo, R, _ = make_operator(L, K, 1.0, args.seed + 17 * b)
        ops.append(cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, device=0))
        fs.append(torch.from_numpy(make_cells(L, K, counts[b], seed=args.seed + b)).cuda())
    rb = RaggedBatch(ops, counts, ["af_sym"] * len(ops), tail_split=0, family="tile")
    qs = [torch.zeros_like(f) for f in fs]
    for _ in range(args.steps + 1):
        rb.q(fs, qs)
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.workload, "launches": args.steps + 1, "B": B}))


def run_profile(args):
    """Minimal launch sequence for ncu: pack once, then steps+1 launches of the plain contraction."""
    import torch

    import cf_b200
    from cf_b200 import _lib

    L, K, B, gamma = WORKLOADS[args.workload]
    geo, R, _ = make_operator(L, K, gamma, args.seed)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, device=0)
    op.set_kernel_path(args.path)
    lib = _lib.load()
    f = torch.from_numpy(make_cells(L, K, B, seed=args.seed, workload=args.workload)).cuda()
    M = geo.n_q * K
    fT = torch.zeros(((B + 31) // 32) * 32 * M, dtype=torch.float64, device="cuda")
    QT = torch.zeros_like(fT)
    sh = int(torch.cuda.current_stream().cuda_stream)
    _lib.check(lib.cf_pack_cells(op._h, int(fT.data_ptr()), int(f.data_ptr()), B, sh))
    Q = torch.zeros_like(f)
    for form in args.form.split(","):
        for _ in range(args.steps + 1):
            if args.entry == "device":
                op.q(f, out=Q, form=form)
            else:
                _lib.check(lib.cf_q_tiled(op._h, int(QT.data_ptr()), int(fT.data_ptr()), B, _lib.FORMS[form], sh))
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.workload, "entry": args.entry, "launches": args.steps + 1, "B": B}))


def run_implicit(args):
    """Implicit relaxation configuration: GMRES(30) on (I - dt J(f)) x = r to 1e-10, 2048 cells,
    hard spheres L=8, K=8, dt*nu in {1, 10, 100}; Maxwellian block preconditioner vs the learned one."""
    import torch

    import cf_b200
    from cf_b200 import implicit, workloads
    from cf_b200.learned import LearnedPreconditioner

    L, K, B = 8, 8, 2048
    geo, R, r_source = make_operator(L, K, 1.0, args.seed)
    op = cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K)
    t0 = time.perf_counter()
    lp = LearnedPreconditioner(op, hidden=512, max_batch=4096, scale=0.1, seed=args.seed)
    train = lp.make_samples(args.train_states, dt_nu_values=(1.0, 10.0, 100.0), n_probes=8, seed=args.seed,
                            amp_range=(0.0, 0.3))
    lp.fit_normalisation(train)
    t_gen = time.perf_counter() - t0
    hist = lp.train(train, epochs=args.epochs, batch=512, lr=1e-3)
    t_train = time.perf_counter() - t0 - t_gen
    del train
    val = lp.make_samples(max(1000, args.train_states // 10), dt_nu_values=(1.0, 10.0, 100.0), n_probes=8,
                          seed=args.seed + 7, amp_range=(0.0, 0.3))
    gains = lp.calibrate(val)
    val_loss = {f"{dtn:g}": {"maxwellian": lp.probe_loss(val, dtn / lp.nu, use_net=False),
                             "learned": lp.probe_loss(val, dtn / lp.nu, use_net=True)} for dtn in (1.0, 10.0, 100.0)}
    del val
    cells = workloads.stress_cells(K, L, B, seed=args.seed + 1, amplitude=0.1)
    rng = np.random.default_rng(args.seed + 2)
    cells[:, 0, 4:9] *= rng.uniform(0.0, 3.0, size=(B, 1))
    f = torch.from_numpy(cells).cuda()
    rhs = op.q(f)
    results = {}
    n_exact = 256  # states whose exact block-Jacobi preconditioner is assembled (K N_Q J.v probes each)
    for dtnu in (1.0, 10.0, 100.0):
        dt = dtnu / lp.nu
        row = {}
        for name in ("block", "learned", "none", "block_exact"):
            fs = f[:n_exact] if name == "block_exact" else f
            rs = rhs[:n_exact] if name == "block_exact" else rhs
            if name == "block_exact":
                torch.cuda.synchronize()
                ta = time.perf_counter()
                P_exact = implicit.exact_block_jacobi(op, fs, dt)
                torch.cuda.synchronize()
                t_assemble = time.perf_counter() - ta

            def solve():
                P = (implicit.block_preconditioner(op, dt) if name == "block"
                     else lp.predict(f, dt) if name == "learned" else P_exact if name == "block_exact" else None)
                return implicit.gmres_solve(op, fs, rs, dt, restart=30, tol=1e-10, max_iters=3000, precond=P,
                                            raise_on_timeout=False)
            solve()  # warm-up
            torch.cuda.synchronize()
            t = time.perf_counter()
            x, it, rel = solve()
            torch.cuda.synchronize()
            row[name] = {"seconds": time.perf_counter() - t, "iters_mean": float(it.mean()), "iters_max": int(it.max()),
                         "relres_max": float(rel.max()), "converged": bool(np.all(rel <= 1e-10))}
            if name == "block_exact":
                row[name]["cells"] = n_exact
                row[name]["assembly_seconds"] = t_assemble
                row[name]["note"] = ("exact diagonal blocks of A(f) = I - dt J(f) per state (K N_Q unit-probe J.v "
                                     "each), inverted: the ceiling of any block-diagonal preconditioner; solve time "
                                     "excludes the assembly")
        row["block_on_exact_sample"] = {"iters_mean": float(np.mean(
            implicit.gmres_solve(op, f[:n_exact], rhs[:n_exact], dt, restart=30, tol=1e-10, max_iters=3000,
                                 precond=implicit.block_preconditioner(op, dt), raise_on_timeout=False)[1]))}
        row["speedup_learned_vs_block"] = row["block"]["seconds"] / row["learned"]["seconds"]
        row["learned_network_used"] = bool(lp.uses_network(dt))
        results[f"dt_nu={dtnu:g}"] = row
    out = {"workload": "implicit_hs_l8_k8_b2048", "cells": B, "M": geo.n_q * K, "R": r_source,
           "gmres": "GMRES(30), right block-Jacobi preconditioning, FP64, tol 1e-10 on |b - A x| / |b| per cell",
           "learned": {"train_states": args.train_states, "epochs": args.epochs, "probes_per_state": 8,
                       "loss_first": hist[0], "loss_last": hist[-1], "sample_s": t_gen, "train_s": t_train,
                       "calibrated_gain_by_dt_nu": {f"{k:.3g}": v for k, v in gains.items()},
                       "calibrated_benefit_by_dt_nu": {f"{10 ** k:.3g}": v for k, v in lp.benefit.items()},
                       "min_benefit": lp.min_benefit,
                       "validation_probe_loss": val_loss},
           "results": results}
    print(json.dumps(out), flush=True)
    op.close()
    return out


def run_ragged(args):
    """Ragged batch: 16384 hard-sphere cells drawn 40/30/20/10 % from (L, K) in {(4,4), (6,6), (8,6), (10,8)},
    one step = Q(f) for every cell through one CUDA-graph replay (layout passes, one fused persistent
    launch for the angular-first buckets, the other buckets' kernels), forms and tail split autotuned."""
    import torch

    import cf_b200
    from cf_b200 import _lib, workloads
    from cf_b200.ragged import RaggedBatch, autotune

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    B = WORKLOADS[args.workload][2]
    assign = workloads.ragged_assignment(B, seed=rank_seed(args.seed, rank))
    counts = [int(np.sum(assign == b)) for b in range(len(RAGGED_BUCKETS))]
    ops, geos, Rs, sources, fs_np = [], [], [], [], []
    for b, (L, K) in enumerate(RAGGED_BUCKETS):
        geo, R, src = make_operator(L, K, 1.0, args.seed + 17 * b)
        geos.append(geo)
        Rs.append(R)
        sources.append(f"L={L} K={K}: {src}")
        ops.append(cf_b200.CollisionOperator(geo.labels, geo.vals, geo.ic_map, R, geo.n_q, K, device=local))
        fs_np.append(make_cells(L, K, counts[b], seed=args.seed + rank * 101 + b))
    t0 = time.perf_counter()
    forms, tail, family, tune = autotune(ops, counts, candidates=("af_sym", "af", "rf"), tail_splits=(0, 4, 16),
                                         families=("pair", "tile"), reps=5)
    tune_s = time.perf_counter() - t0
    rb = RaggedBatch(ops, counts, forms, tail_split=tail, family=family)
    fs = [torch.from_numpy(c).to(dev) for c in fs_np]
    qs = [torch.zeros_like(f) for f in fs]

    # accuracy: every bucket against the reference's exact operation order
    rb.q(fs, qs)
    errs = []
    for op, f, q in zip(ops, fs, qs):
        qe = op.q(f, form="af_exact")
        num = (q - qe).abs().reshape(q.shape[0], -1).amax(dim=1)
        den = qe.abs().reshape(q.shape[0], -1).amax(dim=1).clamp_min(1e-300)
        errs.append(float((num / den).max()) if q.shape[0] else 0.0)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        for q in qs:
            q.zero_()
        rb.q_graph(fs, qs)

    def step_eager():
        for q in qs:
            q.zero_()
        rb.q(fs, qs)

    def step_separate():  # the same forms, one library call per bucket (no fused launch, no graph)
        for op, f, q, form in zip(ops, fs, qs, forms):
            q.zero_()
            op.q(f, out=q, form=form)

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            fn()
            evs[i][1].record(stream)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in evs]

    for _ in range(max(args.warmup, 3)):
        step()
        step_eager()
        step_separate()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    dist_barrier(world)
    torch.cuda.synchronize(dev)
    clocks.start()
    launches0 = _lib.launch_count()
    step_ms = timed(step, args.steps)
    launches = _lib.launch_count() - launches0
    eager_ms = timed(step_eager, max(2, args.steps // 2))
    sep_ms = timed(step_separate, max(2, args.steps // 2))
    step()
    kern_ms = timed(rb.q_resident, max(2, args.steps // 2))  # the contraction alone (Q_tiled accumulates)
    clk = clocks.stop()
    torch.cuda.synchronize(dev)
    dist_barrier(world)
    value, total_s = weak_rate(world, B, args.steps, sum(step_ms) / 1e3)
    kern_s = sum(kern_ms) / len(kern_ms) / 1e3
    probe = ctypes_double()
    _lib.check(_lib.load().cf_fp64_fma_peak(local, probe))
    peak_tf = probe.value
    achieved = rb.flops_q / kern_s / 1e12

    # end to end: the host-array call (cf_ragged_q_host) with pinned f and Q_in in and Q out every
    # step; Q is zeroed by one host thread before each call, outside the timing
    f_h = [torch.from_numpy(c).pin_memory() for c in fs_np]
    q_h = [torch.zeros_like(t).pin_memory() for t in f_h]
    q_np = [t.numpy() for t in q_h]
    rb.q_host(f_h, q_h)  # first call: the handle's device copies of the buckets
    e2e_times = []
    n_e2e = max(3, args.steps // 4)
    for _ in range(n_e2e):
        for q in q_np:
            q.fill(0.0)
        t = time.perf_counter()
        rb.q_host(f_h, q_h)
        e2e_times.append(time.perf_counter() - t)
    e2e_s = dist_max(sum(e2e_times), world)
    nbytes = sum(int(x.numel()) * 8 for x in f_h)

    # DRAM bytes of one fused launch from its ncu capture, for the configuration captured there
    ragged_key = "ragged_cm" if rb.launches_per_step() == 1 else f"ragged_{family}"
    ragged_traffic = NCU_TRAFFIC.get((args.workload, f"{ragged_key}_{tail}", "af_sym")) \
        if all(fm == "af_sym" for fm in forms) else None
    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                per = args.cpu_seconds / len(RAGGED_BUCKETS)
                t_mix, desc, thr = 0.0, [], 0
                for b, (L, K) in enumerate(RAGGED_BUCKETS):
                    rate, n, dt, thr = cpu_reference_rate(geos[b], Rs[b], fs_np[b], K, per)
                    t_mix += counts[b] / rate
                    desc.append(f"5 x {n} cells of L={L} K={K} in {dt:.1f} s (median)")
                cpu = {"value": B / t_mix, "unit": "cell-evals/s", "cores": thr, "kind": "reference",
                       "sample": "angular_first_collision_kernel_mex compiled unmodified (-O3 -mavx2 -mfma), one call "
                                 "per cell under an OpenMP loop, per bucket: " + "; ".join(desc)
                                 + "; combined with the batch's bucket counts"}
            except Exception as e:
                cpu = {"value": None, "unit": "cell-evals/s", "cores": None, "kind": "reference",
                       "sample": f"unavailable: {e}"}
        out = {
            "metric": METRIC, "value": value, "unit": "cell-evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Maxwellians + N(0,1) exp(-0.6(k+l)) perturbation, amplitude 1e-2)",
            "config": {"workload": args.workload, "cells_per_gpu": B, "gamma": 1.0,
                       "buckets": [{"L": L, "K": K, "cells": c, "form": fm, "max_rel_err_vs_fp64": e}
                                   for (L, K), c, fm, e in zip(RAGGED_BUCKETS, counts, forms, errs)],
                       "tail_split": tail, "family": family, "fused_units": rb.n_units, "ctas": rb.ctas, "smem_bytes": rb.smem_bytes,
                       "R": sources, "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"cells sharded, {B} per GPU, no collective"},
            "variants": {"graph_step_cells_per_s": value,
                         "eager_step_cells_per_s": B * len(eager_ms) / (sum(eager_ms) / 1e3),
                         "separate_calls_cells_per_s": B * len(sep_ms) / (sum(sep_ms) / 1e3),
                         "contraction_only_cells_per_s": B / kern_s},
            "autotune": dict(tune, seconds=tune_s),
            "roofline": {"bound": "fp64", "kernel": ("af_ragged_stream_kernel, resident (the tile routine on the buckets' "
                                                    "cell-major arrays: the whole step in one persistent launch)"
                                                    if rb.launches_per_step() == 1 else
                                                    f"af_ragged_kernel<{family} routine> (one persistent launch over "
                                                    "the buckets)"),
                         "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s", "frac": achieved / peak_tf,
                         "traffic": ragged_traffic[0] if ragged_traffic else None,
                         "traffic_source": ragged_traffic[1] if ragged_traffic else None,
                         "algorithmic_flop_per_launch": rb.flops_q, "kernel_ms": kern_s * 1e3,
                         "peak_source": "DFMA probe measured on this GPU in this run"},
            "cpu_baseline": cpu,
            "e2e": {"value": world * B * n_e2e / e2e_s, "unit": "cell-evals/s", "h2d_bytes_per_step": 2 * nbytes,
                    "d2h_bytes_per_step": nbytes,
                    "path": "RaggedBatch.q_host (cf_ragged_q_host): pinned host f and Q_in in, Q out, every step; with "
                            "the tile routine the buckets stream through one launch while they are copied in and out"},
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(out), flush=True)
    rb.close()
    for op in ops:
        op.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return out


def cpu_sumfac_estimate(in_args, s) -> dict:
    """The reference's compute_rtensor_sumfac_mex on the host cores, on a bounded sample.

    The reference parallelises over the radial nodes x (OpenMP), and every node, every u of patch 1
    and every y of patch 2 carries the same work.  Sample: one node per thread (all cores busy, one
    round) and the first 2 of the u and y nodes; the wall time is scaled by the rounds over all
    nodes and by the u / y fraction (N_u1 = N_y2 for these grids)."""
    try:
        from oracle.reference import Reference

        ref = Reference("fast")
        thr = ref.num_threads()
        nx = min(thr, s["N_x"])
        n_u = 2
        smp = list(in_args)
        smp[4], smp[5] = in_args[4][:nx], in_args[5][:nx]
        smp[6], smp[7] = in_args[6][:n_u], in_args[7][:n_u]
        smp[10], smp[11] = in_args[10][:n_u], in_args[11][:n_u]
        smp[22] = np.asfortranarray(in_args[22][:, :n_u, :])
        smp[23] = np.asfortranarray(in_args[23][:, :n_u, :, :])
        smp[24] = np.asfortranarray(in_args[24][:n_u, :])
        smp[25] = np.asfortranarray(in_args[25][:n_u, :, :])
        t = time.perf_counter()
        ref.call("ref_sumfac_mexFunction", smp, nlhs=1)
        dt = time.perf_counter() - t
        rounds = math.ceil(s["N_x"] / thr)
        return {"value": dt * rounds * (s["N_u1"] / n_u), "unit": "s", "cores": thr, "kind": "reference",
                "sample": f"compute_rtensor_sumfac_mex compiled unmodified (-O3 -mavx2 -mfma, OpenMP over x) on "
                          f"{nx} of {s['N_x']} radial nodes (one per thread) and {n_u} of the {s['N_u1']} u and "
                          f"{s['N_y2']} y nodes: {dt:.1f} s wall, scaled by {rounds} node rounds and "
                          f"{s['N_u1']}/{n_u}"}
    except Exception as e:
        return {"value": None, "unit": "s", "cores": None, "kind": "reference", "sample": f"unavailable: {e}"}


def run_reference_rtensor(args):
    """Reference arm of the R-tensor workload: the compiled sumfac MEX on the host cores."""
    if int(os.environ.get("RANK", "0")) != 0:
        return None
    from cf_b200 import geometry, rtensor

    L, K_max, pad = 10, 7, 20
    in_args = rtensor.sumfac_inputs(geometry.generate_geometry(L), K_max, 1.0, pad, pad)
    s = rtensor.grid_sizes(K_max, L, pad, pad)
    cpu = cpu_sumfac_estimate(in_args, s)
    out = {"impl": "reference", "metric": "R-tensor quadrature time (hard spheres, K_max=7, L=10, pad 20)",
           "value": cpu["value"], "unit": "s", "n_gpus": 1, "steps": 1, "warmup": 0, "higher_is_better": False,
           "dtype": "f64", "data": "the reference's quadrature inputs (restated driver)",
           "config": {"workload": args.workload, "K_max": K_max, "L": L, "pad": pad},
           "cpu_baseline": cpu, "e2e": {"value": cpu["value"], "unit": "s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return out


def run_rtensor(args):
    """The reduced radial tensor R of hard spheres (K_max = 7, L = 10, pad 20) by the GPU quadrature
    (cf_rtensor_sumfac), against the reference's compute_rtensor_sumfac_mex on the host cores."""
    import torch

    from cf_b200 import geometry, rtensor

    L, K_max, pad = 10, 7, 20
    geo = geometry.generate_geometry(L)
    t0 = time.perf_counter()
    in_args = rtensor.sumfac_inputs(geo, K_max, 1.0, pad, pad)
    prep_s = time.perf_counter() - t0
    steps = max(1, min(args.steps, 5))
    rtensor.compute_R(in_args)  # warm-up (module load, first allocations)
    times, dev_times = [], []
    for _ in range(steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        tm = {}
        R = rtensor.compute_R(in_args, timing=tm)
        times.append(time.perf_counter() - t)
        dev_times.append(tm["device_seconds"])
    fix = ROOT / "tests" / "golden" / "R_hs_k7_l10_pad20.npy"
    err = float(np.max(np.abs(R - np.load(fix))) / np.max(np.abs(R))) if fix.exists() else None
    s = rtensor.grid_sizes(K_max, L, pad, pad)
    points = s["N_x"] * (s["N_u1"] * s["N_t1"] + s["N_y2"] * s["N_t2"]) * s["N_chi"] * s["N_eps"]
    cpu = None if args.no_cpu_baseline else cpu_sumfac_estimate(in_args, s)
    gpu_s = sum(times) / len(times)
    dev_s = sum(dev_times) / len(dev_times)
    out = {"metric": "R-tensor quadrature time (hard spheres, K_max=7, L=10, pad 20)", "value": gpu_s, "unit": "s",
           "n_gpus": 1, "steps": steps, "warmup": 1, "higher_is_better": False, "dtype": "f64",
           "data": "the reference's quadrature inputs (restated driver)",
           "config": {"workload": args.workload, "K_max": K_max, "L": L, "pad": pad, "N_L": int(in_args[1]),
                      "quadrature_points": points, "input_preparation_s_host": prep_s},
           "device_kernels_s": dev_s,
           "host_side_s": gpu_s - dev_s,
           "max_rel_err_vs_committed_reference_R": err, "cpu_baseline": cpu,
           "speedup_vs_cpu_baseline": (cpu["value"] / gpu_s) if cpu and cpu.get("value") else None}
    print(json.dumps(out), flush=True)
    return out


def load_single_operator():
    """The single-f workload's operator (Maxwell molecules, L = 4, K = 4): the COO lists in
    sortrows([ic_map, q1]) order, R from the reference's quadrature, one seeded f and the reference's
    own angular_first output for it."""
    d = np.load(ROOT / "tests" / "golden" / SINGLE_OPERATOR)
    return {k: d[k] for k in d.files}


def single_cell(K: int, L: int, seed: int) -> np.ndarray:
    """One f, [K, N_Q] row-major (= the MEX's column-major [N_Q x K]): the projection of a two-Maxwellian
    mixture with drifts N(0, 0.5^2)^3 and temperatures U[0.5, 1.5], renormalised to unit density."""
    from cf_b200 import workloads

    return workloads.two_maxwellian_mixture(K, L, seed)


def median_us(xs) -> float:
    return 1e6 * statistics.median(xs)


def run_single(args):
    """One f per call (Maxwell molecules, L = 4, K = 4, M = 100): the latency of a call.

    The timed step is one contraction of one device-resident f, timed with CUDA events behind a
    256 MB L2 flush (so the call's launches are queued when the GPU reaches it and the span is the
    device time of the call).  Beside it: the synchronised round trip of the same call from a host
    thread, the MEX-compatible host call cf_angular_first on pageable host arrays (the e2e figure),
    the floors of one empty launch and of the copies, and the reference's compiled kernel on one host
    core."""
    import ctypes

    import torch

    import cf_b200
    from cf_b200 import _lib, mex

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    L, K, _, gamma = WORKLOADS[args.workload]
    d = load_single_operator()
    lab, vals, ic, R = d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], np.asfortranarray(d["R"])
    NQ = (L + 1) ** 2
    M = NQ * K
    op = cf_b200.CollisionOperator(lab, vals, ic, R, NQ, K, device=local)
    lib = _lib.load()

    # parity on the fixture's f: the MEX entry (fast form) and the exact form against the reference's output
    Qm = np.zeros((NQ, K), order="F")
    mex.angular_first_collision_kernel_mex(Qm, d["f"], lab, vals, ic, R, NQ, K)
    q_ref = d["Q_af"]
    err_mex = float(np.abs(Qm - q_ref).max() / np.abs(q_ref).max())
    Qx = np.zeros((NQ, K), order="F")
    mex.contract_batched(Qx, d["f"], lab, vals, ic, R, NQ, K, form="af_exact")
    exact_bitwise = bool(np.array_equal(Qx, q_ref))

    f_host = single_cell(K, L, rank_seed(args.seed, rank))  # [K, N_Q]
    f = torch.from_numpy(f_host.reshape(1, K, NQ).copy()).to(dev)
    Q = torch.zeros_like(f)
    ws = torch.empty(op.workspace_bytes(1) // 8 + 64, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    steps = max(args.steps, 50)

    def call(form):
        op.q(f, out=Q, form=form, workspace=ws)

    def timed_cold(fn, n):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        for i in range(n):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            fn()
            evs[i][1].record(stream)
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) * 1e-3 for a, b in evs]

    def round_trip(fn, n):
        """Host wall time of fn plus a wait for its work, starting from an idle GPU."""
        out = []
        for _ in range(n):
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            fn()
            stream.synchronize()
            out.append(time.perf_counter() - t)
        return out

    forms = ("af", "af_sym", "af_exact", "rf")
    for form in forms:
        for _ in range(max(args.warmup, 3)):
            call(form)
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(local)
    dist_barrier(world)
    torch.cuda.synchronize(dev)
    clocks.start()
    per_form = {}
    for form in forms:
        n0 = _lib.launch_count()
        dev_s = timed_cold(lambda: call(form), steps)
        launches = (_lib.launch_count() - n0) / steps
        op.q(f, out=Q, form=form, workspace=ws)
        torch.cuda.synchronize(dev)
        per_form[form] = {"device_us": median_us(dev_s), "device_us_mean": 1e6 * sum(dev_s) / len(dev_s),
                          "round_trip_us": median_us(round_trip(lambda: call(form), steps)),
                          "launches_per_call": launches, "path": _lib.PATH_NAMES.get(op.info()["last_path"], "?")}
    # floors: one empty launch (a 1-element fill) and the copies of one f
    one = torch.zeros(1, dtype=torch.float64, device=dev)
    floor_launch = median_us(round_trip(lambda: one.fill_(1.0), steps))
    # the same empty launch timed as the calls are (events behind the L2 flush): the device-side floor
    floor_dev_s = timed_cold(lambda: one.fill_(1.0), steps)
    floor_dev_us = 1e6 * sum(floor_dev_s) / len(floor_dev_s)
    fh_pin = torch.from_numpy(f_host.reshape(1, K, NQ).copy()).pin_memory()
    qh_pin = torch.zeros_like(fh_pin).pin_memory()

    def copies():
        f.copy_(fh_pin, non_blocking=True)
        Q.copy_(qh_pin, non_blocking=True)
        qh_pin.copy_(Q, non_blocking=True)

    floor_copies = median_us(round_trip(copies, steps))

    # e2e: the MEX-compatible host entry points on pageable column-major arrays, as MATLAB passes them
    Dp = ctypes.POINTER(ctypes.c_double)
    lab_f, vals_c, ic_c = np.asfortranarray(lab), np.ascontiguousarray(vals), np.ascontiguousarray(ic)
    n_l = R.size // K ** 3
    fq = np.asfortranarray(f_host.T)  # [N_Q x K]
    Qh = np.zeros((NQ, K), order="F")
    opargs = (lab_f.ctypes.data_as(Dp), vals_c.ctypes.data_as(Dp), ic_c.ctypes.data_as(Dp), R.ctypes.data_as(Dp),
              lab_f.shape[0], n_l, NQ, K)
    qp, fp = Qh.ctypes.data_as(Dp), fq.ctypes.data_as(Dp)
    host_calls = {
        "cf_angular_first": lambda: lib.cf_angular_first(qp, fp, *opargs),
        "cf_radial_first": lambda: lib.cf_radial_first(qp, fp, *opargs),
        "cf_contract_host af_exact": lambda: lib.cf_contract_host(qp, fp, 1, *opargs, _lib.FORMS["af_exact"]),
        "cf_contract_host af_sym": lambda: lib.cf_contract_host(qp, fp, 1, *opargs, _lib.FORMS["af_sym"]),
    }
    host_us = {}
    for name, fn in host_calls.items():
        for _ in range(5):
            _lib.check(fn())
        ts = []
        for _ in range(steps):
            Qh.fill(0.0)
            t = time.perf_counter()
            rc = fn()
            ts.append(time.perf_counter() - t)
            _lib.check(rc)
        host_us[name] = {"python_median_us": median_us(ts), "python_mean_us": 1e6 * sum(ts) / len(ts)}
    # the same calls timed in C (cf_time_contract_host: back-to-back calls, no ctypes cost per call),
    # as the reference's kernel is timed; form af with one cell is cf_angular_first's route
    secs = ctypes.c_double()
    for name, form in (("cf_angular_first", "af"), ("cf_radial_first", "rf"),
                       ("cf_contract_host af_exact", "af_exact"), ("cf_contract_host af_sym", "af_sym")):
        _lib.check(lib.cf_time_contract_host(steps, ctypes.byref(secs), qp, fp, 1, *opargs, _lib.FORMS[form]))
        host_us[name]["c_mean_us"] = 1e6 * secs.value / steps
        host_us[name]["route"] = _lib.few_route_last()
    clk = clocks.stop()
    dist_barrier(world)

    # the chosen form: the fastest device call within 1e-10 of the reference's exact order
    Qd = {}
    for form in ("af", "af_sym", "af_exact"):
        Q.zero_()
        call(form)
        Qd[form] = Q.cpu().numpy()
    den = max(np.abs(Qd["af_exact"]).max(), 1e-300)
    errs = {form: float(np.abs(Qd[form] - Qd["af_exact"]).max() / den) for form in Qd}
    ok = [fm for fm in ("af", "af_sym", "af_exact") if errs[fm] <= 1e-10]
    chosen = min(ok, key=lambda fm: per_form[fm]["device_us_mean"])
    t_dev = per_form[chosen]["device_us_mean"] * 1e-6
    value, total_s = weak_rate(world, 1, steps, t_dev * steps)
    e2e_us = host_us["cf_angular_first"]["c_mean_us"]
    out = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                us, n, dt = cpu_reference_single_us(d, f_host, NQ, K, min(args.cpu_seconds, 10.0))
                cpu = {"value": 1e6 / us, "unit": "cell-evals/s", "cores": 1, "kind": "reference",
                       "us_per_call": us,
                       "sample": f"{n} calls of angular_first_collision_kernel_mex compiled unmodified (-O3 -mavx2 "
                                 f"-mfma) on this f, one host thread, {dt:.1f} s"}
            except Exception as e:
                cpu = {"value": None, "unit": "cell-evals/s", "cores": None, "kind": "reference",
                       "sample": f"unavailable: {e}"}
        flops = op.flops_q
        out = {
            "metric": METRIC, "value": value, "unit": "cell-evals/s", "n_gpus": world, "steps": steps,
            "warmup": max(args.warmup, 3), "ms_per_step": 1e3 * total_s / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (one two-Maxwellian mixture, seeded)",
            "config": {"workload": args.workload, "L": L, "K": K, "M": M, "cells_per_gpu": 1, "gamma": gamma,
                       "n_g": op.n_g, "n_l": op.n_l, "n_slices": op.n_slices, "form": chosen,
                       "R": f"reference quadrature (compute_rtensor_sumfac_mex, K_max = 3, pad 20): {SINGLE_OPERATOR}",
                       "l2": "flushed (256 MB write) before every timed call",
                       "parallelism": "one f per call; ranks are independent replicas"},
            "us_per_call": {"device": per_form[chosen]["device_us_mean"], "device_median": per_form[chosen]["device_us"],
                            "e2e_mex_host_call": e2e_us,
                            "cpu_reference_1_thread": cpu.get("us_per_call") if cpu else None},
            "forms": {**per_form, "max_rel_err_vs_exact": errs, "chosen": chosen},
            "host_calls": host_us,
            "parity": {"mex_fast_vs_reference_max_rel": err_mex, "exact_form_bitwise_equal_to_reference": exact_bitwise},
            "floors_us": {"empty_launch_round_trip": floor_launch, "copies_of_one_f_round_trip": floor_copies,
                          "empty_kernel_device": floor_dev_us},
            "roofline": {
                "bound": "latency", "kernel": f"one call in the {chosen} form ({per_form[chosen]['path']})",
                "achieved": t_dev * 1e6, "peak": floor_dev_us, "unit": "us per call (lower is better)",
                "frac": floor_dev_us / (t_dev * 1e6), "traffic": None,
                "note": "one f is 71 kFLOP and 1.6 KB: the call is bound by launch latency, not by FP64 throughput "
                        "or HBM, so the roofline is the device time of an empty one-element kernel timed the same way "
                        "(events behind the L2 flush); frac = that floor / the call's device time",
                "achieved_tflops": flops / t_dev / 1e12, "algorithmic_flop_per_call": flops,
            },
            "cpu_baseline": cpu,
            "e2e": {"value": world * 1e6 / e2e_us, "unit": "cell-evals/s", "h2d_bytes_per_step": 2 * M * 8,
                    "d2h_bytes_per_step": M * 8,
                    "us_per_call": e2e_us,
                    "path": "cf_angular_first's route (cf_contract_host, form af, one cell) on pageable column-major "
                            "arrays, mean host wall time of back-to-back calls timed in C (cf_time_contract_host); "
                            f"f and Q_in travel by {host_us['cf_angular_first']['route']}"},
            "gpu_launches": int(round(per_form[chosen]["launches_per_call"] * steps)),
            "clocks": clk,
        }
        print(json.dumps(out), flush=True)
    op.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return out


def run_profile_single(args):
    """For ncu: the single-f workload's calls only, steps + 1 of each: the MEX-compatible host call
    (cf_angular_first: af_few_param_kernel), the exact form from host arrays
    (af_few_exact_param_kernel) and the device entry point in the folded form (af_few_kernel)."""
    import ctypes

    import torch

    import cf_b200
    from cf_b200 import _lib

    L, K, _, _ = WORKLOADS[args.workload]
    NQ = (L + 1) ** 2
    d = load_single_operator()
    lab, vals = np.asfortranarray(d["labels_sorted"]), np.ascontiguousarray(d["vals_sorted"])
    ic, R = np.ascontiguousarray(d["ic_map_sorted"]), np.asfortranarray(d["R"])
    f_host = single_cell(K, L, args.seed)
    fq, Qh = np.asfortranarray(f_host.T), np.zeros((NQ, K), order="F")
    lib = _lib.load()
    Dp = ctypes.POINTER(ctypes.c_double)
    opargs = (lab.ctypes.data_as(Dp), vals.ctypes.data_as(Dp), ic.ctypes.data_as(Dp), R.ctypes.data_as(Dp),
              lab.shape[0], R.size // K ** 3, NQ, K)
    for _ in range(args.steps + 1):
        _lib.check(lib.cf_angular_first(Qh.ctypes.data_as(Dp), fq.ctypes.data_as(Dp), *opargs))
    for _ in range(args.steps + 1):  # the exact form: af_few_exact_param_kernel
        _lib.check(lib.cf_contract_host(Qh.ctypes.data_as(Dp), fq.ctypes.data_as(Dp), 1, *opargs,
                                        _lib.FORMS["af_exact"]))
    op = cf_b200.CollisionOperator(lab, vals, ic, R, NQ, K)
    f = torch.from_numpy(f_host.reshape(1, K, NQ).copy()).cuda()
    Q = torch.zeros_like(f)
    for _ in range(args.steps + 1):
        op.q(f, out=Q, form="af_sym")
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.workload, "route": _lib.few_route_last(), "Q_abs_max": float(np.abs(Qh).max())}))
    op.close()


def cpu_reference_single_us(d, f_host, NQ, K, target_seconds):
    """µs per call of the reference's compiled angular_first on one host thread (a C loop of calls)."""
    from oracle.reference import Reference

    ref = Reference("fast")
    lab, vals, ic, R = d["labels_sorted"], d["vals_sorted"], d["ic_map_sorted"], d["R"]
    per = 2048  # calls per batch (1.6 MB of f)
    f = np.asfortranarray(np.repeat(f_host.T[:, :, None], per, axis=2))
    Qc = np.zeros_like(f, order="F")
    n, dt = 0, 0.0
    while dt < target_seconds:
        t = time.perf_counter()
        ref.batch("af", Qc, f, lab, vals, ic, R, NQ, K, nthreads=1)
        dt += time.perf_counter() - t
        n += per
    return 1e6 * dt / n, n, dt


def run_reference_single(args):
    """Reference arm of the single-f workload: its compiled angular_first, one call per step, one thread."""
    if int(os.environ.get("RANK", "0")) != 0:
        return None
    from oracle.reference import reference_available

    if not reference_available("fast"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_fast.so not built"}), flush=True)
        return None
    L, K, _, gamma = WORKLOADS[args.workload]
    d = load_single_operator()
    NQ = (L + 1) ** 2
    f_host = single_cell(K, L, rank_seed(args.seed, 0))
    steps = max(args.steps, 50)
    cpu_reference_single_us(d, f_host, NQ, K, 0.2)  # warm-up
    us, n, dt = cpu_reference_single_us(d, f_host, NQ, K, min(args.cpu_seconds, 10.0))
    value = 1e6 / us
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-evals/s", "n_gpus": 1,
        "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": us * 1e-3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (same f as the GPU arm)",
        "config": {"workload": args.workload, "L": L, "K": K, "M": NQ * K, "gamma": gamma, "cells_per_step": 1},
        "us_per_call": us,
        "cpu_baseline": {"value": value, "unit": "cell-evals/s", "cores": 1, "kind": "reference",
                         "sample": f"{n} calls of angular_first_collision_kernel_mex compiled unmodified on one f, "
                                   f"one host thread, {dt:.1f} s"},
        "e2e": {"value": value, "unit": "cell-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return out


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        if args.workload == "single_g0_l4_k4":
            run_reference_single(args)
        elif args.workload == "implicit_hs_l8_k8_b2048":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no implicit solver, "
                                  "Jacobian apply or preconditioner (it steps explicitly with a dense tensor)"}),
                      flush=True)
        elif args.workload == "rtensor_hs_k7_l10":
            run_reference_rtensor(args)
        else:
            run_reference(args)
    elif args.workload == "rtensor_hs_k7_l10" and args.profile:
        # for ncu: one quadrature of a small operator (hard spheres K_max = 4, L = 4, pad 20)
        from cf_b200 import geometry, rtensor

        R = rtensor.compute_R(rtensor.sumfac_inputs(geometry.generate_geometry(4), 4, 1.0, 20, 20))
        print(json.dumps({"profile": "rtensor hs K_max=4 L=4 pad 20", "R_abs_max": float(np.abs(R).max())}))
    elif args.workload == "rtensor_hs_k7_l10":
        run_rtensor(args)
    elif args.workload == "implicit_hs_l8_k8_b2048":
        run_implicit(args)
    elif args.profile and args.workload == "ragged_hs_b16384":
        run_profile_ragged(args)
    elif args.profile and args.workload == "single_g0_l4_k4":
        run_profile_single(args)
    elif args.profile:
        run_profile(args)
    elif args.workload == "ragged_hs_b16384":
        run_ragged(args)
    elif args.workload == "single_g0_l4_k4":
        run_single(args)
    else:
        run_ours(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
