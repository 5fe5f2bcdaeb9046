"""Build libcf_b200.so for sm_100a.

    python collision-factorization_b200/build.py [--force] [--jobs N] [--mex]

Compiles csrc/plan.cu (host side and C ABI) and csrc/inst.cu once per K (-DCF_K=1..16) in
parallel with nvcc, links them into cf_b200/libcf_b200.so, and keeps each object's ptxas report
(registers, spills, shared memory) under _build/.  Objects are rebuilt only when a source is
newer.  With --mex it also builds the MEX shim against the stub MEX host that the tests use.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "cf_b200" / "libcf_b200.so"
INCLUDE = HERE.parent / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "--expt-relaxed-constexpr"]
K_VALUES = list(range(1, 17))


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "cf_b200.h"]


def _stale(obj: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in _deps())


def _compile(src: Path, obj: Path, defines: list[str]) -> tuple[Path, str]:
    cmd = [nvcc(), *ARCH, *NVFLAGS, "-I", str(INCLUDE), *defines, "-c", "-o", str(obj), str(src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log = obj.with_suffix(".ptxas.log")
    log.write_text(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name} {defines}:\n{r.stderr[-4000:]}")
    return obj, r.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = True) -> Path:
    BUILD.mkdir(exist_ok=True)
    units = [(CSRC / "plan.cu", BUILD / "plan.o", []), (CSRC / "noalloc.cu", BUILD / "noalloc.o", []),
             (CSRC / "krylov.cu", BUILD / "krylov.o", []), (CSRC / "mlp.cu", BUILD / "mlp.o", []),
             (CSRC / "ragged.cu", BUILD / "ragged.o", []), (CSRC / "stepping.cu", BUILD / "stepping.o", []),
             (CSRC / "rtensor.cu", BUILD / "rtensor.o", []), (CSRC / "split.cu", BUILD / "split.o", []),
             (CSRC / "rfdense.cu", BUILD / "rfdense.o", [])]
    units += [(CSRC / "inst.cu", BUILD / f"inst_k{k}.o", [f"-DCF_K={k}"]) for k in K_VALUES]
    todo = [u for u in units if force or _stale(u[1])]
    if todo:
        jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
        if verbose:
            print(f"[cf_b200] compiling {len(todo)} unit(s) with {jobs} job(s)", flush=True)
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for fut in cf.as_completed([ex.submit(_compile, *u) for u in todo]):
                fut.result()
    objs = [str(u[1]) for u in units]
    if force or todo or not LIB.exists():
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB), *objs, "-lcudart", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
        if verbose:
            print(f"[cf_b200] linked {LIB}", flush=True)
    return LIB


def spill_report() -> list[str]:
    """Kernels whose ptxas report shows spills (empty when none)."""
    bad = []
    for log in sorted(BUILD.glob("*.ptxas.log")):
        fn = None
        for line in log.read_text().splitlines():
            if "Compiling entry function" in line:
                fn = line.split("'")[1] if "'" in line else line
            if "bytes spill" in line and not line.strip().endswith("0 bytes spill stores, 0 bytes spill loads"):
                if "0 bytes spill stores, 0 bytes spill loads" not in line:
                    bad.append(f"{log.name}: {fn}: {line.strip()}")
    return bad


def build_mex_shim(stub_include: Path, out_dir: Path) -> Path:
    """Compile the MEX shim (mex/*.cpp) against a MEX header directory into one test library.

    MATLAB users build the shim with `mex` against MATLAB's own mex.h; the tests build it against
    the stub MEX host in the oracle's mexhost/ directory.
    """
    out_dir.mkdir(parents=True, exist_ok=True)
    out = out_dir / "libcf_mex_shim.so"
    srcs = {
        "angular_first_collision_kernel_mex.cpp": "cfmex_angular_first",
        "radial_first_collision_kernel_mex.cpp": "cfmex_radial_first",
        "collision_jacobian_apply_mex.cpp": "cfmex_jacobian_apply",
    }
    objs = []
    for src, sym in srcs.items():
        obj = out_dir / (Path(src).stem + ".o")
        cmd = ["g++", "-O2", "-fPIC", "-std=c++17", f"-DmexFunction={sym}", "-I", str(stub_include), "-I",
               str(INCLUDE), "-c", "-o", str(obj), str(HERE / "mex" / src)]
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    host = out_dir / "mxhost.o"
    subprocess.run(["gcc", "-O2", "-fPIC", "-I", str(stub_include), "-c", "-o", str(host),
                    str(stub_include / "mxhost.c")], check=True)
    subprocess.run(["g++", "-shared", "-o", str(out), *objs, str(host), f"-L{LIB.parent}", "-lcf_b200",
                    f"-Wl,-rpath,{LIB.parent}"], check=True)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    args = ap.parse_args(argv)
    build(force=args.force, jobs=args.jobs)
    bad = spill_report()
    for b in bad:
        print("[cf_b200] spill:", b)
    return 0


if __name__ == "__main__":
    sys.exit(main())
