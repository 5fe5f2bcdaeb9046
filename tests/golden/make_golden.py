"""Generate the golden fixtures under tests/golden/ (TEST INFRASTRUCTURE).

    python tests/golden/make_golden.py [--big | --ragged]

Needs the reference tree (to build oracle/_ref with `make -C oracle`).  Writes:

* ``geometry_counts.json``  -- N_G, N_L, S and a digest of (labels, ic_map) of the sorted COO lists
  for L = 0..16, from this project's restatement of the reference's geometry code.
* ``op_<name>.npz``  -- small operators whose R comes from the reference's own quadrature MEX
  (compute_rtensor_sumfac_mex, compiled unmodified): geometry in the reference's find() order and
  in sortrows([ic_map, q1]) order, R, a seeded f, and the reference's own outputs for that f:
  angular_first, radial_first and naive (all from the compiled reference sources, exact build).
    wcu_k2_l2_g0      K_max=2, L=2, gamma=0, pad 16   (tests/TestWCUEigenvalues.m:6-8,30)
    cfg1_k3_l4_g0     K_max=3, L=4, gamma=0, pad 20   (the CPU-runnable configuration)
    hs_k4_l4_g1       K_max=4, L=4, gamma=1, pad 20   (tutorial_chapman_enscog_decay_rates.m)
    bkw_k5_l1_g0      K_max=5, L=1, gamma=0, pad 16   (tutorial_collisions_bwu_solution.m:23-40)
* with --big: ``R_hs_k7_l8_pad20.npy`` and ``R_hs_k7_l10_pad20.npy`` -- hard-sphere R for the
  L=8 and L=10, K=8 configurations (minutes to hours of CPU quadrature).
* with --ragged: ``R_hs_k3_l4_pad20.npy``, ``R_hs_k5_l6_pad20.npy`` and ``R_hs_k5_l8_pad20.npy`` --
  hard-sphere R of the ragged batch's (L, K) = (4, 4), (6, 6) and (8, 6) buckets.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "collision-factorization_b200"))
sys.path.insert(0, str(ROOT))

from cf_b200 import geometry, workloads  # noqa: E402
from oracle import rtensor  # noqa: E402
from oracle.reference import Reference  # noqa: E402

OUT = Path(__file__).resolve().parent

SMALL = {
    "wcu_k2_l2_g0": dict(K_max=2, L=2, gamma=0.0, pad=16, seed=11),
    "cfg1_k3_l4_g0": dict(K_max=3, L=4, gamma=0.0, pad=20, seed=1),
    "hs_k4_l4_g1": dict(K_max=4, L=4, gamma=1.0, pad=20, seed=7),
    "bkw_k5_l1_g0": dict(K_max=5, L=1, gamma=0.0, pad=16, seed=5),
}


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()[:16]


def geometry_counts():
    out = {}
    for L in range(0, 17):
        g = geometry.sort_for_contraction(geometry.generate_geometry(L))
        out[str(L)] = dict(n_g=g.n_g, n_l=g.n_l, n_slices=geometry.slice_count(g),
                           digest=digest(g.labels, g.ic_map))
    (OUT / "geometry_counts.json").write_text(json.dumps(out, indent=1) + "\n")


def small_operator(name: str, K_max: int, L: int, gamma: float, pad: int, seed: int):
    geo = geometry.generate_geometry(L)
    R = rtensor.generate_R(geo, K_max, gamma, pad, pad, flavour="exact")
    srt = geometry.sort_for_contraction(geo)
    K = K_max + 1
    NQ = geo.n_q
    if name.startswith("cfg1"):
        f = workloads.two_maxwellian_mixture(K, L, seed)  # [K, NQ]
    else:
        f = workloads.maxwellian_cells(K, L, 1, seed, amplitude=1e-2)[0]
    f_cm = np.asfortranarray(f.T)  # [NQ x K] column-major
    ref = Reference("exact")
    outs = {}
    for kern in ("af", "rf", "naive"):
        Q = np.zeros((NQ, K), order="F")
        lab = srt if kern != "naive" else geo
        ref.contract(kern, Q, f_cm, lab.labels, lab.vals, lab.ic_map, R, NQ, K)
        outs[f"Q_{kern}"] = Q
    np.savez_compressed(
        OUT / f"op_{name}.npz",
        K_max=K_max, L=L, gamma=gamma, pad=pad, seed=seed,
        labels=geo.labels, vals=geo.vals, ic_map=geo.ic_map,
        labels_sorted=srt.labels, vals_sorted=srt.vals, ic_map_sorted=srt.ic_map,
        l_triplets=rtensor.l_triplets_of(geo), R=R, f=f_cm, **outs,
    )
    print(f"wrote op_{name}.npz: N_G={geo.n_g} N_L={geo.n_l} |Q|={np.abs(outs['Q_af']).max():.3e}", flush=True)


RAGGED = [(3, 4), (5, 6), (5, 8)]  # (K_max, L) of the ragged batch's (L, K) = (4,4), (6,6), (8,6) buckets


def big(K_max: int, L: int):
    geo = geometry.generate_geometry(L)
    R = rtensor.generate_R(geo, K_max, 1.0, 20, 20, flavour="fast")
    np.save(OUT / f"R_hs_k{K_max}_l{L}_pad20.npy", R)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true")
    ap.add_argument("--ragged", action="store_true",
                    help="only the hard-sphere R of the ragged batch's three smaller buckets")
    ap.add_argument("--only", default=None)
    args = ap.parse_args(argv)
    if args.ragged:
        # (L, K) = (4, 4), (6, 6), (8, 6); the fourth bucket, (10, 8), is R_hs_k7_l10_pad20.npy
        for K_max, L in RAGGED:
            big(K_max, L)
        return
    geometry_counts()
    for name, kw in SMALL.items():
        if args.only and args.only != name:
            continue
        small_operator(name, **kw)
    if args.big:
        big(7, 8)
        big(7, 10)


if __name__ == "__main__":
    main()
