"""Pins from the reference's precomputed operators (src/precalc/*.mat, written by MATLAB).

The nine files hold GeneralCollisionTensor objects for K_max = 4, pad 20 (precompute_collision_operator.m:19-25,
55-61): L in {2, 4, 6} at gamma = 0 and L in {2, ..., 12} at gamma = 1.  They are the only artefacts of
the author's own MATLAB run, so they pin the restated pipeline (Gaunt lists, l-triplet map, R) end to end.
This script reads them with ``cf_b200.matfile`` and writes ``precalc_k4_pins.npz``:

* ``{tag}__labels_sha`` / ``{tag}__ic_sha``: SHA-256 of gaunt_labels / ic_map as int32 (exact pins);
* ``{tag}__vals_proj``: gaunt_vals projected on ``cos(0.618 i)``, ``sin(0.377 i)`` and ones;
* ``{tag}__R_proj``: R [K^3 x N_L] projected on the four seeded rows of ``W`` (one value per channel);
* ``{tag}__R``: the full R for the three smallest operators;
* ``{tag}__meta``: (K_max, L_max, alpha, n_g, n_l).

Run from the repository root with the reference tree at $CF_REFERENCE_DIR (default: a `reference`
directory beside this repository):
    python tests/golden/make_precalc_pins.py
"""
from __future__ import annotations

import hashlib
import os
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "collision-factorization_b200"))

from cf_b200.matfile import load_collision_tensor  # noqa: E402

REFERENCE = Path(os.environ.get("CF_REFERENCE_DIR", ROOT.parent / "reference"))
PRECALC = REFERENCE / "src" / "precalc"
OUT = Path(__file__).resolve().parent / "precalc_k4_pins.npz"
FULL = ("l2_g0", "l4_g1", "l6_g0")


def tag_of(path: Path) -> str:
    m = re.fullmatch(r"collisiontensor_k4_l(\d+)_gamma(\d)\.\d\d\.mat", path.name)
    return f"l{m.group(1)}_g{m.group(2)}"


def sha_int32(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(np.rint(a).astype(np.int32)).tobytes()).hexdigest()


def vals_weights(n: int) -> np.ndarray:
    i = np.arange(n, dtype=np.float64)
    return np.stack([np.cos(0.618 * i), np.sin(0.377 * i), np.ones(n)])


def r_weights() -> np.ndarray:
    return np.random.default_rng(20260412).standard_normal((4, 125))


def main():
    W = r_weights()
    out = {"W": W}
    for f in sorted(PRECALC.glob("collisiontensor_k4_*.mat")):
        tag = tag_of(f)
        c = load_collision_tensor(str(f))
        n_l = c.R.shape[3]
        R2 = c.R.reshape(125, n_l, order="F")
        out[f"{tag}__meta"] = np.array([c.K_max, c.L_max, c.alpha, c.labels.shape[0], n_l], dtype=np.float64)
        out[f"{tag}__labels_sha"] = np.array(sha_int32(c.labels))
        out[f"{tag}__ic_sha"] = np.array(sha_int32(c.ic_map))
        out[f"{tag}__vals_proj"] = vals_weights(c.vals.size) @ c.vals
        out[f"{tag}__R_proj"] = (W @ R2).T
        if tag in FULL:
            out[f"{tag}__R"] = np.asfortranarray(c.R)
        print(f"{f.name}: K_max={c.K_max} L={c.L_max} alpha={c.alpha} n_g={c.labels.shape[0]} n_l={n_l}")
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, OUT.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
