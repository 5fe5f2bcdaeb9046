"""Shared fixtures and the ``gpu`` marker.

``-m "not gpu"`` runs the CPU suite: the oracle against the compiled reference and the golden
fixtures, the host logic, the known-answer tests and the C-ABI export check.  ``-m gpu`` runs the
parity tests proper, which call the sm_100a kernels through the C ABI.
"""
from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "collision-factorization_b200"
GOLDEN = Path(__file__).resolve().parent / "golden"
for p in (str(PKG), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


def load_op(name: str) -> dict:
    with np.load(GOLDEN / f"op_{name}.npz") as z:
        d = {k: z[k] for k in z.files}
    for k in ("K_max", "L", "pad", "seed"):
        d[k] = int(d[k])
    d["gamma"] = float(d["gamma"])
    d["K"] = d["K_max"] + 1
    d["NQ"] = (d["L"] + 1) ** 2
    for k in ("labels", "labels_sorted", "R", "f"):
        d[k] = np.asfortranarray(d[k])
    return d


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle.reference import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference_lib():
    from oracle.reference import Reference, reference_available

    if not reference_available("exact"):
        pytest.skip("oracle/_ref not built (needs the reference tree at build time)")
    return Reference("exact")


@pytest.fixture(scope="session")
def cuda_available():
    try:
        import torch

        ok = torch.cuda.is_available()
    except Exception:
        ok = False
    if not ok:
        pytest.skip("no CUDA device")
    return True


def normwise_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a - b| / max |b| (the parity metric: elementwise relative error is meaningless where Q is 0)."""
    den = float(np.max(np.abs(b))) if b.size else 0.0
    num = float(np.max(np.abs(a - b))) if a.size else 0.0
    return num / den if den > 0 else num


def per_cell_err(a: np.ndarray, b: np.ndarray) -> float:
    """Max over cells of the per-cell normwise error; arrays are [B, ...]."""
    B = a.shape[0]
    a2 = a.reshape(B, -1)
    b2 = b.reshape(B, -1)
    num = np.max(np.abs(a2 - b2), axis=1)
    den = np.max(np.abs(b2), axis=1)
    den = np.where(den > 0, den, 1.0)
    return float(np.max(num / den)) if B else 0.0
