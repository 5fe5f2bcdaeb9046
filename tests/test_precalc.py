"""The reference's precomputed operators (src/precalc/*.mat, MATLAB v7.3) against the restated pipeline.

The nine files are the only outputs of the author's own MATLAB run.  ``tests/golden/precalc_k4_pins.npz``
holds exact hashes of their Gaunt labels and l-triplet maps, projections of their Gaunt values and
R tensors, and three full R tensors (``make_precalc_pins.py`` reads the files with ``cf_b200.matfile``).
"""
from __future__ import annotations

import hashlib
import os
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
# the reference tree: $CF_REFERENCE_DIR, else a `reference` directory beside this repository
REFERENCE = Path(os.environ.get("CF_REFERENCE_DIR", Path(__file__).resolve().parents[2] / "reference"))
PRECALC = REFERENCE / "src" / "precalc"
TAGS = ["l2_g0", "l4_g0", "l6_g0", "l2_g1", "l4_g1", "l6_g1", "l8_g1", "l10_g1", "l12_g1"]


@pytest.fixture(scope="module")
def pins():
    with np.load(GOLDEN / "precalc_k4_pins.npz") as z:
        return {k: z[k] for k in z.files}


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(np.rint(a).astype(np.int32)).tobytes()).hexdigest()


def _vals_weights(n):
    i = np.arange(n, dtype=np.float64)
    return np.stack([np.cos(0.618 * i), np.sin(0.377 * i), np.ones(n)])


@pytest.mark.parametrize("tag", TAGS)
def test_restated_geometry_equals_matlab(tag, pins):
    """Gaunt labels and l-triplet map bit-exact, Gaunt values to rounding, at every saved L."""
    from cf_b200 import geometry

    K_max, L, alpha, n_g, n_l = pins[f"{tag}__meta"]
    geo = geometry.generate_geometry(int(L))
    assert geo.n_g == int(n_g) and geo.n_l == int(n_l)
    assert _sha(geo.labels) == str(pins[f"{tag}__labels_sha"])
    assert _sha(geo.ic_map) == str(pins[f"{tag}__ic_sha"])
    proj = _vals_weights(geo.n_g) @ geo.vals
    ref = pins[f"{tag}__vals_proj"]
    assert np.max(np.abs(proj - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("tag,gamma", [("l2_g0", 0.0), ("l2_g1", 1.0)])
def test_reference_quadrature_reproduces_matlab_R(tag, gamma, pins, reference_lib):
    """The reference's sumfac kernel fed by the restated MATLAB driver gives MATLAB's saved R."""
    from cf_b200 import geometry
    from oracle import rtensor

    geo = geometry.generate_geometry(2)
    R = rtensor.generate_R(geo, 4, gamma, 20, 20)
    n_l = R.shape[3]
    P = (pins["W"] @ R.reshape(125, n_l, order="F")).T
    ref = pins[f"{tag}__R_proj"]
    assert np.max(np.abs(P - ref)) <= 1e-12 * np.max(np.abs(ref))
    if f"{tag}__R" in pins:
        full = pins[f"{tag}__R"]
        assert np.max(np.abs(R - full)) <= 1e-12 * np.max(np.abs(full))


@pytest.mark.skipif(not PRECALC.is_dir(), reason="reference tree not present")
@pytest.mark.parametrize("tag", TAGS)
def test_reader_on_reference_files(tag, pins):
    """Reading the files again reproduces the pins, and the saved objects decode with their classes."""
    from cf_b200.matfile import MatFile, MatObject, load_collision_tensor

    L, g = tag[1:].split("_g")
    path = PRECALC / f"collisiontensor_k4_l{L}_gamma{g}.00.mat"
    c = load_collision_tensor(str(path))
    K_max, L_max, alpha, n_g, n_l = pins[f"{tag}__meta"]
    assert (c.K_max, c.L_max, c.alpha) == (int(K_max), int(L_max), float(g))
    assert c.R.shape == (5, 5, 5, int(n_l)) and c.labels.shape == (int(n_g), 3)
    assert _sha(c.labels) == str(pins[f"{tag}__labels_sha"]) and _sha(c.ic_map) == str(pins[f"{tag}__ic_sha"])
    assert np.array_equal((pins["W"] @ c.R.reshape(125, -1, order="F")).T, pins[f"{tag}__R_proj"])
    mf = MatFile(str(path))
    assert sorted(mf.variables()) == ["Basis", "Kernel", "TensorObj"]
    basis = mf.load("Basis")
    assert isinstance(basis, MatObject) and basis.class_name == "SpectralBasis"
    assert int(basis["N_Q"][0, 0]) == (int(L) + 1) ** 2
    assert isinstance(basis["SH"], MatObject) and basis["SH"].class_name == "SphericalHarmonics"
    t = mf.load("TensorObj")
    assert isinstance(t["Basis"], MatObject) and t["Basis"].class_name == "SpectralBasis"
    assert t["use_mex"].size == 0


def test_contraction_order_matches_restated_sort(pins):
    """The file's arrays go to the operator in the order the reference's callers sort them."""
    from cf_b200 import geometry
    from cf_b200.matfile import CollisionTensorFile

    geo = geometry.generate_geometry(4)
    c = CollisionTensorFile(K_max=4, L_max=4, R=pins["l4_g1__R"], labels=geo.labels, vals=geo.vals,
                            ic_map=geo.ic_map, alpha=1.0)
    lab, vals, ic = c.sorted_for_contraction()
    s = geometry.sort_for_contraction(geo)
    assert np.array_equal(lab, s.labels) and np.array_equal(vals, s.vals) and np.array_equal(ic, s.ic_map)
    assert c.K == 5 and c.N_Q == 25


def test_reader_rejects_other_files(tmp_path):
    from cf_b200.matfile import MatFile, MatFormatError

    p = tmp_path / "v5.mat"
    p.write_bytes(b"MATLAB 5.0 MAT-file, Platform: GLNXA64" + b"\x00" * 200)
    with pytest.raises(MatFormatError):
        MatFile(str(p))
    q = tmp_path / "bad_superblock.mat"
    q.write_bytes(b"\x00" * 512 + b"\x89HDF\r\n\x1a\n" + bytes([2]) + b"\x00" * 100)
    with pytest.raises(MatFormatError):
        MatFile(str(q))
