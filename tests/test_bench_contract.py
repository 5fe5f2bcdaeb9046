"""bench.py's output contract: one JSON line with the keys the round-end tooling reads."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _run(args, timeout=600):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line(reference_lib):
    """The reference arm: the reference's own kernel on the host cores, on the GPU arm's metric."""
    out = _run(["--impl", "reference", "--workload", "hs_l8_k8_b2048", "--steps", "2", "--warmup", "1"])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in out, key
    assert out["impl"] == "reference" and out["value"] > 0 and out["higher_is_better"] is True
    assert out["cpu_baseline"]["kind"] == "reference" and out["cpu_baseline"]["cores"] >= 1
    assert out["e2e"] == {"value": out["value"], "unit": out["unit"], "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
    assert out["config"]["workload"] == "hs_l8_k8_b2048"


def test_reference_arm_without_counterpart():
    out = _run(["--impl", "reference", "--workload", "implicit_hs_l8_k8_b2048"])
    assert out["impl"] == "reference" and "unavailable" in out


@pytest.mark.gpu
def test_gpu_arm_line(cuda_available):
    """The GPU arm on its default workload: every key of the contract, a live roofline and clocks."""
    out = _run(["--steps", "3", "--warmup", "3", "--no-cpu-baseline"])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e", "gpu_launches", "clocks"):
        assert key in out, key
    assert out["n_gpus"] == 1 and out["steps"] == 3 and out["warmup"] >= 3 and out["value"] > 0
    roof = out["roofline"]
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in roof, key
    assert 0 < roof["frac"] < 1.5
    e2e = out["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert out["gpu_launches"] > 0
    assert "sm_mhz" in out["clocks"] and "reasons" in out["clocks"]
    assert out["config"]["workload"] == "hs_l10_k8_b4096"
