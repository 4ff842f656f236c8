"""bench.py's output contract: one JSON line with the keys the harness reads,
the reference arm on the CPU (DUCC's own NUFFT from oracle/_ref), and our arm
on a small workload on the GPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line():
    from oracle import ref
    if ref.load() is None:
        pytest.skip("DUCC's CPU NUFFT is not built (oracle/_ref)")
    d = run_bench("--impl", "reference", "--m", "20000", "--n", "64", "--steps", "2",
                  "--warmup", "1", "--param-threads", "2")
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "config", "cpu_baseline", "e2e", "ducc_choice"):
        assert k in d, k
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["grid"] == [64, 64] and d["config"]["npoints"] == 20000
    assert d["config"]["param_threads"] == 2
    assert d["value"] > 0


@pytest.mark.gpu
def test_our_arm_line_small():
    d = run_bench("--m", "400000", "--n", "256", "--steps", "3", "--warmup", "3",
                  "--no-extra", "--no-cpu", "--param-threads", "2")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "roofline", "kernels", "clocks", "gpu_launches", "e2e", "errors"):
        assert k in d, k
    assert d["config"]["param_threads"] == 2
    assert d["gpu_launches"] > 0
    for k in ("bound", "achieved", "peak", "unit", "frac"):
        assert k in d["roofline"], k
    assert d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    assert d["e2e_concurrent"]["value"] > 0
    if d["errors"] is not None:
        assert d["errors"]["type1"]["tc"] < 1e-6 and d["errors"]["type1"]["plain"] < 1e-6
    assert "alt_plain" in d and "alt_plain_matched" in d
