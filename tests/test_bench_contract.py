"""bench.py's reference arm on the CPU for every Id-Vg workload at a reduced mesh: it runs the
reference core built from its sources (oracle/_ref) and prints one JSON line with the
contract's keys (metric, value, unit, n_gpus, steps, warmup, ms_per_step,
higher_is_better, scaling, vs_baseline, dtype, data, config, impl, cpu_baseline, e2e)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"}


@pytest.mark.parametrize("workload,mesh", [("nmosfet", "16,12,6"), ("finfet", "24,24,16"),
                                           ("graph_mosfet", "16,12,6")])
def test_reference_arm_prints_contract_line(workload, mesh):
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsemisim_ref.so")):
        pytest.skip("reference core not built (make -C oracle)")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", workload,
                          "--mesh", mesh, "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d), KEYS - set(d)
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"].startswith(workload) and d["config"]["nodes"] > 0
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "reference"
