"""bench.py's reference arm on CPU: the JSON line contract and the rank behaviour under torchrun."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    res = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                         cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    return [l for l in res.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    lines = _run({})
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "homogenizations/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "n=64" in d["config"]["workload"] and "oracle fixture n64/a0.5/e1e-06/s0" in d["config"]["extrapolation"]
    # the oracle's own certified count, not a device count
    fixture = json.loads((ROOT / "tests" / "golden" / "config2.json").read_text())["cases"]["n64/a0.5/e1e-06/s0"]
    assert f"{max(fixture['iterations'])} iterations" in d["config"]["extrapolation"]
    # one complete, unextrapolated n=16 homogenization with serial loads per step
    c1 = d["config1_complete"]
    assert len(c1["seconds"]) == 1 and c1["seconds"][0] > 0 and len(c1["iterations"][0]) == 6


def test_reference_arm_runs_on_rank_zero_only():
    assert _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}) == []
