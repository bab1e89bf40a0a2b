"""The reference arm of bench.py (`--impl reference`) on the host cores: one
JSON line with the contract's keys, timing the reference's own CPU
queryAllPairs (the C restatement when the reference library is not built)
on the headline workload, and nothing from ranks other than 0 when it is
launched as several ranks."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def _run(**env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in KEYS:
        assert key in d, key
    assert d["value"] > 0 and d["unit"] == "entries/s" and d["higher_is_better"] is True
    assert (d["steps"], d["warmup"]) == (1, 3)
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["k"] == 256 and d["config"]["grid"] == 512


def test_reference_arm_other_ranks_stay_silent():
    r = _run(RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
