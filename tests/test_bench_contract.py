"""bench.py's JSON contract, checked on the CPU through the reference arm
(the oracle on the host cores; the GPU arm needs a device)."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "small",
                        "--steps", "1", "--warmup", "1"], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=600)
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    return p.returncode, lines


def test_reference_arm_line():
    rc, lines = _run({})
    assert rc == 0
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "unit", "ms_per_step", "scaling", "dtype", "data"):
        assert d[k]
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 1
    assert d["higher_is_better"] is True and "vs_baseline" in d
    assert isinstance(d["config"], dict) and d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"] and cb["cores"] >= 1
    assert cb["kind"] in ("reference", "port") and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_print_nothing():
    rc, lines = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert rc == 0
    assert lines == []
