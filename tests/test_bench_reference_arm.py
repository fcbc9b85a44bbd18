"""bench.py's reference arm on the CPU: its JSON line keeps the bench
contract (the reference program's own CPU path, timed on the host cores,
on the single-large workload), and under torchrun only rank 0 works and
prints."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(REPO, "oracle", "_ref", "mgkde_ref")
CMD = [sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3", "--scale", "0.1"]
KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def run(env=None):
    return subprocess.run(CMD, cwd=REPO, env=env, capture_output=True, text=True, timeout=900)


@pytest.mark.skipif(not os.path.exists(REF), reason="the reference program is not built here")
def test_reference_arm_json_line():
    p = run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in KEYS:
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["unit"] == d["unit"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "halo points" in cb["sample"]


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    p = run(env)
    assert p.returncode == 0, p.stderr[-2000:]
    assert not p.stdout.strip()
