"""The benchmark's reference arm on the host (no GPU): rank 0 prints one JSON
line with the contract's keys, every other rank exits quietly."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

import oracle

ROOT = Path(__file__).resolve().parents[1]


def _bench(env_extra, *args):
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", *args],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"}, "--gpus", "2", "--steps", "1", "--warmup", "3")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


@pytest.mark.skipif(not (oracle.REF_OUT / "libref_cpu_sssp_vertex_cpp.so").exists(),
                    reason="reference CPU programs not built")
def test_reference_arm_line():
    r = _bench({"RANK": "0", "LOCAL_RANK": "0", "WORLD_SIZE": "1"}, "--steps", "1", "--warmup", "3")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GTEPS" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 3 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "sssp_rmat22_ef16_edge_data_push"
