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


# Runs bench.py's main() in this interpreter, then reports on stderr whether
# the engine package or its library was ever loaded into the process.
_PROBE = """
import runpy, sys
sys.argv = ["bench.py"] + sys.argv[1:]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
sys.stderr.write("ENGINE_LOADED=%d\\n" % ("libi2b200" in maps or "indigo2suite_b200" in sys.modules))
"""


def _bench(env_extra, *args):
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run([sys.executable, "-c", _PROBE, "--impl", "reference", *args],
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
    # the reference arm runs no engine code, not even to build its input
    assert "ENGINE_LOADED=0" in r.stderr
    # and reports the config the GPU arm reports for the same graph
    import argparse

    import indigo2suite_b200 as i2

    sys.path.insert(0, str(ROOT))
    import bench

    g = i2.gen_rmat(22, 16, 0.57, 0.19, 0.19, seed=22)
    args = argparse.Namespace(variant="vp_cta", loop="graph", delta=0, budget=-1)
    assert d["config"] == bench.bench_config(args, g, 1)
