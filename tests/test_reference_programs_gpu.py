"""The engine behind the reference's own harness, and the reference's own CUDA
programs, on the same graph files.

* shim_<alg>_<kind>: the reference's unchanged include/<alg>_<kind>_cuda.h
  (main, ECLgraph reader, timing, serial verifier) linked with this project's
  drop-in GPU<alg>_<kind> bodies; the reference's verifier must pass for every
  variant.
* cuda_*: the reference's CUDA variants compiled for sm_100a; their printed
  summary (max-distance vertex, component count) must match ours.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref not built")]


def _run(exe, args, env=None, timeout=600):
    e = dict(os.environ)
    e.update(env or {})
    p = subprocess.run([str(oracle.REF_OUT / exe), *map(str, args)], capture_output=True, text=True, env=e,
                       timeout=timeout)
    return p.returncode, p.stdout + p.stderr


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("egr")
    out = {}
    for name, g in [("rmat12", i2.gen_rmat(12, 16, seed=21)), ("grid40", i2.gen_grid(40, 0.05, 0.01, 2)),
                    ("er", i2.gen_er(5000, 20000, 9))]:
        p = d / f"{name}.egr"
        oracle.write_egr(g, str(p))
        out[name] = (str(p), g)
    return out


@pytest.mark.parametrize("shim", ["bfs_vertex", "bfs_edge", "sssp_vertex", "sssp_edge", "cc_vertex", "cc_edge"])
def test_reference_harness_verifies_engine(gpu, files, shim):
    for name, (path, g) in files.items():
        src = int(np.argmax(g.degrees()))
        args = [path, 1] if shim.startswith("cc") else [path, src, 1]
        styles = ["heuristic", "vp_thread", "vp_warp", "vp_cta", "vp_block", "pull_frontier", "pull_topo",
                  "edge_topo", "push_topo"] + (["union_find"] if shim.startswith("cc") else [])
        for v in styles:
            rc, out = _run(f"shim_{shim}", args, {"I2_VARIANT": v})
            assert rc == 0 and "verification passed" in out, f"{shim} {name} {v}\n{out[-2000:]}"
        rc, out = _run(f"shim_{shim}", args, {"I2_LOOP": "host"})
        assert rc == 0 and "verification passed" in out, out[-2000:]


@pytest.mark.parametrize("shim", ["mis_vertex", "mis_edge"])
def test_reference_mis_harness_verifies_engine(gpu, files, shim):
    # The MIS harness's verifier (independent, maximal, nothing undecided)
    # exits non-zero with "ERROR" on a failure and prints nothing on success.
    for name, (path, g) in files.items():
        for env in ({}, {"I2_LOOP": "host"}):
            rc, out = _run(f"shim_{shim}", [path, 1], env)
            assert rc == 0 and "ERROR" not in out, f"{shim} {name} {env}\n{out[-2000:]}"


def _summary(out):
    m = re.findall(r"vertex (\d+) has maximum distance (\d+)", out)
    c = re.findall(r"number of connected components: (\d+)", out)
    return (tuple(map(int, m[-1])) if m else None), (int(c[-1]) if c else None)


def test_reference_cuda_programs_agree(gpu, files):
    for name, (path, g) in files.items():
        src = int(np.argmax(g.degrees()))
        dg = i2.DeviceGraph.upload(g)
        d_b = dg.bfs(src)[0]
        d_s = dg.sssp(src)[0]
        lab = dg.cc()[0]
        rc, out = _run("cuda_bfs_vertex_k2", [path, src, 1])
        assert rc == 0 and "verification passed" in out, out[-2000:]
        (mv, md), _ = _summary(out)
        assert d_b[mv] == md and d_b.max() == md
        rc, out = _run("cuda_sssp_edge_s1", [path, src, 1])
        assert rc == 0 and "verification passed" in out, out[-2000:]
        (mv, md), _ = _summary(out)
        assert d_s[mv] == md and d_s.max() == md
        rc, out = _run("cuda_cc_vertex_c1", [path, 1])
        assert rc == 0 and "verification passed" in out, out[-2000:]
        _, ncomp = _summary(out)
        assert ncomp == len(np.unique(lab))
        dg.free()
