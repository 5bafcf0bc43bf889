import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "golden.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine's kernels")
    lib = ROOT / "indigo2suite_b200" / "libi2b200.so"
    if not lib.exists():
        import __graft_entry__

        __graft_entry__.build()


def has_gpu() -> bool:
    import indigo2suite_b200 as i2

    return i2.device_count() > 0


@pytest.fixture(scope="session")
def golden():
    z = np.load(GOLDEN)
    import indigo2suite_b200 as i2

    cases = {}
    for name in z["cases"]:
        name = str(name)
        ni = z[f"{name}/nindex"]
        nl = z[f"{name}/nlist"]
        w = z[f"{name}/eweight"]
        g = i2.ECLGraph(len(ni) - 1, len(nl), ni.astype(np.int32), nl.astype(np.int32), w.astype(np.int32))
        srcs = [int(s) for s in z[f"{name}/sources"]]
        cases[name] = {
            "graph": g,
            "sources": srcs,
            "bfs": {s: z[f"{name}/bfs/{s}"] for s in srcs},
            "sssp": {s: z[f"{name}/sssp/{s}"] for s in srcs},
            "cc": z[f"{name}/cc"],
        }
    return cases


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("no CUDA device: -m gpu tests need a B200")
    return True
