"""Autotuner of the batched traversal: style, resident blocks per SM and heavy
threshold for BFS + SSSP over a batch of graphs, measured on the device and
written as a table that `bench.py --workload batch512` (and any caller of
`Batch.tune`) applies.

The tuning batch is drawn like the benchmark's 512-graph batch (log-uniform
vertex counts in [1e3, 1e6], ER / RMAT / grid families) but from another seed,
so the table is not fitted to the graphs it is later measured on. For every
candidate the batch runs BFS and SSSP from each graph's highest-degree vertex
(CUDA-graph traversals, device time by CUDA events, median of `reps`), results
are checked against the untuned run, and the candidate with the smallest
BFS + SSSP time is chosen.

Usage:
    python -m indigo2suite_b200.autotune [--graphs 128] [--out PATH]
"""
from __future__ import annotations

import argparse
import itertools
import json
import statistics
import time
from pathlib import Path

import numpy as np

from . import I2_BFS, I2_SSSP, Batch
from . import workloads

TABLE_PATH = Path(__file__).with_name("tuning_table.json")
STYLES = ("vp_cta", "vp_thread", "vp_warp", "heuristic")
BLOCKS_PER_SM = (2, 4, 6, 8)
HEAVY = (1024, 4096, 16384)


def candidates():
    """(style, blocks per SM, heavy threshold); the heavy threshold only
    matters to the vertex-granular push styles."""
    for style, bps in itertools.product(STYLES, BLOCKS_PER_SM):
        for heavy in (HEAVY if style in ("vp_thread", "vp_warp") else (4096,)):
            yield style, bps, heavy


def _time(b, algo, srcs, style, reps):
    import torch

    stream = torch.cuda.Stream()
    ts = []
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run_device(algo, srcs, variant=style, stream=stream.cuda_stream, report=False)
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts[1:])


def tune(graphs: int = 128, seed: int = 11, reps: int = 3, log=print) -> dict:
    specs = workloads.batch_specs(graphs, seed=seed)
    gs = [workloads.build(s) for s in specs]
    srcs = [workloads.source(g) for g in gs]
    b = Batch(gs)
    ref = {}
    for algo in (I2_BFS, I2_SSSP):
        b.run_device(algo, srcs, variant="vp_cta")
        ref[algo] = np.concatenate(b.result())
    rows = []
    for style, bps, heavy in candidates():
        b.tune(heavy_threshold=heavy, blocks_per_sm=bps)
        ms = {}
        for name, algo in (("bfs", I2_BFS), ("sssp", I2_SSSP)):
            ms[name] = _time(b, algo, srcs, style, reps)
            if not np.array_equal(np.concatenate(b.result()), ref[algo]):
                raise RuntimeError(f"{style} bps={bps} heavy={heavy}: {name} result differs")
        row = {"style": style, "blocks_per_sm": bps, "heavy_threshold": heavy, "bfs_ms": ms["bfs"],
               "sssp_ms": ms["sssp"], "total_ms": ms["bfs"] + ms["sssp"]}
        rows.append(row)
        if log:
            log(json.dumps(row))
    b.free()
    best = min(rows, key=lambda r: r["total_ms"])
    return {"workload": f"{graphs} graphs drawn like the 512-graph batch (seed {seed}), BFS + SSSP",
            "chosen": {k: best[k] for k in ("style", "blocks_per_sm", "heavy_threshold")},
            "chosen_total_ms": best["total_ms"], "candidates": rows,
            "measured": time.strftime("%Y-%m-%d")}


def load(path: Path | str = TABLE_PATH) -> dict | None:
    p = Path(path)
    return json.loads(p.read_text())["chosen"] if p.exists() else None


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--graphs", type=int, default=128)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=str(TABLE_PATH))
    a = ap.parse_args(argv)
    table = tune(a.graphs, reps=a.reps)
    Path(a.out).write_text(json.dumps(table, indent=1) + "\n")
    print(json.dumps(table["chosen"]))


if __name__ == "__main__":
    main()
