"""Autotuners, measured on the device and written as committed tables.

1. The batched traversal: style, resident blocks per SM and heavy threshold
   for BFS + SSSP over a batch of graphs (`tuning_table.json`, applied by
   `bench.py --workload batch512` and any caller of `Batch.tune`).
2. Single traversals, keyed by the graph's shape (`traversal_table.json`):
   per degree class (from `i2_graph_info`: skewed when the degree's coefficient
   of variation is 1 or more, else sparse when the average degree is below 6,
   else uniform), per size class (log2 of the vertex count) and algorithm, the
   resident blocks per SM and, for SSSP, the near/far edge budget (the size of
   each near set: the traversal's chunk of work per iteration). `apply(dg,
   algo)` looks a graph up and tunes it; unknown shapes keep the defaults.

The tuning batch is drawn like the benchmark's 512-graph batch (log-uniform
vertex counts in [1e3, 1e6], ER / RMAT / grid families) but from another seed,
so the table is not fitted to the graphs it is later measured on. For every
candidate the batch runs BFS and SSSP from each graph's highest-degree vertex
(CUDA-graph traversals, device time by CUDA events, median of `reps`), results
are checked against the untuned run, and the candidate with the smallest
BFS + SSSP time is chosen.

Usage:
    python -m indigo2suite_b200.autotune [--graphs 128] [--out PATH]
    python -m indigo2suite_b200.autotune --traversals [--out PATH]
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


# ---------------------------------------------------------------------------
# Single traversals keyed by shape.

TRAVERSAL_TABLE = Path(__file__).with_name("traversal_table.json")
TUNE_BLOCKS = (2, 4, 8)  # 8: the engine's default cap (the kernels' occupancy allows 6)
TUNE_BUDGETS = (0, 1 << 20, 1 << 21, 1 << 22, 1 << 23)  # SSSP near/far edge budget (0: off)
TUNE_GRAPHS = [(fam, scale) for fam in ("rmat", "er", "grid") for scale in (18, 20, 22)]


def degree_class(info: dict) -> str:
    if info["degcv"] >= 1.0:
        return "skewed"
    return "sparse" if info["avgdeg"] < 6.0 else "uniform"


def size_class(nodes: int) -> int:
    """log2 of the vertex count, rounded to even (18, 20, 22, ...)."""
    import math

    b = int(round(math.log2(max(2, nodes))))
    return b + (b & 1)


def traversal_candidates(algo: str):
    for bps in TUNE_BLOCKS:
        for budget in (TUNE_BUDGETS if algo == "sssp" else (0,)):
            yield bps, budget


def _graph(fam: str, scale: int, seed: int):
    from . import DeviceGraph

    n = 1 << scale
    if fam == "rmat":
        return DeviceGraph.generate_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
    if fam == "er":
        return DeviceGraph.generate_er(n, 4 * n, seed)
    return DeviceGraph.generate_grid(int(round(n ** 0.5)), 0.05, 0.001, seed=seed)


def tune_traversals(seed: int = 17, reps: int = 5, log=print) -> dict:
    """For each tuning graph (RMAT / ER / grid of 2^18, 2^20, 2^22 vertices,
    seeds disjoint from the benchmark's) and algorithm: every candidate's
    device time (median of `reps` resident traversals, results checked against
    the default), the fastest chosen; the default (the engine's cap of 8
    blocks per SM, no budget) is reported beside it."""
    import torch

    from . import I2_CC, VARIANTS

    algos = {"bfs": (I2_BFS, "heuristic"), "sssp": (I2_SSSP, "vp_cta"), "cc": (I2_CC, "heuristic")}
    rows = []
    stream = torch.cuda.Stream()
    for k, (fam, scale) in enumerate(TUNE_GRAPHS):
        dg = _graph(fam, scale, seed + k)
        info = dg.info
        src = dg.hub()
        for an, (algo, style) in algos.items():
            ref = dg._run(algo, src, style, 0, 0, False, None)[0]
            res = []
            for bps, budget in traversal_candidates(an):
                dg.tune(blocks_per_sm=bps)
                got = dg._run(algo, src, style, 0, 0, False, None, budget=budget)[0]
                if not np.array_equal(got, ref):
                    raise RuntimeError(f"{fam}{scale} {an} bps={bps} budget={budget}: result differs")
                ts = []
                for _ in range(reps + 1):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    dg.run_device(algo, src, variant=style, stream=stream.cuda_stream, report=False, budget=budget)
                    e1.record(stream)
                    e1.synchronize()
                    ts.append(e0.elapsed_time(e1))
                res.append({"blocks_per_sm": bps, "budget": budget, "ms": statistics.median(ts[1:])})
            dg.tune(blocks_per_sm=8)
            best = min(res, key=lambda r: r["ms"])
            default = next(r for r in res if r["blocks_per_sm"] == 8 and r["budget"] == 0)
            row = {"graph": f"{fam}{scale}", "class": degree_class(info), "log2v": size_class(info["nodes"]),
                   "algo": an, "style": style, "blocks_per_sm": best["blocks_per_sm"], "budget": best["budget"],
                   "ms": best["ms"], "default_ms": default["ms"], "candidates": res}
            rows.append(row)
            if log:
                log(json.dumps({k: row[k] for k in row if k != "candidates"}))
        dg.free()
    return {"workload": "RMAT / ER / grid of 2^18, 2^20, 2^22 vertices; BFS and CC with the heuristic "
                        "selector, SSSP with the edge-balanced push",
            "default": {"blocks_per_sm": 8, "budget": 0}, "rows": rows, "measured": time.strftime("%Y-%m-%d")}


def lookup(info: dict, algo: str, path: Path | str = TRAVERSAL_TABLE) -> dict | None:
    """The table's choice for a graph of this shape, or None."""
    p = Path(path)
    if not p.exists():
        return None
    cls, sz = degree_class(info), size_class(info["nodes"])
    rows = [r for r in json.loads(p.read_text())["rows"] if r["class"] == cls and r["algo"] == algo]
    if not rows:
        return None
    r = min(rows, key=lambda r: abs(r["log2v"] - sz))  # nearest size class of the same shape
    return {"blocks_per_sm": r["blocks_per_sm"], "budget": r["budget"], "row": r["graph"]}


def apply(dg, algo: str, path: Path | str = TRAVERSAL_TABLE) -> dict:
    """Tune a DeviceGraph for `algo` from the table; returns the options to pass
    to its traversal ({"budget": ...} for SSSP), empty when the shape is unknown."""
    t = lookup(dg.info, algo, path)
    if t is None:
        return {}
    dg.tune(blocks_per_sm=t["blocks_per_sm"])
    return {"budget": t["budget"]} if algo == "sssp" else {}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--graphs", type=int, default=128)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--out", default=None)
    ap.add_argument("--traversals", action="store_true", help="tune single traversals by shape")
    a = ap.parse_args(argv)
    if a.traversals:
        table = tune_traversals(reps=max(3, a.reps))
        Path(a.out or TRAVERSAL_TABLE).write_text(json.dumps(table, indent=1) + "\n")
        return
    table = tune(a.graphs, reps=a.reps)
    Path(a.out or TABLE_PATH).write_text(json.dumps(table, indent=1) + "\n")
    print(json.dumps(table["chosen"]))


if __name__ == "__main__":
    main()
