"""Learned style selector: training data, training and evaluation.

The engine records, for every iteration of a traversal, how long each relax
style takes from the same frontier state (``i2_sweep``: the state is saved on
the device, each style is launched from it and timed with CUDA events, and the
state is restored). Those timings, keyed by the 16 frontier features the
engine itself computes on the device, train a 16-64-64-8 MLP with the engine's
hand-written CUDA forward/backward/Adam kernels (``i2_mlp_train``). At run time
(``I2_AUTO_LEARNED``) the last block of each relax launch evaluates the MLP and
picks the next iteration's style on the device, without a host round trip.

Every style reaches the same fixed point, so the selector changes time only.

Usage:
    python -m indigo2suite_b200.selector train [--graphs 200] [--max-scale 21] [--out PATH]
        (also writes PATH with the suffix .json: the command, the sweep's and
        the parameters' SHA-256, the row count and the final loss)
    python -m indigo2suite_b200.selector eval [--params PATH] [--json OUT]
"""
from __future__ import annotations

import argparse
import json
import math
import statistics
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import (I2_AUTO_HEURISTIC, I2_AUTO_LEARNED, I2_BFS, I2_CC, I2_NUM_VARIANTS, I2_SSSP, VARIANTS, DeviceGraph,
               gen_er, gen_grid, gen_rmat, mlp_param_count, mlp_set_params, mlp_train)

PARAMS_PATH = Path(__file__).with_name("selector_params.bin")
ALGOS = {"bfs": I2_BFS, "sssp": I2_SSSP, "cc": I2_CC}
F, H, O = 16, 64, I2_NUM_VARIANTS


@dataclass(frozen=True)
class GraphSpec:
    family: str  # rmat | er | grid
    scale: int   # log2 of the vertex count
    seed: int

    @property
    def name(self) -> str:
        return f"{self.family}{self.scale}_s{self.seed}"

    def build(self):
        n = 1 << self.scale
        if self.family == "rmat":
            return gen_rmat(self.scale, 16, 0.57, 0.19, 0.19, seed=self.seed)
        if self.family == "er":
            return gen_er(n, 4 * n, self.seed)  # average degree 8
        side = int(round(math.sqrt(n)))
        return gen_grid(side, 0.05, 0.001, seed=self.seed)


def training_specs(count: int = 200, seed: int = 2024, max_scale: int = 21) -> list[GraphSpec]:
    """`count` seeded graphs, families RMAT/ER/grid in turn, scales 16..max_scale."""
    rng = np.random.default_rng(seed)
    fams = ("rmat", "er", "grid")
    return [GraphSpec(fams[k % 3], 16 + int(rng.integers(0, max_scale - 15)), int(rng.integers(1, 2**31 - 1)))
            for k in range(count)]


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights and zero biases in the engine's blob layout."""
    rng = np.random.default_rng(seed)
    p = np.zeros(mlp_param_count(), np.float32)
    off_w1 = 2 * F
    off_b1 = off_w1 + F * H
    off_w2 = off_b1 + H
    off_b2 = off_w2 + H * H
    off_w3 = off_b2 + H
    p[F:2 * F] = 1.0
    p[off_w1:off_b1] = rng.normal(0, math.sqrt(2.0 / F), F * H)
    p[off_w2:off_b2] = rng.normal(0, math.sqrt(2.0 / H), H * H)
    p[off_w3:off_w3 + H * O] = rng.normal(0, math.sqrt(1.0 / H), H * O)
    return p


def _source(g) -> int:
    return int(np.argmax(np.diff(g.nindex.astype(np.int64))))


def record(specs, algos=("bfs", "sssp", "cc"), follows=(I2_AUTO_HEURISTIC, 2), reps: int = 2, log=print):
    """Per-iteration timings of every style along the trajectories `follows`."""
    X, T, M, meta = [], [], [], []
    for gi, spec in enumerate(specs):
        t0 = time.time()
        g = spec.build()
        dg = DeviceGraph.upload(g)
        src = _source(g)
        rows = 0
        for an in algos:
            for fol in follows:
                recs, times = dg.sweep(ALGOS[an], src, follow=fol, reps=reps, cap=1 << 14)
                times = _union_find_equivalent(recs, times)
                for r, t in zip(recs, times):
                    ok = t > 0
                    if not ok.any():
                        continue
                    X.append(r["feat"])
                    T.append(np.where(ok, np.log2(np.maximum(t, 1.0)), 0.0))
                    M.append(ok.astype(np.float32))
                    meta.append((gi, an, fol, r["iter"]))
                    rows += 1
        dg.free()
        if log:
            log(f"[{gi + 1}/{len(specs)}] {spec.name}: V={g.nodes} E={g.edges} rows={rows} ({time.time() - t0:.1f}s)")
    return (np.asarray(X, np.float32), np.asarray(T, np.float32), np.asarray(M, np.float32), meta)


UF = VARIANTS.index("union_find")


def _union_find_equivalent(recs, times):
    """(Union-find is chosen before the first iteration by a rule shared with
    the heuristic, so the selector reads this column only as training data.)
    Union-find finishes the whole traversal in one choice, so its time is
    not comparable with one iteration of another style. Along the followed
    trajectory (per-iteration times f_k, remaining time R_k after iteration
    k), its time at iteration k is scaled to the share of the remaining work
    that one iteration represents: t_uf * f_k / (f_k + R_k). The selector then
    prefers it exactly when t_uf < f_k + R_k, i.e. when it beats finishing
    along the trajectory."""
    times = np.array(times, np.float64, copy=True)
    if len(recs) == 0:
        return times
    f = np.array([times[k, r["variant"]] if times[k, r["variant"]] > 0 else 0.0 for k, r in enumerate(recs)])
    rest = np.concatenate([np.cumsum(f[::-1])[::-1][1:], [0.0]])
    for k in range(len(recs)):
        if times[k, UF] > 0 and f[k] > 0:
            times[k, UF] *= f[k] / (f[k] + rest[k])
    return times


def train(X, T, M, epochs: int = 200, batch: int = 512, lr: float = 2e-3, seed: int = 1):
    """Train on the device with the engine's kernels; returns (params, final loss)."""
    return mlp_train(init_params(seed), X, T, M, epochs=epochs, batch=batch, lr=lr, seed=seed)


def _time_runs(dg, algo, src, variant, runs: int = 3) -> float:
    dg.run_device(algo, src, variant=variant)
    ts = [dg.run_device(algo, src, variant=variant).seconds for _ in range(runs)]
    return statistics.median(ts)


def evaluate(params, specs, algos=("bfs", "sssp", "cc"), log=print) -> list[dict]:
    """For each graph and algorithm: traversal time of every fixed style, the
    heuristic and the learned selector (CUDA-graph runs), and, along the learned
    trajectory, the per-iteration oracle (best measured style per iteration)."""
    mlp_set_params(params)
    out = []
    for spec in specs:
        g = spec.build() if isinstance(spec, GraphSpec) else spec[1]
        name = spec.name if isinstance(spec, GraphSpec) else spec[0]
        dg = DeviceGraph.upload(g)
        src = _source(g)
        sym = dg.info["symmetric"] == 1
        for an in algos:
            algo = ALGOS[an]
            fixed = {}
            for v in range(I2_NUM_VARIANTS):
                if v in (4, 5, 8) and not sym:
                    continue
                if v == 8 and an != "cc":  # union-find computes CC labels only
                    continue
                fixed[VARIANTS[v]] = _time_runs(dg, algo, src, v)
            heur = _time_runs(dg, algo, src, I2_AUTO_HEURISTIC)
            learned = _time_runs(dg, algo, src, I2_AUTO_LEARNED)
            recs, times = dg.sweep(algo, src, follow=I2_AUTO_LEARNED, reps=2, cap=1 << 14)
            chosen = np.array([r["variant"] for r in recs], int)
            t_ok = np.where(times > 0, times, np.inf)
            oracle_ns = float(t_ok.min(axis=1).sum())
            learned_ns = float(t_ok[np.arange(len(recs)), chosen].sum())
            best = min(fixed, key=fixed.get)
            row = {"graph": name, "algo": an, "V": g.nodes, "E": g.edges, "fixed_s": fixed, "best_fixed": best,
                   "best_fixed_s": fixed[best], "heuristic_s": heur, "learned_s": learned,
                   "speedup_vs_best_fixed": fixed[best] / learned, "speedup_heuristic": fixed[best] / heur,
                   "per_iteration_oracle_ns": oracle_ns, "learned_sweep_ns": learned_ns,
                   "regret_vs_oracle": learned_ns / oracle_ns - 1.0, "iterations": len(recs),
                   "choices": {VARIANTS[k]: int((chosen == k).sum()) for k in range(I2_NUM_VARIANTS)
                               if (chosen == k).any()}}
            out.append(row)
            if log:
                log(f"{name} {an}: best fixed {best} {1e3 * fixed[best]:.3f} ms, heuristic {1e3 * heur:.3f} ms, "
                    f"learned {1e3 * learned:.3f} ms (x{row['speedup_vs_best_fixed']:.2f}), "
                    f"regret vs per-iteration oracle {100 * row['regret_vs_oracle']:.1f}%")
        dg.free()
    return out


def summary(rows: list[dict]) -> dict:
    gm = lambda xs: float(math.exp(np.mean(np.log(xs))))  # noqa: E731
    return {"cases": len(rows),
            "geomean_speedup_learned_vs_best_fixed": gm([r["speedup_vs_best_fixed"] for r in rows]),
            "geomean_speedup_heuristic_vs_best_fixed": gm([r["speedup_heuristic"] for r in rows]),
            "geomean_learned_over_oracle": gm([1 + r["regret_vs_oracle"] for r in rows]),
            "max_regret_vs_oracle": max(r["regret_vs_oracle"] for r in rows)}


def eval_specs() -> list[GraphSpec]:
    """Held-out graphs (seeds disjoint from training_specs' draws)."""
    return [GraphSpec(f, s, 7000 + k) for k, (f, s) in enumerate(
        [("rmat", 18), ("rmat", 20), ("er", 18), ("er", 20), ("grid", 18), ("grid", 20)])]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "eval"])
    ap.add_argument("--graphs", type=int, default=200)
    ap.add_argument("--max-scale", type=int, default=21)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--out", default=str(PARAMS_PATH))
    ap.add_argument("--params", default=str(PARAMS_PATH))
    ap.add_argument("--json", default=None)
    ap.add_argument("--data", default=None, help="npz of recorded rows to reuse / write")
    a = ap.parse_args(argv)
    if a.cmd == "train":
        if a.data and Path(a.data).exists():
            z = np.load(a.data)
            X, T, M = z["X"], z["T"], z["M"]
        else:
            X, T, M, _ = record(training_specs(a.graphs, max_scale=a.max_scale))
            if a.data:
                np.savez_compressed(a.data, X=X, T=T, M=M)
        p, loss = train(X, T, M, epochs=a.epochs)
        p.astype(np.float32).tofile(a.out)
        import hashlib

        digest = hashlib.sha256(X.tobytes() + T.tobytes() + M.tobytes()).hexdigest()
        meta = {"command": f"python -m indigo2suite_b200.selector train --graphs {a.graphs} "
                           f"--max-scale {a.max_scale} --epochs {a.epochs}",
                "rows": int(X.shape[0]), "final_loss": loss, "sweep_sha256": digest,
                "params_sha256": hashlib.sha256(p.astype(np.float32).tobytes()).hexdigest(), "out": a.out}
        Path(a.out).with_suffix(".json").write_text(json.dumps(meta, indent=1) + "\n")
        print(json.dumps(meta))
    else:
        p = np.fromfile(a.params, np.float32)
        rows = evaluate(p, eval_specs())
        res = {"summary": summary(rows), "rows": rows}
        print(json.dumps(res["summary"]))
        if a.json:
            Path(a.json).write_text(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
