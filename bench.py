#!/usr/bin/env python
"""Benchmark of the Indigo2 SSSP/BFS/CC relaxation path on B200.

Workload (one GPU): SSSP on an RMAT graph of scale 22 (4,194,304 vertices,
edge factor 16, a=0.57 b=0.19 c=0.19 d=0.05, seed 22), symmetrised,
deduplicated, no self-loops, int32 weights uniform in [1,255] (one per
undirected edge), source = highest-degree vertex (lowest ID on ties); fixed
style: edge-centric data-driven push (the engine's vp_cta: one thread per
frontier edge), with the budgeted near/far ordering (each iteration relaxes
the frontier vertices below a distance threshold that keeps about 4.2M edges
below it; --budget 0 turns it off). A step is one complete SSSP traversal
(init + all iterations) with the graph resident in HBM; nlist + eweight (1 GB)
exceed L2, so every step streams them from HBM.

value   : GTEPS, reference definition (1e-9 * g.edges / seconds per traversal,
          include/bfs_vertex_cuda.h:163), summed over all ranks.
e2e     : the same metric through the public C ABI from pinned host buffers:
          i2_graph_upload (H2D of nindex/nlist/eweight) + i2_sssp (D2H of dist)
          + i2_graph_free, per step.
roofline: the relax kernel, from algorithmic bytes B_alg = 12*E_r + 20*V_r
          (E_r = sum of degrees of reached vertices, V_r = reached vertices)
          over the sum of its launch durations (CUDA events on its stream).
Multi-GPU (torchrun): independent replicas, one per rank ("replicas only":
a single traversal does not shard); timing is the max over ranks.

--impl reference: the reference's own CPU SSSP (codes/cpp/sssp-cpp
V_Data_Push ... NonDup, its fastest CPU SSSP; built unchanged into oracle/_ref)
on the same graph with all host threads, one traversal per step, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GTEPS & HBM GB/s: learned-style vs best fixed style, BFS/SSSP/CC bit-exact"
UNIT = "GTEPS"
# kernel that runs each style's iterations
KERNEL_NAMES = {"vp_thread": "relax_push", "vp_warp": "relax_push", "vp_cta": "relax_edge_balanced",
                "vp_block": "relax_push", "pull_frontier": "relax_pull", "pull_topo": "relax_pull",
                "edge_topo": "relax_edge_topo", "push_topo": "relax_push_topo"}
WORKLOAD = {"workload": "sssp_rmat22_ef16_edge_data_push", "graph": "rmat", "scale": 22, "edge_factor": 16,
            "a": 0.57, "b": 0.19, "c": 0.19, "seed": 22, "weights": "uniform[1,255]",
            "source": "highest-degree vertex", "algorithm": "sssp",
            "style": "vp_cta (edge-centric data-driven push; vertices relaxed in distance order by the budgeted "
                     "near/far ordering unless near_far_budget is off)",
            "l2": "inputs larger than L2 (nlist+eweight 1.0 GB)"}
SELECTOR_PARAMS = ROOT / "indigo2suite_b200" / "selector_params.bin"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    def __init__(self, world: int, backend: str):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch.distributed as td

            td.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
            self.td = td

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def max(self, x: float, device) -> float:
        if self.world == 1:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=device)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


class Clocks:
    """nvidia-smi samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # wait for its first sample: its start-up queries the device, which
            # would land inside a short timed region
            t0 = time.time()
            while time.time() - t0 < 3.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


_PINNED = []


def pinned_copy(a: np.ndarray) -> np.ndarray:
    import torch

    t = torch.empty(a.size, dtype=torch.int32, pin_memory=True)
    _PINNED.append(t)  # keeps the page-locked buffer alive for the numpy view
    out = t.numpy()
    out[:] = a
    return out


def graph_source(g) -> int:
    return int(np.argmax(g.degrees()))  # first maximum: lowest ID on ties


def ref_cpu_baseline(g, src: int, runs: int, name: str) -> dict:
    import oracle

    threads = os.cpu_count() or 1
    ts = []
    for _ in range(runs):
        t, _ = oracle.ref_cpu_run(name, g, src, threads)
        ts.append(t)
    med = statistics.median(ts)
    return {"value": 1e-9 * g.edges / med, "unit": UNIT, "cores": threads, "kind": "reference",
            "program": name, "sample": f"full workload graph, {runs} traversals, median of the reference's own timer"}


def ref_cuda_baseline(g, src: int) -> dict:
    """The reference's own CUDA SSSP in the benchmark's style (E_Data_Push, S1:
    codes/cuda/sssp-cuda/SSSP_CUDA_E_Data_Push_..._NonDup.cu, built unchanged for
    sm_100a in oracle/_ref) on the same graph file, timed by its own main."""
    import tempfile

    import oracle

    if not (oracle.REF_OUT / "cuda_sssp_edge_s1").exists():
        return {"unavailable": "oracle/_ref/cuda_sssp_edge_s1 not built"}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "g.egr")
        oracle.write_egr(g, path)
        r = oracle.run_ref_program("cuda_sssp_edge_s1", [path, str(src), "0"], timeout=900)
    if r["rc"] != 0 or not r["runtime"]:
        return {"unavailable": f"S1 exited {r['rc']}: {r['out'][-200:]}"}
    return {"program": "cuda_sssp_edge_s1 (reference S1, E_Data_Push, sm_100a)", "runtime_s": r["runtime"],
            "value": 1e-9 * g.edges / r["runtime"], "unit": UNIT,
            "sample": "full workload graph; the program's own runtime print (device loop, verification off)"}


def graph_digest(g) -> str:
    """First 16 hex digits of SHA-256 over nindex, nlist and eweight: both arms
    put it in `config`, so equal configs mean the same graph."""
    import hashlib

    h = hashlib.sha256()
    for a in (g.nindex, g.nlist, g.eweight):
        h.update(np.ascontiguousarray(a, np.int32)[: len(a)].tobytes())
    return h.hexdigest()[:16]


def bench_config(args, g, world: int) -> dict:
    """The benchmark line's `config`, identical in both arms."""
    return dict(WORKLOAD, variant=args.variant, edges=g.edges, nodes=g.nodes, graph_sha16=graph_digest(g),
                parallelism=f"replicas x{world}", loop=args.loop,
                near_far_step=args.delta if args.delta > 0 else "off",
                near_far_budget=("off" if args.delta > 0 or args.budget == 0 else
                                 "auto (28672 edges per SM)" if args.budget < 0 else args.budget))


def run_reference(args, rank: int, world: int):
    """The reference's own CPU SSSP on the benchmark graph. The graph comes from
    the oracle's independent C generator (oracle/graphgen.c, the same CSR as the
    engine's generators), so this arm loads no engine code."""
    if rank != 0:
        return
    import oracle

    if not (oracle.REF_OUT / "libref_cpu_sssp_vertex_cpp.so").exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference CPU programs)"}))
        return
    g = oracle.gen_rmat(22, 16, 0.57, 0.19, 0.19, seed=22)
    src = graph_source(g)
    threads = os.cpu_count() or 1
    prog = "sssp_vertex_cpp"
    for _ in range(args.warmup):
        oracle.ref_cpu_run(prog, g, src, threads)
    ts = []
    for _ in range(args.steps):
        t, _ = oracle.ref_cpu_run(prog, g, src, threads)
        ts.append(t)
    total = sum(ts)
    value = 1e-9 * g.edges * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic", "config": bench_config(args, g, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "program": prog + " (codes/cpp/sssp-cpp/SSSP_CPP_V_Data_Push_..._NonDup.cpp, "
                                               "built unchanged)",
                             "sample": "full workload graph, one traversal per step, the program's own timer"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local: int):
    import torch

    import indigo2suite_b200 as i2

    torch.cuda.set_device(local)
    dist = Dist(world, "nccl")
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream

    dg = i2.DeviceGraph.generate_rmat(22, 16, 0.57, 0.19, 0.19, seed=22)
    host = dg.download()
    E, V = host.edges, host.nodes
    src = graph_source(host)
    variant = args.variant

    # correctness of the measured configuration (shortest-path certificate)
    delta = args.delta
    budget = -1 if args.budget < 0 else args.budget  # I2_SSSP_BUDGET_AUTO when negative
    d, rep = dg.sssp(src, variant=variant, delta=delta, budget=budget)
    import oracle

    cert = oracle.certify_distances(host, src, d, weighted=True)
    if cert is not None:
        raise SystemExit(f"result certificate failed: {cert}")

    loop = {"graph": i2.I2_LOOP_GRAPH, "host": i2.I2_LOOP_HOST, "relaunch": i2.I2_LOOP_RELAUNCH}[args.loop]

    def steps(n, v=variant, b=None):
        for _ in range(n):
            dg.run_device(i2.I2_SSSP, src, variant=v, stream=sp, loop=loop, report=loop == i2.I2_LOOP_HOST,
                          delta=delta, budget=budget if b is None else b)

    with torch.cuda.stream(stream):
        steps(args.warmup)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()  # (settles for a moment: starting nvidia-smi queries the device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    steps(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    ms_max = dist.max(ms, dev)
    value = world * 1e-9 * E / (ms_max * 1e-3)

    # Dominant kernel. With the graph loop one resident launch runs every
    # iteration of a step, so its duration is the step's (CUDA events on the
    # launching stream, over the timed region; the reset/fill/seed launches
    # before it are < 2% of the step and are charged to it). The host-driven
    # loop's per-iteration launches, each bracketed by CUDA events, are
    # reported beside it.
    rep_h = dg.run_device(i2.I2_SSSP, src, variant=variant, loop=i2.I2_LOOP_HOST, stream=sp, delta=delta,
                          budget=budget)
    rep_g = dg.run_device(i2.I2_SSSP, src, variant=variant, stream=sp, delta=delta, budget=budget)
    b_alg = 12.0 * rep_g.reached_edges + 20.0 * rep_g.reached_vertices
    graph_loop = loop == i2.I2_LOOP_GRAPH
    kernel_s = ms_max * 1e-3 if graph_loop else rep_h.relax_seconds
    achieved = b_alg / kernel_s / 1e9
    peak, peak_kind = peaks()
    kname = KERNEL_NAMES.get(variant, str(variant))
    if variant == "vp_cta" and (delta > 0 or budget != 0):
        kname = "relax_near_far"  # the edge-balanced push with the near/far ordering
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "peak_source": peak_kind,
                "kernel": (f"relax_resident<SSSP,{variant}>" if graph_loop else kname + "<SSSP>"),
                "launches_per_step": 1 if graph_loop else rep_h.iterations, "iterations": rep_g.iterations,
                "b_alg_bytes_per_step": b_alg, "kernel_ms_per_step": 1e3 * kernel_s,
                "host_loop": {"kernel": kname + "<SSSP>", "launches": rep_h.iterations,
                              "relax_ms_events": 1e3 * rep_h.relax_seconds,
                              "achieved_gbs": b_alg / rep_h.relax_seconds / 1e9}}
    prof = ROOT / "profiles" / "relax_sssp_rmat22_traffic.json"
    if prof.exists():
        tr = json.loads(prof.read_text())
        if tr.get("kernel") == roofline["kernel"]:  # a capture of this configuration's kernel
            roofline["traffic"] = tr.get("dram_bytes_per_launch")
            roofline["traffic_note"] = tr.get("note")
            roofline["traffic_captured_with"] = tr.get("captured_with")

    # the other styles and the selectors (a few steps each)
    styles = {}
    cand = list(range(i2.I2_NUM_VARIANTS)) + ["vp_cta_plain", "heuristic"]
    if SELECTOR_PARAMS.exists():
        i2.mlp_set_params(np.fromfile(SELECTOR_PARAMS, np.float32))
        cand.append("learned")
    for v in ([] if args.no_styles else cand):
        name = v if isinstance(v, str) else i2.VARIANTS[v]
        if v in (4, 5) and not dg.info["symmetric"]:
            continue
        if v == 8:  # union-find computes CC labels only
            continue
        b = None
        if v == "vp_cta_plain":  # the edge-balanced push without the near/far ordering
            v, b = "vp_cta", 0
        with torch.cuda.stream(stream):
            steps(1, v, b)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        steps(args.style_steps, v, b)
        f1.record(stream)
        f1.synchronize()
        styles[name] = 1e-9 * E / (f0.elapsed_time(f1) / args.style_steps * 1e-3)
    fixed = {k: v for k, v in styles.items() if k not in ("heuristic", "learned")} or {variant: value / world}

    # end to end through the C ABI from pinned host buffers
    hp = i2.ECLGraph(V, E, pinned_copy(host.nindex), pinned_copy(host.nlist), pinned_copy(host.eweight))
    out = pinned_copy(np.zeros(V, np.int32))
    # Median over steps: single upload/run/free cycles on the shared host
    # occasionally stall for 100-600 ms in driver calls, in any phase.
    ts, parts = [], []
    for k in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        gg = i2.DeviceGraph.upload(hp)
        t1 = time.perf_counter()
        gg.sssp(src, variant=variant, out=out, delta=delta, budget=budget)
        t2 = time.perf_counter()
        gg.free()
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        if k > 0:
            ts.append(t3 - t0)
            parts.append((t1 - t0, t2 - t1, t3 - t2))
    e2e_s = dist.max(statistics.median(ts), dev)
    e2e = {"value": world * 1e-9 * E / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": 4 * (V + 1) + 8 * E, "d2h_bytes_per_step": 4 * V,
           "ms_per_step": 1e3 * e2e_s,
           "ms_upload_sssp_free": [round(1e3 * statistics.median(p[j] for p in parts), 3) for j in range(3)],
           "query_only_note": "per-query C-ABI call on a resident graph: see e2e_query"}
    q0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        dg.sssp(src, variant=variant, out=out, delta=delta, budget=budget)
    q_s = (time.perf_counter() - q0) / args.e2e_steps
    e2e_query = {"value": world * 1e-9 * E / dist.max(q_s, dev), "unit": UNIT, "h2d_bytes_per_step": 4,
                 "d2h_bytes_per_step": 4 * V}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = ref_cpu_baseline(host, src, 3, "sssp_vertex_cpp")
            g18 = i2.gen_rmat(18, 16, 0.57, 0.19, 0.19, seed=22)
            same = ref_cpu_baseline(g18, graph_source(g18), 1, "sssp_edge_cpp")
            cpu["same_style"] = {"program": "sssp_edge_cpp (E_Data_Push)", "value": same["value"],
                                 "sample": "RMAT scale 18 (same parameters), 1 traversal"}
        except Exception as exc:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {exc}"}
    ref_cuda = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            ref_cuda = ref_cuda_baseline(host, src)
        except Exception as exc:  # reported, not fatal
            ref_cuda = {"unavailable": str(exc)}

    # per step: k_reset, k_fill, k_seed and the relax launch(es)
    launches = args.steps * (3 + (1 if graph_loop else rep_g.iterations))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": bench_config(args, host, world),
            "roofline": roofline, "cpu_baseline": cpu, "reference_cuda": ref_cuda, "e2e": e2e,
            "e2e_query": e2e_query,
            "gpu_launches": launches, "clocks": clk,
            "styles_gteps": styles, "best_fixed_style": max(fixed, key=fixed.get),
            "iterations": rep_g.iterations, "reached_vertices": rep_g.reached_vertices,
            "reached_edges": rep_g.reached_edges, "verified": "shortest-path certificate"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    dg.free()
    dist.close()


def _event_time(torch, stream, fn, steps: int) -> float:
    """Device seconds per step of fn() on `stream` (CUDA events)."""
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / steps


def er16_cpu_programs(g) -> dict:
    """Every reference OpenMP (38) and C++-threads (40) BFS program, built
    unchanged, on the ER graph from vertex 0 through its own main(): the
    median of its 3 runs and its own verifier's verdict, at all host threads
    and at one. Best and median over the programs whose verifier passed."""
    import oracle

    progs = oracle.bfs_programs()
    if not progs:
        return {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                "sample": "unavailable: oracle/_ref/bfs_{omp,cpp} not built"}
    nproc = os.cpu_count() or 1
    runs = {}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "er16.egr")
        oracle.write_egr(g, path)
        for th in (nproc, 1):
            for model, name in progs:
                r = oracle.run_bfs_program(model, name, path, 0, th)
                runs.setdefault(str(th), {})[f"{model}/{name}"] = {
                    "gteps": 1e-9 * g.edges / r["runtime"] if r["runtime"] else None,
                    "seconds": r["runtime"], "verified": r["verified"] and r["rc"] == 0}
    summary = {}
    for th, rs in runs.items():
        ok = {k: v["gteps"] for k, v in rs.items() if v["verified"] and v["gteps"]}
        best = max(ok, key=ok.get) if ok else None
        summary[th] = {"programs": len(rs), "verified": len(ok),
                       "failed_own_verifier": sorted(k for k, v in rs.items() if not v["verified"]),
                       "best": {"program": best, "gteps": ok[best]} if best else None,
                       "median_gteps": statistics.median(ok.values()) if ok else None}
    top = summary[str(nproc)]["best"]
    return {"value": top["gteps"] if top else None, "unit": UNIT, "cores": nproc, "kind": "reference",
            "program": top["program"] if top else None,
            "sample": "full graph; each program's own main(): median of its 3 runs, its own verifier",
            "summary": summary, "all": runs}


def run_er16(args, rank: int, world: int, local: int):
    """Config: ER G(n=65,536, m=262,144 distinct undirected pairs) = 524,288 CSR
    entries, BFS from vertex 0 -- the reference's CPU configuration. Our GPU
    BFS (fixed edge-balanced style and the heuristic), beside the reference's
    OpenMP and C++-threads BFS programs on this host at all cores and at one.
    Replicas only: each rank runs the same traversal."""
    import torch

    import indigo2suite_b200 as i2
    import oracle

    torch.cuda.set_device(local)
    dist = Dist(world, "nccl")
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    g = i2.gen_er(65536, 262144, 1)
    if g.edges != 524288:
        raise SystemExit(f"ER graph has {g.edges} CSR entries, expected 524288")
    dg = i2.DeviceGraph.upload(g)
    ref = oracle.bfs(g, 0)
    res = {}
    clocks = Clocks(local)
    clocks.start()
    for v in ("vp_cta", "heuristic"):
        d, _ = dg.bfs(0, variant=v)
        if not np.array_equal(d, ref):
            raise SystemExit(f"BFS {v} differs from the oracle")
        run = lambda: dg.run_device(i2.I2_BFS, 0, variant=v, stream=sp, report=False)  # noqa: E731
        for _ in range(args.warmup):
            run()
        torch.cuda.synchronize()
        res[v] = _event_time(torch, stream, run, args.steps)
    clk = clocks.stop()
    dist.barrier()
    t = dist.max(res["vp_cta"], dev)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = er16_cpu_programs(g)
    line = {"metric": METRIC, "value": world * 1e-9 * g.edges / t, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "er16_bfs_cpu_config", "nodes": g.nodes, "edges": g.edges, "source": 0,
                       "variant": "vp_cta", "l2": "graph fits in L2 (2.4 MB): launch-latency bound",
                       "parallelism": f"replicas x{world}"},
            "heuristic_gteps": world * 1e-9 * g.edges / dist.max(res["heuristic"], dev),
            "cpu_baseline": cpu,
            "clocks": clk, "verified": "bit-exact vs the oracle (GPU and reference CPU programs)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    dg.free()
    dist.close()


def run_batch512(args, rank: int, world: int, local: int):
    """Config: 512 graphs (log-uniform 1e3..1e6 vertices, ER/RMAT/grid), BFS +
    SSSP from each graph's highest-degree vertex; batched (one device loop for
    all graphs) vs one launch sequence per graph. Graphs shard across ranks."""
    import torch

    import indigo2suite_b200 as i2
    from indigo2suite_b200 import shard, workloads

    torch.cuda.set_device(local)
    dist = Dist(world, "nccl")
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    specs = workloads.batch_specs(512)
    lo, hi = shard.shard_range(len(specs), rank, world)
    # every graph generated on the device (the same CSR as the host
    # generators), then copied into the disjoint union on the device
    t0 = time.time()
    per = [workloads.build_device(x) for x in specs[lo:hi]]
    torch.cuda.synchronize()
    gen_s = time.time() - t0
    graphs = per
    srcs = [g.hub() for g in per]
    E = sum(g.edges for g in per)
    V = sum(g.nodes for g in per)
    t0 = time.time()
    b = i2.Batch(per)
    union_s = time.time() - t0
    variant = args.variant
    # the autotuner's committed table (style, blocks per SM, heavy threshold),
    # applied to the batched and the per-graph runs alike
    from indigo2suite_b200 import autotune

    tuned = autotune.load()
    if tuned:
        variant = tuned["style"]
        b.tune(heavy_threshold=tuned["heavy_threshold"], blocks_per_sm=tuned["blocks_per_sm"])
        for g in per:
            g.tune(heavy_threshold=tuned["heavy_threshold"], blocks_per_sm=tuned["blocks_per_sm"])
    # parity: batched == per-graph, for both algorithms
    for algo in (i2.I2_BFS, i2.I2_SSSP):
        b.run_device(algo, srcs, variant=variant)
        got = b.result()
        for k in range(0, len(graphs), 37):
            d, _ = per[k]._run(algo, srcs[k], variant, i2.I2_LOOP_GRAPH, 0, False, None, None)
            if not np.array_equal(d, got[k]):
                raise SystemExit(f"batched result differs from per-graph result (graph {k}, algo {algo})")

    def batched():
        for algo in (i2.I2_BFS, i2.I2_SSSP):
            b.run_device(algo, srcs, variant=variant, stream=sp, report=False)

    def per_graph():
        for k, g in enumerate(per):
            for algo in (i2.I2_BFS, i2.I2_SSSP):
                g.run_device(algo, srcs[k], variant=variant, stream=sp, report=False)

    for _ in range(args.warmup):
        batched()
        per_graph()
    torch.cuda.synchronize()
    dist.barrier()
    clocks = Clocks(local)
    clocks.start()  # (settles for a moment: starting nvidia-smi queries the device)
    t_b = _event_time(torch, stream, batched, args.steps)
    clk = clocks.stop()
    t_p = _event_time(torch, stream, per_graph, max(1, args.steps // 3))
    # reference-shaped per-graph runs: host loop with one read-back per iteration
    def per_graph_host():
        for k, g in enumerate(per):
            for algo in (i2.I2_BFS, i2.I2_SSSP):
                g.run_device(algo, srcs[k], variant=variant, stream=sp, loop=i2.I2_LOOP_HOST)
    t_h = _event_time(torch, stream, per_graph_host, 1)
    t_b = dist.max(t_b, dev)
    t_p = dist.max(t_p, dev)
    t_h = dist.max(t_h, dev)
    Etot = int(dist.max(float(E), dev)) if world == 1 else E
    value = world * 2 * 1e-9 * E / t_b  # weak per-rank shares are equal in count
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_b, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "batch512_bfs_sssp", "graphs": len(specs), "graphs_this_rank": len(graphs),
                       "nodes_this_rank": V, "edges_this_rank": E, "variant": variant,
                       "tuning": tuned or "untuned (no indigo2suite_b200/tuning_table.json)",
                       "families": "ER(avg deg 8)/RMAT(ef16)/grid, n log-uniform [1e3,1e6]",
                       "parallelism": f"graphs sharded x{world}", "generation_s": gen_s,
                       "generation": "on the device", "union_s": union_s},
            "batched_ms": 1e3 * t_b, "per_graph_ms": 1e3 * t_p, "per_graph_host_loop_ms": 1e3 * t_h,
            "speedup_vs_per_graph": t_p / t_b, "speedup_vs_per_graph_host_loop": t_h / t_b,
            "clocks": clk, "verified": "batched == per-graph on every 37th graph"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.free()
    for g in per:
        g.free()
    dist.close()


def run_grid4096(args, rank: int, world: int, local: int):
    """Config: BFS and CC on the 4096 x 4096 grid (5% removed, 0.1% long-range),
    every fixed style, the heuristic and the learned selector."""
    import torch

    import indigo2suite_b200 as i2

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    import oracle

    g = i2.gen_grid(4096, 0.05, 0.001, seed=3)
    dg = i2.DeviceGraph.upload(g)
    if SELECTOR_PARAMS.exists():
        i2.mlp_set_params(np.fromfile(SELECTOR_PARAMS, np.float32))
    # every measured configuration's result, bit-exact against the oracle
    refs = {i2.I2_BFS: oracle.bfs(g, 0), i2.I2_CC: oracle.cc(g)}
    verified = {}
    clocks = Clocks(local)
    clocks.start()
    out = {}
    for an, algo in (("bfs", i2.I2_BFS), ("cc", i2.I2_CC)):
        res = {}
        for v in list(range(i2.I2_NUM_VARIANTS)) + ["heuristic", "learned"]:
            name = v if isinstance(v, str) else i2.VARIANTS[v]
            if v == 8 and algo != i2.I2_CC:  # union-find computes CC labels only
                continue
            run = lambda: dg.run_device(algo, 0, variant=v, stream=sp, report=False)  # noqa: E731
            run()
            torch.cuda.synchronize()
            res[name] = 1e3 * _event_time(torch, stream, run, max(1, args.steps // 5))
            got = dg._run(algo, 0, v, i2.I2_LOOP_GRAPH, 0, False, None)[0]
            if not np.array_equal(got, refs[algo]):
                raise SystemExit(f"grid4096 {an} {name}: result differs from the oracle")
            verified[f"{an}/{name}"] = "bit-exact vs oracle"
        rep = dg.run_device(algo, 0, variant="learned")
        fixed = {k: t for k, t in res.items() if k not in ("heuristic", "learned")}
        best = min(fixed, key=fixed.get)
        out[an] = {"ms": res, "best_fixed": best, "learned_vs_best_fixed": fixed[best] / res["learned"],
                   "learned_vs_heuristic": res["heuristic"] / res["learned"], "iterations_learned": rep.iterations,
                   "variant_hist_learned": rep.variant_hist, "gteps_learned": 1e-9 * g.edges / (res["learned"] * 1e-3)}
    line = {"metric": METRIC, "value": out["bfs"]["gteps_learned"], "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "grid4096_bfs_cc_selector", "nodes": g.nodes, "edges": g.edges,
                       "remove": 0.05, "long_range": 0.001, "source": 0},
            "results": out, "clocks": clocks.stop(), "verified": verified}
    print(json.dumps(line), flush=True)
    dg.free()


def run_rmat26(args, rank: int, world: int, local: int):
    """Config: RMAT scale 26 (--scale), 64 seeded sources (--sources; degree
    >= 1) for BFS and SSSP, CC once; the edge-balanced fixed style (SSSP also
    with the budgeted near/far ordering), the heuristic and the learned
    selector; BFS, SSSP and CC on the graph's degree-ordered copy unless
    --order none. Sources shard across ranks."""
    import torch

    import indigo2suite_b200 as i2
    from indigo2suite_b200 import shard

    torch.cuda.set_device(local)
    dist = Dist(world, "nccl")
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    t0 = time.time()
    loop = {"graph": i2.I2_LOOP_GRAPH, "host": i2.I2_LOOP_HOST, "relaunch": i2.I2_LOOP_RELAUNCH}[args.loop]
    nsrc = args.sources
    dg = i2.DeviceGraph.generate_rmat(args.scale, 16, 0.57, 0.19, 0.19, seed=args.scale)
    gen_s = time.time() - t0
    # BFS, SSSP and CC on the degree-ordered copy, results in original IDs
    t1 = time.time()
    dg.reorder(args.order)
    torch.cuda.synchronize()
    order_s = time.time() - t1
    if SELECTOR_PARAMS.exists():
        i2.mlp_set_params(np.fromfile(SELECTOR_PARAMS, np.float32))
    rng = np.random.default_rng(args.scale)
    srcs = []
    while len(srcs) < nsrc:
        v = int(rng.integers(0, dg.nodes))
        if dg.degree(v) > 0:
            srcs.append(v)
    lo, hi = shard.shard_range(nsrc, rank, world)
    mine = srcs[lo:hi]
    res = {}
    peak, peak_kind = peaks()
    clocks = Clocks(local)
    clocks.start()
    algos = [x for x in (("bfs", i2.I2_BFS), ("sssp", i2.I2_SSSP), ("cc", i2.I2_CC)) if x[0] in args.algos.split(",")]
    keep = lambda name: args.rows == "all" or name in args.rows.split(",")
    for an, algo in algos:
        # algorithmic bytes per traversal (reached counts of the first source:
        # every source with an edge lies in the giant component)
        rep = dg.run_device(algo, mine[0], variant="vp_cta", stream=sp)
        b_alg = {"bfs": 8.0 * rep.reached_edges + 20.0 * rep.reached_vertices,
                 "sssp": 12.0 * rep.reached_edges + 20.0 * rep.reached_vertices,
                 "cc": 8.0 * dg.edges + 12.0 * dg.nodes}[an]
        rows = [("vp_cta", "vp_cta", 0), ("heuristic", "heuristic", 0), ("learned", "learned", 0)]
        if algo == i2.I2_SSSP:
            rows.insert(1, ("vp_cta_budget", "vp_cta", i2.I2_SSSP_BUDGET_AUTO))
        for name, v, budget in filter(lambda r: keep(r[0]), rows):
            ss = mine if algo != i2.I2_CC else mine[:1]
            run = lambda s_: dg.run_device(algo, s_, variant=v, loop=loop, stream=sp, report=False,
                                           budget=budget)
            run(ss[0])
            torch.cuda.synchronize()
            it = iter(ss)
            t = _event_time(torch, stream, lambda: run(next(it)), len(ss))
            t = dist.max(t, dev)
            res[f"{an}/{name}"] = {"ms_per_traversal": 1e3 * t, "gteps": 1e-9 * dg.edges / t,
                                   "b_alg_gb": 1e-9 * b_alg, "achieved_gbs": 1e-9 * b_alg / t,
                                   "roofline_frac": 1e-9 * b_alg / t / peak}
    clk = clocks.stop()
    # results of the measured configurations from two of this rank's sources,
    # checked by the size-independent certificates (no serial run over 2e9 edges)
    import oracle

    host = dg.download()
    verified = {}
    styles = [v for v in ("vp_cta", "heuristic", "learned") if keep(v)]
    for s_ in mine[:2]:
        for v in styles:
            for an, algo, wt in (("bfs", i2.I2_BFS, False), ("sssp", i2.I2_SSSP, True)):
                if an not in args.algos.split(","):
                    continue
                d = dg._run(algo, s_, v, loop, 0, False, None)[0]
                c = oracle.certify_distances(host, s_, d, weighted=wt)
                if c is not None:
                    raise SystemExit(f"rmat26 {an} {v} source {s_}: certificate failed: {c}")
                verified[f"{an}/{v}/src{s_}"] = "shortest-path certificate"
        if "sssp" in args.algos.split(",") and keep("vp_cta_budget"):
            d = dg._run(i2.I2_SSSP, s_, "vp_cta", loop, 0, False, None, budget=i2.I2_SSSP_BUDGET_AUTO)[0]
            c = oracle.certify_distances(host, s_, d, weighted=True)
            if c is not None:
                raise SystemExit(f"rmat26 sssp vp_cta_budget source {s_}: certificate failed: {c}")
            verified[f"sssp/vp_cta_budget/src{s_}"] = "shortest-path certificate"
    for v in styles if "cc" in args.algos.split(",") else ():
        lab = dg._run(i2.I2_CC, 0, v, loop, 0, False, None)[0]
        c = oracle.certify_cc(host, lab)
        if c is not None:
            raise SystemExit(f"rmat26 cc {v}: certificate failed: {c}")
        verified[f"cc/{v}"] = "minimum-label certificate"
    del host
    head = res.get("bfs/learned") or next(iter(res.values()))
    line = {"metric": METRIC, "value": world * head["gteps"], "unit": UNIT, "n_gpus": world,
            "steps": nsrc, "warmup": 1, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "int32", "data": "synthetic",
            "config": {"workload": f"rmat{args.scale}_{'_'.join(a for a, _ in algos)}_{nsrc}src",
                       "nodes": dg.nodes, "edges": dg.edges, "generation_s": gen_s, "loop": args.loop,
                       "vertex_order": args.order, "reorder_s": order_s,
                       "rows": args.rows,
                       "parallelism": f"sources sharded x{world}"},
            "roofline_peak_gbs": peak, "roofline_peak_source": peak_kind,
            "results": res, "clocks": clk, "verified": verified}
    if rank == 0:
        print(json.dumps(line), flush=True)
    dg.free()
    dist.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--variant", default="vp_cta")
    ap.add_argument("--budget", type=int, default=-1,
                    help="SSSP budgeted near/far ordering of the vp_cta style: < 0 the engine's default "
                         "budget (28672 edges per SM), 0 off, > 0 edges per near set")
    ap.add_argument("--delta", type=int, default=0,
                    help="SSSP near/far threshold step of the vp_cta style: <= 0 off, > 0 this step")
    ap.add_argument("--style-steps", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-styles", action="store_true", help="skip the per-style comparison")
    ap.add_argument("--workload", choices=["sssp_rmat22", "batch512", "grid4096", "rmat26", "er16"],
                    default="sssp_rmat22",
                    help="sssp_rmat22 is the benchmark line; the others are the other configurations")
    ap.add_argument("--scale", type=int, default=26, help="rmat26 workload: RMAT scale")
    ap.add_argument("--sources", type=int, default=64, help="rmat26 workload: BFS/SSSP sources")
    ap.add_argument("--algos", default="bfs,sssp,cc", help="rmat26 workload: algorithms to run")
    ap.add_argument("--rows", default="all",
                    help="rmat26 workload: rows to run (vp_cta, vp_cta_budget, heuristic, learned) or all")
    ap.add_argument("--order", choices=["none", "degree"], default="degree",
                    help="rmat26 workload: vertex numbering BFS, SSSP and CC run under (degree: a copy "
                         "renumbered by descending degree, results in original IDs)")
    ap.add_argument("--loop", choices=["graph", "host", "relaunch"], default="graph",
                    help="graph: one CUDA graph whose resident kernel runs every iteration (default); "
                         "host: one host launch per iteration; relaunch: one launch per iteration "
                         "from the graph's device-side loop")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if world != args.gpus and not (world == 1 and args.gpus == 1):
        if rank == 0:
            print(f"warning: --gpus {args.gpus} but WORLD_SIZE {world}", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    {"sssp_rmat22": run_ours, "batch512": run_batch512, "grid4096": run_grid4096, "er16": run_er16,
     "rmat26": run_rmat26}[args.workload](args, rank, world, local)


if __name__ == "__main__":
    main()
