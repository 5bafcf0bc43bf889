"""Bit-exact parity of the CUDA engine with the oracle and the golden vectors,
for every variant, both loop modes, and the per-iteration selectors."""
import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle

pytestmark = pytest.mark.gpu

FIXED = list(range(i2.I2_NUM_VARIANTS))
ALL = FIXED + ["heuristic", "learned"]


@pytest.fixture(autouse=True, scope="module")
def _selector_params():
    from indigo2suite_b200 import selector

    if i2.device_count() > 0:
        i2.mlp_set_params(np.fromfile(selector.PARAMS_PATH, np.float32))


def _variants_for(dg):
    out = []
    for v in ALL:
        if v in (4, 5, 8) and not dg.info["symmetric"]:
            continue
        out.append(v)
    return out


def _for(algo, v):
    """Union-find (style 8) computes CC labels only."""
    return v != 8 or algo == "cc"


def test_golden_all_variants_both_loops(gpu, golden):
    for name, case in golden.items():
        dg = i2.DeviceGraph.upload(case["graph"])
        assert dg.info["symmetric"] == 1, name
        for v in _variants_for(dg):
            for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_HOST, i2.I2_LOOP_RELAUNCH):
                for s in case["sources"] if _for("bfs", v) else []:
                    d, _ = dg.bfs(s, variant=v, loop=loop)
                    np.testing.assert_array_equal(d, case["bfs"][s], err_msg=f"{name} bfs {v} {loop} {s}")
                    d, _ = dg.sssp(s, variant=v, loop=loop)
                    np.testing.assert_array_equal(d, case["sssp"][s], err_msg=f"{name} sssp {v} {loop} {s}")
                lab, _ = dg.cc(variant=v, loop=loop)
                np.testing.assert_array_equal(lab, case["cc"], err_msg=f"{name} cc {v} {loop}")
        dg.free()


def _graphs():
    return {
        "er": i2.gen_er(20000, 80000, 3),
        "rmat14": i2.gen_rmat(14, 16, seed=5),
        "grid": i2.gen_grid(96, 0.05, 0.002, 7),
        "rmat16": i2.gen_rmat(16, 16, seed=1),
    }


@pytest.fixture(scope="module")
def seeded():
    return _graphs()


@pytest.mark.parametrize("name", ["er", "rmat14", "grid", "rmat16"])
def test_seeded_all_variants_vs_oracle(gpu, seeded, name):
    g = seeded[name]
    dg = i2.DeviceGraph.upload(g)
    src = int(np.argmax(g.degrees()))
    ref_b, ref_s, ref_c = oracle.bfs(g, src), oracle.sssp(g, src), oracle.cc(g)
    for v in _variants_for(dg):
        for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_RELAUNCH):
            if _for("bfs", v):
                d, rep = dg.bfs(src, variant=v, loop=loop)
                np.testing.assert_array_equal(d, ref_b, err_msg=f"bfs {v} {loop}")
                assert rep.reached_vertices == int((ref_b != i2.INF).sum())
                d, _ = dg.sssp(src, variant=v, loop=loop)
                np.testing.assert_array_equal(d, ref_s, err_msg=f"sssp {v} {loop}")
            lab, _ = dg.cc(variant=v, loop=loop)
            np.testing.assert_array_equal(lab, ref_c, err_msg=f"cc {v} {loop}")
    dg.free()


def test_heavy_path_and_queue_overflow(gpu, seeded):
    # A low heavy threshold sends many frontier vertices through the grid-wide
    # heavy path; a high one keeps hubs in the thread variant (staging overflow).
    g = seeded["rmat16"]
    src = int(np.argmax(g.degrees()))
    ref_b, ref_s, ref_c = oracle.bfs(g, src), oracle.sssp(g, src), oracle.cc(g)
    dg = i2.DeviceGraph.upload(g)
    for heavy in (32, 200, 1 << 20):
        dg.tune(heavy_threshold=heavy)
        for v in (0, 1, 2, 3, 7, "heuristic"):
            np.testing.assert_array_equal(dg.bfs(src, variant=v)[0], ref_b, err_msg=f"{heavy} {v}")
            np.testing.assert_array_equal(dg.sssp(src, variant=v)[0], ref_s, err_msg=f"{heavy} {v}")
            np.testing.assert_array_equal(dg.cc(variant=v)[0], ref_c, err_msg=f"{heavy} {v}")
    dg.free()


def test_blocks_per_sm_do_not_change_results(gpu, seeded):
    g = seeded["er"]
    ref = oracle.sssp(g, 0)
    dg = i2.DeviceGraph.upload(g)
    for bps in (1, 2, 8):
        dg.tune(blocks_per_sm=bps)
        for v in (0, 2, 4, 6):
            np.testing.assert_array_equal(dg.sssp(0, variant=v)[0], ref)
    dg.free()


def test_repeated_runs_are_identical_and_independent(gpu, seeded):
    g = seeded["rmat14"]
    dg = i2.DeviceGraph.upload(g)
    ref = oracle.sssp(g, 7)
    for _ in range(5):
        np.testing.assert_array_equal(dg.sssp(7, variant="heuristic")[0], ref)
        dg.bfs(3, variant=1)
        dg.cc(variant=6)
    dg.free()


def test_multi_source_sources_of_every_vertex_class(gpu, seeded):
    g = seeded["grid"]
    dg = i2.DeviceGraph.upload(g)
    deg = g.degrees()
    for src in (0, g.nodes - 1, int(np.argmin(deg)), int(np.argmax(deg))):
        np.testing.assert_array_equal(dg.bfs(src)[0], oracle.bfs(g, src))
        np.testing.assert_array_equal(dg.sssp(src)[0], oracle.sssp(g, src))
    dg.free()


def test_directed_graph_push_variants_and_pull_refused(gpu):
    # 0 -> 1 -> 2 -> 3, 4 -> 2 (not symmetric)
    g = i2.ECLGraph(5, 4, np.array([0, 1, 2, 3, 3, 4], np.int32), np.array([1, 2, 3, 2], np.int32),
                    np.array([3, 1, 4, 2], np.int32))
    dg = i2.DeviceGraph.upload(g)
    assert dg.info["symmetric"] == 0
    for v in (0, 1, 2, 3, 6, 7, "heuristic"):
        np.testing.assert_array_equal(dg.bfs(0, variant=v)[0], oracle.bfs(g, 0))
        np.testing.assert_array_equal(dg.sssp(4, variant=v)[0], oracle.sssp(g, 4))
        np.testing.assert_array_equal(dg.cc(variant=v)[0], oracle.cc(g))
    for v in (4, 5):
        with pytest.raises(i2.I2Error) as e:
            dg.bfs(0, variant=v)
        assert e.value.status == i2._capi.I2_ERR_UNSUPPORTED
    with pytest.raises(i2.I2Error) as e:  # union-find needs a symmetric graph
        dg.cc(variant="union_find")
    assert e.value.status == i2._capi.I2_ERR_UNSUPPORTED
    dg.free()


def test_single_vertex_and_edgeless_graphs(gpu):
    g1 = i2.ECLGraph(1, 0, np.array([0, 0], np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    g2 = i2.ECLGraph(70, 0, np.zeros(71, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    for g in (g1, g2):
        dg = i2.DeviceGraph.upload(g)
        for v in ALL:
            if _for("bfs", v):
                np.testing.assert_array_equal(dg.bfs(0, variant=v)[0], oracle.bfs(g, 0))
                np.testing.assert_array_equal(dg.sssp(0, variant=v)[0], oracle.sssp(g, 0))
            np.testing.assert_array_equal(dg.cc(variant=v)[0], np.arange(g.nodes))
        dg.free()


def test_records_and_report(gpu, seeded):
    g = seeded["rmat14"]
    dg = i2.DeviceGraph.upload(g)
    src = int(np.argmax(g.degrees()))
    d, rep = dg.bfs(src, variant="heuristic", record=True)
    recs = dg.records()
    assert len(recs) == rep.iterations > 0
    assert sum(rep.variant_hist) == rep.iterations
    assert recs[0]["size"] == 1
    assert all(r["t_ns"] > 0 for r in recs)
    assert rep.seconds > 0 and 0 < rep.relax_seconds <= rep.seconds * 1.5
    reached = d != i2.INF
    assert rep.reached_vertices == reached.sum()
    assert rep.reached_edges == g.degrees()[reached].sum()
    dg.free()


def test_reference_interface_mirror(gpu, golden):
    case = golden["rmat_s10_ef16_s3"]
    g = case["graph"]
    dg = i2.DeviceGraph.upload(g)
    out = np.empty(g.nodes, np.int32)
    for fn in (i2.GPUbfs_vertex, i2.GPUbfs_edge):
        t = fn(0, dg, out)
        assert t > 0
        np.testing.assert_array_equal(out, case["bfs"][0])
    for fn in (i2.GPUsssp_vertex, i2.GPUsssp_edge):
        fn(0, dg, out)
        np.testing.assert_array_equal(out, case["sssp"][0])
    for fn in (i2.GPUcc_vertex, i2.GPUcc_edge):
        fn(dg, out)
        np.testing.assert_array_equal(out, case["cc"])
    dg.free()


def _directed_chain():
    # 0 -> 1 -> 2 -> 3 (3 has no out-edges), 4 -> 2, heavy first hop
    return i2.ECLGraph(5, 4, np.array([0, 1, 2, 3, 3, 4], np.int32), np.array([1, 2, 3, 2], np.int32),
                       np.array([300, 1, 4, 2], np.int32))


@pytest.mark.parametrize("name", ["er", "rmat14", "grid", "rmat16", "directed", "unit"])
def test_sssp_near_far_ordering_any_step(gpu, seeded, name):
    # Near/far ordering defers pushes at or above a rising threshold; the
    # distances must not depend on the step, including steps far below and far
    # above every weight, on graphs with vertices that have no out-edges.
    if name == "directed":
        g = _directed_chain()
    elif name == "unit":
        g0 = seeded["rmat14"]
        g = i2.ECLGraph(g0.nodes, g0.edges, g0.nindex, g0.nlist, np.ones(g0.edges, np.int32))
    else:
        g = seeded[name]
    dg = i2.DeviceGraph.upload(g)
    deg = g.degrees()
    srcs = [0, int(np.argmax(deg))]
    if name == "directed":
        srcs = [0, 4]
    for s in srcs:
        ref = oracle.sssp(g, s)
        for delta in (-1, 0, 1, 3, 100, 5000, 1 << 20, 1 << 30):
            for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_HOST):
                d, rep = dg.sssp(s, variant="vp_cta", loop=loop, delta=delta)
                np.testing.assert_array_equal(d, ref, err_msg=f"{name} src {s} delta {delta} loop {loop}")
                assert rep.reached_vertices == int((ref != i2.INF).sum())
    dg.free()


def test_sssp_near_far_golden_and_repeat(gpu, golden):
    for name, case in golden.items():
        dg = i2.DeviceGraph.upload(case["graph"])
        for s in case["sources"]:
            for delta in (0, 1, 64, 1 << 16):
                for _ in range(2):  # the piles' state must not leak into the next run
                    d, _ = dg.sssp(s, variant="vp_cta", delta=delta)
                    np.testing.assert_array_equal(d, case["sssp"][s], err_msg=f"{name} {s} {delta}")
        dg.free()


def test_sssp_near_far_reduces_relaxed_work(gpu, seeded):
    # The point of the ordering: fewer vertices are relaxed more than once.
    # With a step of a few mean weights over the mean degree the per-iteration
    # records must show fewer frontier edges in total than plain
    # frontier-driven relaxation, which is also what delta <= 0 runs. (How
    # many edges plain relaxation scans depends on the order of the atomics,
    # so the comparison is a bound, not an equality.)
    g = seeded["rmat16"]
    dg = i2.DeviceGraph.upload(g)
    src = int(np.argmax(g.degrees()))
    base = []
    for delta in (-1, 0):
        _, rep = dg.sssp(src, variant="vp_cta", delta=delta, record=True)
        base.append((rep.iterations, sum(r["edges"] for r in dg.records())))
    step = max(1, int(round(4 * g.eweight.mean() / g.degrees().mean())))
    _, rep = dg.sssp(src, variant="vp_cta", delta=step, record=True)
    near_far = sum(r["edges"] for r in dg.records())
    assert near_far < 0.8 * min(b[1] for b in base)
    assert rep.iterations > max(b[0] for b in base)
    dg.free()


@pytest.mark.parametrize("name", ["er", "rmat14", "grid", "rmat16", "directed", "unit"])
def test_sssp_budget_ordering_any_budget(gpu, seeded, name):
    # The budgeted near/far ordering keeps each near frontier at about B edges:
    # it trims large frontiers (the threshold falls), histograms the far pile
    # when the frontier runs dry (the threshold rises) and drops pile entries a
    # near push superseded. Distances must not depend on B, including B far
    # below one vertex's degree and far above the graph, in every loop mode.
    if name == "directed":
        g = _directed_chain()
    elif name == "unit":
        g0 = seeded["rmat14"]
        g = i2.ECLGraph(g0.nodes, g0.edges, g0.nindex, g0.nlist, np.ones(g0.edges, np.int32))
    else:
        g = seeded[name]
    dg = i2.DeviceGraph.upload(g)
    deg = g.degrees()
    srcs = [0, int(np.argmax(deg))] if name != "directed" else [0, 4]
    for s in srcs:
        ref = oracle.sssp(g, s)
        for budget in (1, 7, 100, 5000, 1 << 20, i2.I2_SSSP_BUDGET_AUTO):
            for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_HOST, i2.I2_LOOP_RELAUNCH):
                d, rep = dg.sssp(s, variant="vp_cta", loop=loop, budget=budget)
                np.testing.assert_array_equal(d, ref, err_msg=f"{name} src {s} budget {budget} loop {loop}")
                assert rep.reached_vertices == int((ref != i2.INF).sum())
    dg.free()


def test_sssp_budget_golden_repeat_and_step_precedence(gpu, golden):
    # Piles, histograms and thresholds must not leak into the next run, and a
    # fixed step (sssp_delta > 0) takes precedence over a budget.
    for name, case in golden.items():
        dg = i2.DeviceGraph.upload(case["graph"])
        for s in case["sources"][:8]:
            for budget, delta in ((3, 0), (64, 0), (i2.I2_SSSP_BUDGET_AUTO, 0), (3, 64)):
                for _ in range(2):
                    d, _ = dg.sssp(s, variant="vp_cta", delta=delta, budget=budget)
                    np.testing.assert_array_equal(d, case["sssp"][s], err_msg=f"{name} {s} {budget} {delta}")
        dg.free()


def test_sssp_budget_reduces_relaxed_work(gpu, seeded):
    # On a skewed graph from its hub, plain frontier-driven relaxation scans
    # the reached edges more than twice; a budget of a few percent of the edges
    # must cut the edges relaxed (relaxation launches only: trims and moves
    # relax nothing) well below that, and the launch records must show the
    # trims and moves that do it.
    g = seeded["rmat16"]
    dg = i2.DeviceGraph.upload(g)
    src = int(np.argmax(g.degrees()))
    _, rep0 = dg.sssp(src, variant="vp_cta", record=True)
    plain = sum(r["edges"] for r in dg.records())
    d, rep = dg.sssp(src, variant="vp_cta", budget=g.edges // 32, record=True)
    np.testing.assert_array_equal(d, oracle.sssp(g, src))
    recs = dg.records()
    relaxed = sum(r["edges"] for r in recs if r["kind"] == 0)
    kinds = {r["kind"] for r in recs}
    assert {0, 1, 3} <= kinds, kinds
    assert plain > 1.5 * rep0.reached_edges
    assert relaxed < 0.75 * plain, (relaxed, plain, rep0.reached_edges)
    dg.free()


def test_union_find_cc(gpu, seeded, golden):
    # Union-find CC reaches the minimum-ID labels from the initial labels and,
    # switched to mid-traversal by a selector, from any label-propagation
    # state; it is refused for BFS and SSSP.
    for name, g in list(seeded.items()) + [(k, c["graph"]) for k, c in golden.items()]:
        dg = i2.DeviceGraph.upload(g)
        ref = oracle.cc(g)
        for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_HOST, i2.I2_LOOP_RELAUNCH):
            lab, rep = dg.cc(variant="union_find", loop=loop)
            np.testing.assert_array_equal(lab, ref, err_msg=f"{name} {loop}")
            assert rep.iterations == 3  # two hook launches, one compress launch
            lab, rep = dg.cc(variant="heuristic", loop=loop)
            np.testing.assert_array_equal(lab, ref, err_msg=f"{name} heuristic {loop}")
        with pytest.raises(i2.I2Error) as e:
            dg.bfs(0, variant="union_find")
        assert e.value.status == i2._capi.I2_ERR_UNSUPPORTED
        dg.free()


@pytest.mark.parametrize("name", ["grid", "rmat14"])
def test_switching_style_at_any_iteration(gpu, seeded, name):
    # The frontier contract lets a selector change style at any iteration. Run
    # style a for the first k iterations and style b after (then_at,
    # then_variant), for several pairs and switch points: results must not
    # change. For CC this includes union-find from a label-propagation state.
    g = seeded[name]
    dg = i2.DeviceGraph.upload(g)
    src = int(np.argmax(g.degrees()))
    ref = {"bfs": oracle.bfs(g, src), "sssp": oracle.sssp(g, src), "cc": oracle.cc(g)}
    pairs = [(2, 4), (4, 2), (0, 6), (6, 3), (7, 1), (5, 2), (2, 8), (4, 8), (6, 8)]
    for a, b in pairs:
        for k in (1, 2, 3, 5):
            for an in ("bfs", "sssp", "cc"):
                if not (_for(an, a) and _for(an, b)):
                    continue
                src_arg = () if an == "cc" else (src,)
                out, _ = getattr(dg, an)(*src_arg, variant=a, then_variant=b, then_at=k)
                np.testing.assert_array_equal(out, ref[an], err_msg=f"{name} {an} {a}->{b} at {k}")
    dg.free()


def test_batch_tuning_keeps_results(gpu):
    from indigo2suite_b200 import workloads

    gs = [workloads.build(s) for s in workloads.batch_specs(12, seed=21, nmax=2e4)]
    srcs = [workloads.source(g) for g in gs]
    b = i2.Batch(gs)
    for heavy, bps, style in ((1024, 2, "vp_thread"), (16384, 8, "vp_warp"), (4096, 6, "heuristic")):
        b.tune(heavy_threshold=heavy, blocks_per_sm=bps)
        for algo, ref in ((i2.I2_BFS, oracle.bfs), (i2.I2_SSSP, oracle.sssp)):
            got, _ = b.run(algo, srcs, variant=style)
            for k, g in enumerate(gs):
                np.testing.assert_array_equal(got[k], ref(g, srcs[k]), err_msg=f"{style} {bps} {heavy} graph {k}")
    b.free()


def test_pooled_memory_reuse_and_trim(gpu):
    # Graphs freed and uploaded again reuse the pool's memory; results do not
    # depend on what the reused blocks held, and trimming the pool leaves
    # later uploads working.
    g1 = i2.gen_rmat(14, 16, seed=41)
    g2 = i2.gen_er(30000, 120000, 42)
    src1, src2 = int(np.argmax(g1.degrees())), int(np.argmax(g2.degrees()))
    ref1, ref2 = oracle.sssp(g1, src1), oracle.bfs(g2, src2)
    for k in range(3):
        dg = i2.DeviceGraph.upload(g1)
        np.testing.assert_array_equal(dg.sssp(src1)[0], ref1)
        dg.free()
        dg = i2.DeviceGraph.upload(g2)
        np.testing.assert_array_equal(dg.bfs(src2, variant="heuristic")[0], ref2)
        np.testing.assert_array_equal(dg.cc(variant="union_find")[0], oracle.cc(g2))
        dg.free()
        if k == 1:
            i2.trim_device_memory()
    i2.trim_device_memory()
