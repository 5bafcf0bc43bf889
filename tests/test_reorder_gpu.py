"""Traversals on the degree-ordered copy of a graph (i2_graph_reorder).

BFS and SSSP run on a copy renumbered by descending degree and their values
are gathered back to the original IDs; these tests check that every style,
selector, ordering and loop mode still returns exactly the oracle's levels,
distances and minimum-ID labels in the original numbering, that MIS and CC of
directed graphs keep the original CSR, and that
dropping, re-tuning and re-weighting a reordered graph keep it right."""
import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle

pytestmark = pytest.mark.gpu

STYLES = list(range(8)) + ["heuristic", "learned"]


@pytest.fixture(autouse=True, scope="module")
def _selector_params():
    from indigo2suite_b200 import selector

    if i2.device_count() > 0:
        i2.mlp_set_params(np.fromfile(selector.PARAMS_PATH, np.float32))


def _directed(full):
    deg = np.diff(full.nindex)
    u = np.repeat(np.arange(full.nodes, dtype=np.int32), deg)
    keep = u < full.nlist
    ni = np.zeros(full.nodes + 1, np.int32)
    np.cumsum(np.bincount(u[keep], minlength=full.nodes), out=ni[1:])
    return i2.ECLGraph(full.nodes, int(keep.sum()), ni, np.ascontiguousarray(full.nlist[keep]),
                       np.ascontiguousarray(full.eweight[keep]))


def _sources(g, k=3):
    deg = g.degrees()
    rng = np.random.default_rng(g.nodes)
    out = [int(np.argmax(deg))]
    out += [int(v) for v in rng.choice(np.flatnonzero(deg > 0), k - 1, replace=False)]
    iso = np.flatnonzero(deg == 0)
    if iso.size:
        out.append(int(iso[0]))
    return out


def test_reordered_bfs_sssp_match_oracle_every_style_and_loop(gpu):
    graphs = {"rmat14": i2.gen_rmat(14, 16, seed=61), "er": i2.gen_er(30000, 120000, 62),
              "grid": i2.gen_grid(120, 0.05, 0.002, 63)}
    for name, g in graphs.items():
        dg = i2.DeviceGraph.upload(g)
        dg.reorder("degree")
        for s in _sources(g):
            want_b, want_s = oracle.bfs(g, s), oracle.sssp(g, s)
            for v in STYLES:
                for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_HOST, i2.I2_LOOP_RELAUNCH):
                    d, rep = dg.bfs(s, variant=v, loop=loop)
                    np.testing.assert_array_equal(d, want_b, err_msg=f"{name} bfs {v} {loop} {s}")
                    assert rep.seconds > 0
                    d, _ = dg.sssp(s, variant=v, loop=loop)
                    np.testing.assert_array_equal(d, want_s, err_msg=f"{name} sssp {v} {loop} {s}")
            for budget in (i2.I2_SSSP_BUDGET_AUTO, 4096):
                d, _ = dg.sssp(s, variant="vp_cta", budget=budget)
                np.testing.assert_array_equal(d, want_s, err_msg=f"{name} sssp budget {budget} {s}")
            d, _ = dg.sssp(s, variant="vp_cta", delta=256)
            np.testing.assert_array_equal(d, want_s, err_msg=f"{name} sssp delta {s}")
        # CC runs on the copy (symmetric graphs), labels mapped back to each
        # component's smallest original ID; MIS keeps the original CSR
        want_c = oracle.cc(g)
        for v in STYLES + ["union_find"]:
            for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_HOST):
                lab, _ = dg.cc(variant=v, loop=loop)
                np.testing.assert_array_equal(lab, want_c, err_msg=f"{name} cc {v} {loop}")
        np.testing.assert_array_equal(dg.mis()[0], oracle.mis(g), err_msg=f"{name} mis")
        dg.free()


def test_reordered_directed_graph_and_device_results(gpu):
    import torch

    g = _directed(i2.gen_rmat(12, 8, seed=64))
    dg = i2.DeviceGraph.upload(g)
    dg.reorder("degree")
    out = torch.full((g.nodes,), -5, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    for s in _sources(g):
        for algo, ref in ((i2.I2_BFS, oracle.bfs(g, s)), (i2.I2_SSSP, oracle.sssp(g, s))):
            for v in ("vp_cta", "vp_warp", "edge_topo", "push_topo", "heuristic"):
                dg.run_device(algo, s, out_ptr=out.data_ptr(), variant=v, stream=stream.cuda_stream, report=False)
                stream.synchronize()
                np.testing.assert_array_equal(out.cpu().numpy(), ref, err_msg=f"algo {algo} {v} src {s}")
    # pull styles still refuse a directed graph; CC keeps the original CSR
    with pytest.raises(i2.I2Error):
        dg.bfs(0, variant="pull_frontier")
    for v in ("vp_cta", "heuristic"):
        np.testing.assert_array_equal(dg.cc(variant=v)[0], oracle.cc(g), err_msg=f"directed cc {v}")
    dg.free()


def test_reorder_drop_tune_and_weights(gpu):
    g = i2.gen_rmat(16, 16, seed=65)
    s = int(np.argmax(g.degrees()))
    want_b, want_s = oracle.bfs(g, s), oracle.sssp(g, s)
    dg = i2.DeviceGraph.upload(g)
    dg.reorder("degree")
    # a lower heavy threshold re-sizes the copy's heavy lists too
    dg.tune(heavy_threshold=64, blocks_per_sm=4)
    for v in ("vp_thread", "vp_warp", "vp_block", "vp_cta", "heuristic"):
        np.testing.assert_array_equal(dg.bfs(s, variant=v)[0], want_b, err_msg=f"tuned bfs {v}")
        np.testing.assert_array_equal(dg.sssp(s, variant=v)[0], want_s, err_msg=f"tuned sssp {v}")
    recs = dg.bfs(s, variant="vp_cta", record=True)[1]
    assert len(dg.records()) == recs.iterations > 0
    dg.reorder("none")
    np.testing.assert_array_equal(dg.sssp(s, variant="vp_cta")[0], want_s)
    dg.reorder("degree")
    dg.reorder("degree")  # rebuilding replaces the copy
    np.testing.assert_array_equal(dg.sssp(s, variant="heuristic")[0], want_s)
    dg.free()

    # synthetic weights are a function of the original IDs: the copy follows them
    u = i2.ECLGraph(g.nodes, g.edges, g.nindex.copy(), g.nlist.copy(), None)
    du = i2.DeviceGraph.upload(u)
    du.reorder("degree")
    du.synth_weights()
    w = i2.synth_weights(i2.ECLGraph(g.nodes, g.edges, g.nindex.copy(), g.nlist.copy(), None))
    np.testing.assert_array_equal(du.sssp(s, variant="vp_cta")[0], oracle.sssp(w, s))
    du.free()


def test_reorder_rejects_unknown_order(gpu):
    dg = i2.DeviceGraph.upload(i2.gen_rmat(10, 8, seed=66))
    assert i2.lib.i2_graph_reorder(dg._h, 7) == i2.capi.I2_ERR_ARG
    dg.free()


def test_reorder_tiny_and_edgeless_graphs(gpu):
    graphs = {
        "edgeless": i2.ECLGraph(5, 0, np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32)),
        "one_vertex": i2.ECLGraph(1, 0, np.zeros(2, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32)),
        "one_edge": i2.ECLGraph(3, 2, np.array([0, 1, 1, 2], np.int32), np.array([2, 0], np.int32),
                                np.array([7, 7], np.int32)),
    }
    for name, g in graphs.items():
        dg = i2.DeviceGraph.upload(g)
        dg.reorder("degree")
        for s in range(g.nodes):
            np.testing.assert_array_equal(dg.bfs(s)[0], oracle.bfs(g, s), err_msg=f"{name} bfs {s}")
            np.testing.assert_array_equal(dg.sssp(s)[0], oracle.sssp(g, s), err_msg=f"{name} sssp {s}")
        np.testing.assert_array_equal(dg.cc(variant="heuristic")[0], oracle.cc(g), err_msg=f"{name} cc")
        dg.free()
