"""The oracle (oracle/oracle.c) pinned against the reference's own code and the
golden vectors, and the reference verifier's sensitivity to planted mistakes."""
import os
import tempfile

import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle

INF = np.iinfo(np.int32).max


def test_oracle_matches_golden(golden):
    for name, case in golden.items():
        g = case["graph"]
        for s in case["sources"]:
            np.testing.assert_array_equal(oracle.bfs(g, s), case["bfs"][s], err_msg=name)
            np.testing.assert_array_equal(oracle.sssp(g, s), case["sssp"][s], err_msg=name)
        np.testing.assert_array_equal(oracle.cc(g), case["cc"], err_msg=name)
        assert oracle.cc_check(g, case["cc"]) == 0


def test_golden_small_inputs_cover_reference_edge_cases(golden):
    # isolated vertices, unreachable vertices and a triangle are all present
    small = [c for n, c in golden.items() if n.startswith("small_")]
    assert len(small) == 7
    assert any((c["bfs"][0] == INF).any() for c in small)
    assert any(c["graph"].edges == 6 for c in small)
    assert any(len(np.unique(c["cc"])) == 2 for c in small)  # one isolated vertex


@pytest.mark.skipif(not oracle.have_ref(), reason="reference programs not built")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_reference_serial(seed):
    graphs = [i2.gen_er(3000, 9000, seed), i2.gen_rmat(12, 16, seed=seed), i2.gen_grid(48, 0.05, 0.01, seed)]
    for g in graphs:
        src = int(np.argmax(g.degrees()))
        np.testing.assert_array_equal(oracle.bfs(g, src), oracle.ref_serial("bfs", g, src))
        ref = oracle.ref_serial("sssp_edge", g, src)
        np.testing.assert_array_equal(oracle.sssp(g, src), ref)
        np.testing.assert_array_equal(oracle.ref_serial("sssp_vertex", g, src), ref)


@pytest.mark.skipif(not oracle.have_ref(), reason="reference programs not built")
def test_reference_verifier_accepts_oracle_and_rejects_planted_mistakes():
    g = i2.gen_rmat(10, 8, seed=11)
    src = int(np.argmax(g.degrees()))
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.egr")
        oracle.write_egr(g, p)
        d = oracle.sssp(g, src)
        assert oracle.ref_verify("sssp_edge", p, d, src)[0]
        bad = d.copy()
        bad[np.flatnonzero(d < INF)[-1]] -= 1
        assert not oracle.ref_verify("sssp_edge", p, bad, src)[0]
        lab = oracle.cc(g)
        assert oracle.ref_verify("cc_vertex", p, lab, None)[0]
        # merge two components' labels: the reference verifier must object
        comps = np.unique(lab)
        bad = lab.copy()
        bad[lab == comps[1]] = comps[0]
        assert not oracle.ref_verify("cc_vertex", p, bad, None)[0]
        assert oracle.cc_check(g, bad) != 0


def test_cc_check_detects_each_failure_mode():
    g = i2.gen_grid(8, 0.2, 0.0, 3)
    lab = oracle.cc(g)
    assert oracle.cc_check(g, lab) == 0
    bad = lab.copy()
    v = int(np.flatnonzero(g.degrees() > 0)[0])
    bad[v] = (bad[v] + 1) % g.nodes
    assert oracle.cc_check(g, bad) == 1
    bad = lab.copy()
    iso = np.flatnonzero(g.degrees() == 0)
    if len(iso):
        bad[iso[0]] = g.nodes
        assert oracle.cc_check(g, bad) == 2


def test_synth_weights_oracle_matches_library():
    # includes products i*nei that overflow int32 (n > 46341)
    g = i2.gen_er(70000, 50000, 5, weighted=False)
    w = i2.synth_weights(g).eweight
    np.testing.assert_array_equal(w, oracle.synth_weights(g))
    assert (w >= 1).all() and (w <= g.nodes).all()


def test_sp_oracle_matches_library():
    g = i2.gen_rmat(9, 8, seed=2)
    np.testing.assert_array_equal(i2.build_sp(g), oracle.sp(g))


def test_minlabel_is_reachability_minimum_on_directed_graph():
    # 0 -> 1 -> 2, 3 -> 2: label = min vertex that reaches v
    g = i2.ECLGraph(4, 3, np.array([0, 1, 2, 2, 3], np.int32), np.array([1, 2, 2], np.int32))
    np.testing.assert_array_equal(oracle.cc(g), [0, 0, 0, 3])
