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


def _greedy_mis(g, unsigned_priority):
    """Pure-Python restatement: vertices in decreasing rank, each in the set
    iff no neighbour already in it."""
    prio = i2.mis_priority(np.arange(g.nodes))
    key = prio.view(np.uint32).astype(np.int64) if unsigned_priority else prio.astype(np.int64)
    order = sorted(range(g.nodes), key=lambda v: (-int(key[v]), -v))
    st = np.zeros(g.nodes, np.int32)
    for v in order:
        nb = g.nlist[g.nindex[v]:g.nindex[v + 1]]
        st[v] = 2 if any(st[u] == 1 for u in nb if u != v) else 1
    return st


def test_mis_priority_matches_oracle():
    vs = np.array([0, 1, 2, 77, 1 << 20, (1 << 31) - 712313888, 2_000_000_000], np.int64)
    got = i2.mis_priority(vs)
    assert [oracle.mis_priority(int(v)) for v in vs] == got.tolist()


@pytest.mark.parametrize("unsigned", [False, True])
def test_mis_oracle_is_the_greedy_set(unsigned):
    for g in (i2.gen_er(300, 900, 2), i2.gen_rmat(9, 8, seed=3), i2.gen_grid(12, 0.1, 0.02, 5)):
        st = oracle.mis(g, unsigned_priority=unsigned)
        np.testing.assert_array_equal(st, _greedy_mis(g, unsigned))
        # independent and maximal
        for v in range(g.nodes):
            nb = [u for u in g.nlist[g.nindex[v]:g.nindex[v + 1]] if u != v]
            if st[v] == 1:
                assert all(st[u] != 1 for u in nb)
            else:
                assert any(st[u] == 1 for u in nb)


def test_mis_certificate_accepts_oracle_and_rejects_planted_mistakes():
    g = i2.gen_rmat(12, 8, seed=4)
    st = oracle.mis(g)
    assert oracle.certify_mis(g, st) is None
    v_in = int(np.flatnonzero((st == 1) & (g.degrees() > 0))[0])
    bad = st.copy()
    bad[g.nlist[g.nindex[v_in]]] = 1  # a neighbour of a vertex in the set
    assert oracle.certify_mis(g, bad) == "adjacent vertices in the set"
    bad = st.copy()
    bad[v_in] = 2  # it has no neighbour in the set
    assert oracle.certify_mis(g, bad) == "set is not maximal"
    bad = st.copy()
    bad[0] = 0
    assert oracle.certify_mis(g, bad) == "undecided vertex"


@pytest.mark.skipif(not oracle.have_ref(), reason="reference programs not built")
def test_mis_oracle_matches_reference_cpu_program():
    # The reference's C++ MIS codes compare priorities as unsigned int; the
    # oracle's unsigned order must give exactly their set. (Its CUDA codes
    # compare them as int: the GPU tests pin that order against one of them.)
    for g in (i2.gen_rmat(14, 16, seed=5), i2.gen_er(20000, 80000, 3), i2.gen_grid(96, 0.05, 0.002, 7),
              i2.gen_rmat(16, 16, seed=2)):
        _, ref = oracle.ref_cpu_run("mis_cpp", g, 0, 4)
        np.testing.assert_array_equal(oracle.mis(g, unsigned_priority=True), ref)
    assert not np.array_equal(oracle.mis(g, unsigned_priority=False), ref)  # the two orders differ


def test_oracle_rmat_generator_equals_engine_generator():
    """oracle.gen_rmat (oracle/graphgen.c) restates the engine's seeded RMAT
    graph independently; the benchmark's reference arm builds its input with it."""
    for scale, seed in ((8, 3), (12, 22), (16, 5)):
        a = oracle.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
        b = i2.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed)
        assert (a.nodes, a.edges) == (b.nodes, b.edges)
        assert np.array_equal(a.nindex, b.nindex)
        assert np.array_equal(a.nlist, b.nlist)
        assert np.array_equal(a.eweight, b.eweight)
    u = oracle.gen_rmat(10, 8, seed=1, weighted=False)
    assert u.eweight is None and u.edges == i2.gen_rmat(10, 8, seed=1, weighted=False).edges


def test_certificates_accept_oracle_results_and_catch_planted_mistakes():
    """The size-independent certificates (oracle/certify.c) used at full size
    accept the oracle's own answers and reject each kind of planted error."""
    g = i2.gen_rmat(14, 16, seed=9)
    src = int(np.argmax(g.degrees()))
    d = oracle.sssp(g, src)
    b = oracle.bfs(g, src)
    assert oracle.certify_distances(g, src, d, weighted=True) is None
    assert oracle.certify_distances(g, src, b, weighted=False) is None
    assert oracle.certify_distances(g, src, d, weighted=False) is not None  # wrong metric
    reached = np.flatnonzero((d != INF) & (np.arange(g.nodes) != src))
    v = int(reached[len(reached) // 2])
    bad = d.copy()
    bad[v] += 1  # too large: an in-edge is relaxable
    assert oracle.certify_distances(g, src, bad, weighted=True) == "relaxable edge"
    bad = d.copy()
    bad[v] -= 1  # too small: no tight in-edge
    assert oracle.certify_distances(g, src, bad, weighted=True) == "reached vertex without a tight in-edge"
    bad = d.copy()
    bad[v] = INF
    assert oracle.certify_distances(g, src, bad, weighted=True) == "unreached neighbour of a reached vertex"
    bad = d.copy()
    bad[src] = 1
    assert oracle.certify_distances(g, src, bad, weighted=True) == "dist[src] != 0"
    lab = oracle.cc(g)
    assert oracle.certify_cc(g, lab) is None
    bad = lab.copy()
    u = int(np.flatnonzero(g.degrees() > 0)[-1])
    bad[u] = u  # splits a component
    assert oracle.certify_cc(g, bad) in ("adjacent labels differ", "label is not its own label")
    # two components merged under one label: the labels are consistent across
    # edges, but the second component is not connected to the label's root
    comps = {}
    for x in range(g.nodes):
        comps.setdefault(int(lab[x]), []).append(x)
    roots = sorted(r for r, m in comps.items() if len(m) > 1)
    if len(roots) < 2:  # an extra edge pair component for the case
        pytest.skip("graph has one non-trivial component")
    r0, r1 = roots[0], roots[1]
    bad = lab.copy()
    bad[np.array(comps[r1])] = r0
    assert oracle.certify_cc(g, bad) == "vertex not connected to its label"
    bad = lab.copy()
    bad[r1] = r1 + 1 if r1 + 1 < g.nodes else r1 - 1
    assert oracle.certify_cc(g, bad) is not None


def test_cc_certificate_on_a_graph_of_many_components():
    g = i2.gen_grid(40, 0.45, 0.0, seed=11)  # many small components
    lab = oracle.cc(g)
    assert len(np.unique(lab)) > 10
    assert oracle.certify_cc(g, lab) is None
    comps = sorted(set(int(x) for x in lab))
    bad = lab.copy()
    bad[lab == comps[-1]] = comps[-2]
    assert oracle.certify_cc(g, bad) == "vertex not connected to its label"
