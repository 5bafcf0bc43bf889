"""Maximal independent set on the GPU: the engine against the oracle (the
greedy set in the reference CUDA codes' priority order) and against the
reference's own CUDA MIS variant, in every loop mode."""
import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle

pytestmark = pytest.mark.gpu


def _graphs():
    return {
        "er": i2.gen_er(20000, 80000, 3),
        "rmat14": i2.gen_rmat(14, 16, seed=5),
        "grid": i2.gen_grid(96, 0.05, 0.002, 7),
        "rmat18": i2.gen_rmat(18, 16, seed=2),
    }


@pytest.mark.parametrize("name", ["er", "rmat14", "grid", "rmat18"])
def test_mis_matches_oracle_every_loop(gpu, name):
    g = _graphs()[name]
    ref = oracle.mis(g)
    dg = i2.DeviceGraph.upload(g)
    for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_HOST, i2.I2_LOOP_RELAUNCH):
        for _ in range(2):
            st, rep = dg.mis(loop=loop)
            np.testing.assert_array_equal(st, ref, err_msg=f"{name} loop {loop}")
            assert rep.iterations >= 1
    dg.free()


def test_mis_golden_graphs(gpu, golden):
    for name, case in golden.items():
        g = case["graph"]
        dg = i2.DeviceGraph.upload(g)
        np.testing.assert_array_equal(dg.mis()[0], oracle.mis(g), err_msg=name)
        dg.free()


@pytest.mark.skipif(not oracle.have_ref(), reason="oracle/_ref not built")
def test_mis_matches_reference_cuda_variant(gpu):
    for name, g in _graphs().items():
        ref = oracle.ref_cuda_mis(g)
        np.testing.assert_array_equal(oracle.mis(g), ref, err_msg=f"oracle vs reference CUDA, {name}")
        dg = i2.DeviceGraph.upload(g)
        np.testing.assert_array_equal(dg.mis()[0], ref, err_msg=f"engine vs reference CUDA, {name}")
        dg.free()


def test_mis_edge_cases_and_refusals(gpu):
    # no edges: every vertex is in the set
    g0 = i2.ECLGraph(50, 0, np.zeros(51, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    dg = i2.DeviceGraph.upload(g0)
    assert (dg.mis()[0] == i2.MIS_IN).all()
    dg.free()
    # a directed graph is refused
    gd = i2.ECLGraph(3, 2, np.array([0, 1, 2, 2], np.int32), np.array([1, 2], np.int32), np.ones(2, np.int32))
    dg = i2.DeviceGraph.upload(gd)
    with pytest.raises(i2.I2Error) as e:
        dg.mis()
    assert e.value.status == i2._capi.I2_ERR_UNSUPPORTED
    dg.free()
    # the reference-interface mirror fills status and priority
    g = _graphs()["grid"]
    dg = i2.DeviceGraph.upload(g)
    prio = np.zeros(g.nodes, np.int32)
    st = np.zeros(g.nodes, np.int32)
    assert i2.GPUmis_vertex(dg, prio, st) > 0
    np.testing.assert_array_equal(st, oracle.mis(g))
    np.testing.assert_array_equal(prio, [oracle.mis_priority(v) for v in range(g.nodes)])
    dg.free()
