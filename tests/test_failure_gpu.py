"""Failure handling that faults no GPU: every error is a status code."""
import numpy as np
import pytest

import indigo2suite_b200 as i2
from indigo2suite_b200 import _capi

pytestmark = pytest.mark.gpu


def test_iteration_cap_is_a_status(gpu):
    # a path needs nodes - 1 iterations; cap it at 3
    n = 50
    nindex = np.concatenate([[0], np.cumsum([1] + [2] * (n - 2) + [1])]).astype(np.int32)
    nl = []
    for v in range(n):
        if v > 0:
            nl.append(v - 1)
        if v < n - 1:
            nl.append(v + 1)
    g = i2.ECLGraph(n, len(nl), nindex, np.array(nl, np.int32), np.ones(len(nl), np.int32))
    dg = i2.DeviceGraph.upload(g)
    for loop in (i2.I2_LOOP_GRAPH, i2.I2_LOOP_HOST, i2.I2_LOOP_RELAUNCH):
        with pytest.raises(i2.I2Error) as e:
            dg.bfs(0, iter_cap=3, loop=loop)
        assert e.value.status == _capi.I2_ERR_ITER_CAP
    # the context stays usable
    d, rep = dg.bfs(0)
    assert d[-1] == n - 1 and rep.iterations == n
    dg.free()


def test_bad_arguments(gpu):
    g = i2.gen_er(100, 300, 2)
    dg = i2.DeviceGraph.upload(g)
    for src in (-1, 100):
        with pytest.raises(i2.I2Error) as e:
            dg.bfs(src)
        assert e.value.status == _capi.I2_ERR_ARG
    with pytest.raises(i2.I2Error):
        dg.bfs(0, variant=99)
    dg.free()
    nw = i2.DeviceGraph.upload(i2.ECLGraph(g.nodes, g.edges, g.nindex, g.nlist, None))
    with pytest.raises(i2.I2Error) as e:
        nw.sssp(0)
    assert e.value.status == _capi.I2_ERR_ARG
    nw.synth_weights()  # the reference harness's weights, made on the device
    ref = i2.synth_weights(i2.ECLGraph(g.nodes, g.edges, g.nindex, g.nlist, None))
    np.testing.assert_array_equal(nw.download().eweight, ref.eweight)
    import oracle
    np.testing.assert_array_equal(nw.sssp(0)[0], oracle.sssp(ref, 0))
    nw.free()


def test_malformed_device_graph_rejected_before_any_traversal(gpu):
    import torch

    g = i2.gen_er(64, 128, 3)
    ni = torch.tensor(g.nindex, dtype=torch.int32, device="cuda")
    nl = torch.tensor(g.nlist, dtype=torch.int32, device="cuda")
    ok = i2.DeviceGraph.wrap_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr())
    assert np.array_equal(ok.bfs(0)[0], __import__("oracle").bfs(g, 0))
    ok.free()
    nl[5] = 1000  # out of range
    with pytest.raises(i2.I2Error) as e:
        i2.DeviceGraph.wrap_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr())
    assert e.value.status == _capi.I2_ERR_FORMAT
    nl[5] = 1
    ni[3] = ni[4] + 1  # non-monotone
    with pytest.raises(i2.I2Error) as e:
        i2.DeviceGraph.wrap_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr())
    assert e.value.status == _capi.I2_ERR_FORMAT
    torch.cuda.synchronize()


def test_wrap_refuses_host_pointers(gpu):
    # The reference's BFS/CC harnesses keep d_g.eweight on the host; a host
    # pointer handed over as device memory must be refused, not dereferenced.
    g = i2.gen_er(64, 128, 4)
    with pytest.raises(i2.I2Error) as e:
        i2.DeviceGraph.wrap_device(g.nodes, g.edges, g.nindex.ctypes.data, g.nlist.ctypes.data)
    assert e.value.status == _capi.I2_ERR_ARG
    import torch

    ni = torch.tensor(g.nindex, dtype=torch.int32, device="cuda")
    nl = torch.tensor(g.nlist, dtype=torch.int32, device="cuda")
    with pytest.raises(i2.I2Error) as e:
        i2.DeviceGraph.wrap_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), g.eweight.ctypes.data)
    assert e.value.status == _capi.I2_ERR_ARG
    ok = i2.DeviceGraph.wrap_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr())
    ok.free()


def test_resident_barrier_wait_is_bounded(gpu, monkeypatch):
    # The resident loop's blocks meet at a barrier between iterations. With
    # the first release withheld (a release that nothing gives), every block's
    # wait must run out after the stall limit and the run must end with
    # I2_ERR_STALL, leaving the context usable.
    import time

    g = i2.gen_er(5000, 20000, 4)
    dg = i2.DeviceGraph.upload(g)
    ref, _ = dg.bfs(0, loop=i2.I2_LOOP_HOST)
    monkeypatch.setenv("I2_TEST_HOLD_BARRIER", "1")
    monkeypatch.setenv("I2_STALL_MS", "300")
    for variant in ("vp_cta", "heuristic"):
        t0 = time.perf_counter()
        with pytest.raises(i2.I2Error) as e:
            dg.bfs(0, variant=variant)
        dt = time.perf_counter() - t0
        assert e.value.status == _capi.I2_ERR_STALL
        assert 0.25 < dt < 10.0
    monkeypatch.delenv("I2_TEST_HOLD_BARRIER")
    monkeypatch.delenv("I2_STALL_MS")
    for variant in ("vp_cta", "heuristic"):
        d, _ = dg.bfs(0, variant=variant)
        np.testing.assert_array_equal(d, ref)
    dg.free()


def test_bad_loop_mode_is_refused(gpu):
    g = i2.gen_er(100, 300, 2)
    dg = i2.DeviceGraph.upload(g)
    with pytest.raises(i2.I2Error) as e:
        dg.bfs(0, loop=3)
    assert e.value.status == _capi.I2_ERR_ARG
    dg.free()


def test_malformed_host_graph_rejected_on_upload(gpu):
    # The upload checks the entries on the device after the copy; a malformed
    # CSR must still be refused before any traversal reads it.
    g = i2.gen_er(64, 128, 3)
    nl = g.nlist.copy()
    nl[5] = 1000  # out of range
    with pytest.raises(i2.I2Error) as e:
        i2.DeviceGraph.upload(i2.ECLGraph(g.nodes, g.edges, g.nindex, nl, g.eweight))
    assert e.value.status == _capi.I2_ERR_FORMAT
    ni = g.nindex.copy()
    ni[3] = ni[4] + 1  # non-monotone
    with pytest.raises(i2.I2Error) as e:
        i2.DeviceGraph.upload(i2.ECLGraph(g.nodes, g.edges, ni, g.nlist, g.eweight))
    assert e.value.status == _capi.I2_ERR_FORMAT
    dg = i2.DeviceGraph.upload(g)  # and a good one still works
    assert np.array_equal(dg.bfs(0)[0], __import__("oracle").bfs(g, 0))
    dg.free()
