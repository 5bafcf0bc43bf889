"""i2_run_noalloc: traversal for callers that cannot allocate device memory.

Such callers (a process whose device memory is held by another allocator, a
query loop that cannot afford cudaMalloc's device synchronisation, a service
that must not fail with out-of-memory at query time) pass the CSR and the
output in device memory; the engine's scratch for this call is a fixed device
array inside the library. These tests call it through the C ABI and check that
it returns exactly what the allocating entry point returns, on two calls in a
row (the second call reuses the scratch the first one left behind), and what
the oracle returns: after a larger graph has filled the scratch, on a directed
graph, from a source without edges, and on a caller's stream.
"""
import ctypes as C

import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle
from indigo2suite_b200 import _capi

pytestmark = pytest.mark.gpu

MAX_NODES = 1 << 17


def _device_csr(torch, g):
    ni = torch.tensor(g.nindex, dtype=torch.int32, device="cuda")
    nl = torch.tensor(g.nlist, dtype=torch.int32, device="cuda")
    w = torch.tensor(g.eweight, dtype=torch.int32, device="cuda")
    P = C.POINTER(C.c_int)
    cg = _capi.EclGraphC(g.nodes, g.edges, C.cast(C.c_void_p(ni.data_ptr()), P),
                         C.cast(C.c_void_p(nl.data_ptr()), P), C.cast(C.c_void_p(w.data_ptr()), P))
    return cg, (ni, nl, w)


def _noalloc(torch, algo, cg, src, nodes, stream=None):
    out = torch.full((nodes,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    iters = C.c_int(-1)
    sp = C.c_void_p(stream.cuda_stream) if stream is not None else None
    st = i2.lib.i2_run_noalloc(algo, C.byref(cg), src, C.c_void_p(out.data_ptr()), sp, C.byref(iters))
    torch.cuda.synchronize()
    return st, out.cpu().numpy(), iters.value


def _oracle(algo, g, src):
    return {i2.I2_BFS: lambda: oracle.bfs(g, src), i2.I2_SSSP: lambda: oracle.sssp(g, src),
            i2.I2_CC: lambda: oracle.cc(g)}[algo]()


def test_noalloc_matches_allocating_entry_point_twice(gpu):
    import torch

    graphs = [i2.gen_rmat(14, 16, seed=41), i2.gen_er(MAX_NODES, 4 * MAX_NODES, 42), i2.gen_grid(200, 0.05, 0.01, 43)]
    for g in graphs:
        cg, keep = _device_csr(torch, g)
        dg = i2.DeviceGraph.upload(g)
        src = int(np.argmax(g.degrees()))
        for algo in (i2.I2_BFS, i2.I2_SSSP, i2.I2_CC):
            ref, _ = dg._run(algo, src, "vp_cta", i2.I2_LOOP_GRAPH, 0, False, None, None)
            for call in range(2):
                st, got, iters = _noalloc(torch, algo, cg, src, g.nodes)
                assert st == _capi.I2_OK, i2.lib.i2_status_string(st)
                np.testing.assert_array_equal(got, ref, err_msg=f"algo {algo} call {call}")
                assert iters > 0
        dg.free()
        del keep


def test_noalloc_refuses_graphs_above_its_scratch(gpu):
    import torch

    g = i2.gen_er(MAX_NODES + 1, 3 * MAX_NODES, 44)
    cg, keep = _device_csr(torch, g)
    st, _, _ = _noalloc(torch, i2.I2_BFS, cg, 0, g.nodes)
    assert st == _capi.I2_ERR_CAPACITY
    assert b"fixed scratch" in i2.lib.i2_status_string(st)
    del keep


def test_noalloc_small_graph_after_large_one_matches_oracle(gpu):
    """A graph at the scratch's limit leaves its frontier lists and bitmaps
    behind; a small graph run next must not see any of it."""
    import torch

    big = i2.gen_er(MAX_NODES, 4 * MAX_NODES, 45)
    small = i2.gen_rmat(10, 8, seed=46)
    for g in (big, small, big, small):
        cg, keep = _device_csr(torch, g)
        src = int(np.argmax(g.degrees()))
        for algo in (i2.I2_BFS, i2.I2_SSSP, i2.I2_CC):
            st, got, _ = _noalloc(torch, algo, cg, src, g.nodes)
            assert st == _capi.I2_OK, i2.lib.i2_status_string(st)
            np.testing.assert_array_equal(got, _oracle(algo, g, src), err_msg=f"algo {algo} n {g.nodes}")
        del keep


def test_noalloc_directed_graph_isolated_source_and_caller_stream(gpu):
    import torch

    full = i2.gen_rmat(12, 8, seed=47)
    # directed: keep each undirected edge in one direction only (u < v)
    deg = np.diff(full.nindex)
    u = np.repeat(np.arange(full.nodes, dtype=np.int32), deg)
    keep_e = u < full.nlist
    nl = np.ascontiguousarray(full.nlist[keep_e])
    w = np.ascontiguousarray(full.eweight[keep_e])
    ni = np.zeros(full.nodes + 1, np.int32)
    np.cumsum(np.bincount(u[keep_e], minlength=full.nodes), out=ni[1:])
    g = i2.ECLGraph(full.nodes, int(nl.size), ni, nl, w)
    stream = torch.cuda.Stream()
    cg, keep = _device_csr(torch, g)
    srcs = [int(np.argmax(np.diff(ni)))]
    isolated = np.flatnonzero(np.diff(ni) == 0)
    assert isolated.size > 0
    srcs.append(int(isolated[0]))
    for src in srcs:
        for algo in (i2.I2_BFS, i2.I2_SSSP, i2.I2_CC):
            for _ in range(2):
                st, got, _ = _noalloc(torch, algo, cg, src, g.nodes, stream)
                assert st == _capi.I2_OK, i2.lib.i2_status_string(st)
                np.testing.assert_array_equal(got, _oracle(algo, g, src), err_msg=f"algo {algo} src {src}")
    del keep


def test_noalloc_refuses_negative_weights_like_i2_sssp(gpu):
    import torch

    g = i2.gen_rmat(10, 8, seed=48)
    g.eweight[5] = -3
    cg, keep = _device_csr(torch, g)
    st, _, _ = _noalloc(torch, i2.I2_SSSP, cg, 0, g.nodes)
    assert st == _capi.I2_ERR_UNSUPPORTED
    dg = i2.DeviceGraph.upload(g)
    with pytest.raises(i2.I2Error) as e:
        dg.sssp(0)
    assert e.value.status == _capi.I2_ERR_UNSUPPORTED
    dg.free()
    # BFS ignores weights
    st, got, _ = _noalloc(torch, i2.I2_BFS, cg, 0, g.nodes)
    assert st == _capi.I2_OK
    np.testing.assert_array_equal(got, oracle.bfs(g, 0))
    del keep
