"""i2_run_noalloc: traversal for callers that cannot allocate device memory.

Such callers (a process whose device memory is held by another allocator, a
query loop that cannot afford cudaMalloc's device synchronisation, a service
that must not fail with out-of-memory at query time) pass the CSR and the
output in device memory; the engine's scratch for this call is a fixed device
array inside the library. These tests call it through the C ABI and check that
it returns exactly what the allocating entry point returns, on two calls in a
row (the second call reuses the scratch the first one left behind).
"""
import ctypes as C

import numpy as np
import pytest

import indigo2suite_b200 as i2
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


def _noalloc(torch, algo, cg, src, nodes):
    out = torch.full((nodes,), -7, dtype=torch.int32, device="cuda")
    iters = C.c_int(-1)
    st = i2.lib.i2_run_noalloc(algo, C.byref(cg), src, C.c_void_p(out.data_ptr()), None, C.byref(iters))
    torch.cuda.synchronize()
    return st, out.cpu().numpy(), iters.value


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
