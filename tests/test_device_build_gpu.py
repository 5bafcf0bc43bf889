"""Graphs built on the device: the seeded ER, grid and RMAT-on-n-vertices
generators give the very CSR the host generators give; the COO-to-CSR entry
point equals a host restatement (symmetrise, drop self-loops, merge duplicates
keeping the smallest weight, sort); a batch assembled from device graphs equals
the batch uploaded from host graphs, with the same traversal results; and the
device-built sp[] equals the oracle's."""
import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle
from indigo2suite_b200 import workloads

pytestmark = pytest.mark.gpu


def _same(dg, h, what):
    d = dg.download()
    assert (d.nodes, d.edges) == (h.nodes, h.edges), what
    np.testing.assert_array_equal(d.nindex, h.nindex, err_msg=what)
    np.testing.assert_array_equal(d.nlist, h.nlist, err_msg=what)
    if h.eweight is None:
        assert d.eweight is None, what
    else:
        np.testing.assert_array_equal(d.eweight, h.eweight, err_msg=what)


@pytest.mark.parametrize("n,m,seed,weighted", [(2, 1, 1, True), (1000, 4000, 7, True), (65536, 262144, 1, True),
                                               (100, 3000, 3, False), (300000, 1200000, 9, True)])
def test_device_er_equals_host(gpu, n, m, seed, weighted):
    dg = i2.DeviceGraph.generate_er(n, m, seed, weighted)
    _same(dg, i2.gen_er(n, m, seed, weighted), f"er {n} {m}")
    dg.free()


def test_device_er_refuses_what_the_host_refuses(gpu):
    # all 4950 pairs of 100 vertices are not drawn within the candidate limit
    for make in (lambda: i2.gen_er(100, 4950, 3, False), lambda: i2.DeviceGraph.generate_er(100, 4950, 3, False)):
        with pytest.raises(i2.I2Error) as e:
            make()
        assert e.value.status == i2._capi.I2_ERR_ARG


@pytest.mark.parametrize("side,rem,add,seed", [(2, 0.0, 0.0, 1), (32, 0.05, 0.01, 5), (300, 0.05, 0.001, 3),
                                               (1024, 0.3, 0.02, 11)])
def test_device_grid_equals_host(gpu, side, rem, add, seed):
    dg = i2.DeviceGraph.generate_grid(side, rem, add, seed)
    _same(dg, i2.gen_grid(side, rem, add, seed), f"grid {side}")
    dg.free()


@pytest.mark.parametrize("n,seed", [(1000, 3), (12345, 5), (300000, 8)])
def test_device_rmat_n_equals_host(gpu, n, seed):
    dg = i2.DeviceGraph.generate_rmat_n(n, 16, 0.57, 0.19, 0.19, seed=seed)
    _same(dg, i2.gen_rmat_n(n, 16, 0.57, 0.19, 0.19, seed=seed), f"rmat_n {n}")
    dg.free()


def _host_coo_csr(n, src, dst, w, sym):
    u, v = np.asarray(src, np.int64), np.asarray(dst, np.int64)
    ww = np.asarray(w, np.int64) if w is not None else np.zeros(len(u), np.int64)
    if sym:
        u, v, ww = np.concatenate([u, v]), np.concatenate([v, u]), np.concatenate([ww, ww])
    keep = u != v
    u, v, ww = u[keep], v[keep], ww[keep]
    order = np.lexsort((ww, v, u))  # by (u, v), smallest weight first
    u, v, ww = u[order], v[order], ww[order]
    first = np.ones(len(u), bool)
    first[1:] = (u[1:] != u[:-1]) | (v[1:] != v[:-1])
    u, v, ww = u[first], v[first], ww[first]
    nindex = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(u, minlength=n), out=nindex[1:])
    return nindex.astype(np.int32), v.astype(np.int32), (ww.astype(np.int32) if w is not None else None)


@pytest.mark.parametrize("sym", [False, True])
@pytest.mark.parametrize("weighted", [False, True])
def test_coo_to_csr_on_device(gpu, sym, weighted):
    import torch

    rng = np.random.default_rng(5 + 2 * sym + weighted)
    n, m = 5000, 60000
    src = rng.integers(0, n, m).astype(np.int32)
    dst = rng.integers(0, n, m).astype(np.int32)
    dst[:50] = src[:50]  # self-loops
    src[100:200], dst[100:200] = src[200:300], dst[200:300]  # duplicates
    w = rng.integers(1, 256, m).astype(np.int32) if weighted else None
    ts, td = torch.tensor(src, device="cuda"), torch.tensor(dst, device="cuda")
    tw = torch.tensor(w, device="cuda") if weighted else None
    dg = i2.DeviceGraph.from_coo_device(n, m, ts.data_ptr(), td.data_ptr(), tw.data_ptr() if weighted else 0, sym)
    ni, nl, ew = _host_coo_csr(n, src, dst, w, sym)
    d = dg.download()
    np.testing.assert_array_equal(d.nindex, ni)
    np.testing.assert_array_equal(d.nlist, nl)
    if weighted:
        np.testing.assert_array_equal(d.eweight, ew)
    if sym and weighted:  # a usable SSSP input: bit-exact with the oracle
        s = int(np.argmax(np.diff(ni)))
        np.testing.assert_array_equal(dg.sssp(s)[0], oracle.sssp(d, s))
    dg.free()
    bad = torch.tensor(np.array([0, n], np.int32), device="cuda")
    with pytest.raises(i2.I2Error) as e:
        i2.DeviceGraph.from_coo_device(n, 2, bad.data_ptr(), bad.data_ptr())
    assert e.value.status == i2._capi.I2_ERR_FORMAT


def test_device_batch_equals_uploaded_batch_and_sp(gpu):
    specs = workloads.batch_specs(24, seed=31, nmin=1e3, nmax=1e5)
    host = [workloads.build(x) for x in specs]
    dev = [workloads.build_device(x) for x in specs]
    for h, d in zip(host, dev):
        _same(d, h, "batch member")
        assert d.hub() == workloads.source(h)
    bh, bd = i2.Batch(host), i2.Batch(dev)
    np.testing.assert_array_equal(bh.voff, bd.voff)
    srcs = [workloads.source(h) for h in host]
    for algo in (i2.I2_BFS, i2.I2_SSSP, i2.I2_CC):
        rh, _ = bh.run(algo, srcs)
        rd, _ = bd.run(algo, srcs)
        for k in range(len(specs)):
            np.testing.assert_array_equal(rh[k], rd[k])
    np.testing.assert_array_equal(dev[3].sp(), oracle.sp(host[3]))
    bh.free()
    bd.free()
    for d in dev:
        d.free()
