"""Host side of the library (no GPU): ECLgraph files, generators, C ABI surface."""
import ctypes as C
import os
import re
import tempfile
from pathlib import Path

import numpy as np
import pytest

import indigo2suite_b200 as i2
from indigo2suite_b200 import _capi

ROOT = Path(__file__).resolve().parents[1]


def _is_symmetric_simple(g):
    deg = g.degrees()
    src = np.repeat(np.arange(g.nodes), deg)
    assert (src != g.nlist).all(), "self-loop"
    key = src.astype(np.int64) * g.nodes + g.nlist
    assert len(np.unique(key)) == g.edges, "duplicate"
    rkey = g.nlist.astype(np.int64) * g.nodes + src
    assert np.array_equal(np.sort(key), np.sort(rkey)), "not symmetric"
    for v in range(0, g.nodes, max(1, g.nodes // 97)):
        a = g.nlist[g.nindex[v]:g.nindex[v + 1]]
        assert (np.diff(a) > 0).all(), "unsorted adjacency"
    if g.eweight is not None:
        order = np.argsort(key)
        rorder = np.argsort(rkey)
        assert np.array_equal(g.eweight[order], g.eweight[rorder]), "weights not symmetric"
        assert g.eweight.min() >= 1 and g.eweight.max() <= 255


def test_er_exact_size_and_simple():
    g = i2.gen_er(65536, 262144, 1)
    assert g.nodes == 65536 and g.edges == 524288
    _is_symmetric_simple(g)


def test_generators_are_deterministic_and_seeded():
    a = i2.gen_rmat(11, 16, seed=9)
    b = i2.gen_rmat(11, 16, seed=9)
    c = i2.gen_rmat(11, 16, seed=10)
    assert np.array_equal(a.nlist, b.nlist) and np.array_equal(a.eweight, b.eweight)
    assert not np.array_equal(a.nindex, c.nindex)
    _is_symmetric_simple(a)


def test_rmat_is_skewed_and_dedup_ratio():
    g = i2.gen_rmat(14, 16, seed=1)
    ratio = g.edges / (2 * 16 * g.nodes)
    assert 0.8 < ratio < 0.95
    assert g.degrees().max() > 50 * g.degrees().mean()


def test_grid_shape():
    side = 64
    g = i2.gen_grid(side, 0.05, 0.001, 4)
    _is_symmetric_simple(g)
    full = 2 * 2 * side * (side - 1)
    assert 0.9 * full < g.edges < full
    assert g.degrees().max() <= 8


def test_eclgraph_roundtrip_and_reference_layout(tmp_path):
    g = i2.gen_rmat(8, 4, seed=2)
    p = tmp_path / "g.egr"
    i2.write_eclgraph(g, str(p))
    raw = np.fromfile(p, np.int32)
    assert raw[0] == g.nodes and raw[1] == g.edges
    assert np.array_equal(raw[2:2 + g.nodes + 1], g.nindex)
    assert np.array_equal(raw[3 + g.nodes:3 + g.nodes + g.edges], g.nlist)
    assert np.array_equal(raw[3 + g.nodes + g.edges:], g.eweight)
    h = i2.read_eclgraph(str(p))
    assert np.array_equal(h.nindex, g.nindex) and np.array_equal(h.eweight, g.eweight)
    # without weights: the reader reports none (include/ECLgraph.h:70-76)
    q = tmp_path / "nw.egr"
    i2.write_eclgraph(i2.ECLGraph(g.nodes, g.edges, g.nindex, g.nlist, None), str(q))
    assert i2.read_eclgraph(str(q)).eweight is None


def test_reads_reference_small_inputs(golden):
    for name, case in golden.items():
        g = case["graph"]
        assert g.nindex[0] == 0 and g.nindex[-1] == g.edges


@pytest.mark.parametrize("mutate,status", [
    (lambda raw: raw[:1], _capi.I2_ERR_FORMAT),                       # header truncated
    (lambda raw: raw[:5], _capi.I2_ERR_FORMAT),                       # nindex truncated
    (lambda raw: np.concatenate([raw, raw[-3:-1]]), _capi.I2_ERR_FORMAT),  # partial weights
    (lambda raw: np.concatenate([[0], raw[1:]]), _capi.I2_ERR_FORMAT),     # nodes < 1
    (lambda raw: np.concatenate([raw[:1], [-1], raw[2:]]), _capi.I2_ERR_FORMAT),  # edges < 0
])
def test_malformed_files_are_status_codes(tmp_path, mutate, status):
    g = i2.gen_er(50, 100, 1, weighted=False)
    p = tmp_path / "g.egr"
    i2.write_eclgraph(g, str(p))
    raw = np.fromfile(p, np.int32)
    bad = tmp_path / "bad.egr"
    np.asarray(mutate(raw), np.int32).tofile(bad)
    with pytest.raises(i2.I2Error) as e:
        i2.read_eclgraph(str(bad))
    assert e.value.status == status


def test_out_of_range_neighbour_rejected(tmp_path):
    g = i2.gen_er(50, 100, 1, weighted=False)
    nl = g.nlist.copy()
    nl[3] = g.nodes + 7
    p = tmp_path / "bad.egr"
    i2.write_eclgraph(i2.ECLGraph(g.nodes, g.edges, g.nindex, nl, None), str(p))
    with pytest.raises(i2.I2Error) as e:
        i2.read_eclgraph(str(p))
    assert e.value.status == _capi.I2_ERR_FORMAT
    with pytest.raises(i2.I2Error):
        i2.read_eclgraph(str(tmp_path / "missing.egr"))


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "i2b200.h").read_text()
    names = set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(i2_[a-z0-9_]+)\(", header, re.M))
    assert len(names) >= 35
    lib = C.CDLL(str(ROOT / "indigo2suite_b200" / "libi2b200.so"))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_capi.SIGNATURES) <= names | {"i2_gen_rmat_n"}


def test_status_and_variant_names():
    assert i2.lib.i2_status_string(0) == b"ok"
    assert b"iteration cap" in i2.lib.i2_status_string(_capi.I2_ERR_ITER_CAP)
    assert [i2.lib.i2_variant_name(k).decode() for k in range(i2.I2_NUM_VARIANTS)] == i2.VARIANTS
    assert i2.mlp_param_count() == 16 * 2 + 16 * 64 + 64 + 64 * 64 + 64 + 64 * 9 + 9


def test_upload_without_device_is_a_status_not_a_crash():
    if i2.device_count() > 0:
        pytest.skip("a device is present")
    g = i2.gen_er(100, 200, 1)
    with pytest.raises(i2.I2Error) as e:
        i2.DeviceGraph.upload(g)
    assert e.value.status == _capi.I2_ERR_NO_DEVICE


def test_autotune_candidates_and_table():
    from indigo2suite_b200 import autotune

    cands = list(autotune.candidates())
    assert len(cands) == len(set(cands))
    assert {c[0] for c in cands} == set(autotune.STYLES)
    assert {c[1] for c in cands} == set(autotune.BLOCKS_PER_SM)
    # the heavy threshold is swept only where it matters
    assert {c[2] for c in cands if c[0] == "vp_cta"} == {4096}
    assert {c[2] for c in cands if c[0] == "vp_thread"} == set(autotune.HEAVY)
    assert autotune.load("/nonexistent/table.json") is None
    if autotune.TABLE_PATH.exists():
        t = autotune.load()
        assert t["style"] in autotune.STYLES and t["blocks_per_sm"] in autotune.BLOCKS_PER_SM
        # the committed table covers every candidate and chose the fastest
        import json
        table = json.loads(autotune.TABLE_PATH.read_text())
        rows = table["candidates"]
        assert {(r["style"], r["blocks_per_sm"], r["heavy_threshold"]) for r in rows} == set(cands)
        best = min(rows, key=lambda r: r["total_ms"])
        assert (best["style"], best["blocks_per_sm"], best["heavy_threshold"]) == \
            (t["style"], t["blocks_per_sm"], t["heavy_threshold"])


def test_trim_without_device_is_a_status():
    if i2.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(i2.I2Error) as e:
        i2.trim_device_memory()
    assert e.value.status == _capi.I2_ERR_NO_DEVICE


def test_noalloc_argument_checks_come_before_any_device_work():
    """i2_run_noalloc refuses bad arguments with a status before it touches a
    device (so these hold on a machine without one)."""
    P = C.POINTER(C.c_int)
    out = C.c_void_p(0x1000)
    g = _capi.EclGraphC(10, 0, C.cast(C.c_void_p(0x1000), P), P(), P())
    assert i2.lib.i2_run_noalloc(i2.I2_BFS, None, 0, out, None, None) == _capi.I2_ERR_ARG
    assert i2.lib.i2_run_noalloc(i2.I2_BFS, C.byref(g), 0, None, None, None) == _capi.I2_ERR_ARG
    assert i2.lib.i2_run_noalloc(7, C.byref(g), 0, out, None, None) == _capi.I2_ERR_ARG
    assert i2.lib.i2_run_noalloc(i2.I2_BFS, C.byref(g), 10, out, None, None) == _capi.I2_ERR_ARG
    assert i2.lib.i2_run_noalloc(i2.I2_SSSP, C.byref(g), 0, out, None, None) == _capi.I2_ERR_ARG  # no weights
    big = _capi.EclGraphC((1 << 17) + 1, 0, C.cast(C.c_void_p(0x1000), P), P(), P())
    assert i2.lib.i2_run_noalloc(i2.I2_BFS, C.byref(big), 0, out, None, None) == _capi.I2_ERR_CAPACITY


def test_traversal_tuning_table_lookup(tmp_path):
    """Single traversals are tuned by shape: degree class and nearest size
    class of the same algorithm; unknown shapes keep the defaults."""
    import json

    from indigo2suite_b200 import autotune

    assert autotune.degree_class({"degcv": 3.0, "avgdeg": 30.0}) == "skewed"
    assert autotune.degree_class({"degcv": 0.3, "avgdeg": 8.0}) == "uniform"
    assert autotune.degree_class({"degcv": 0.2, "avgdeg": 3.8}) == "sparse"
    assert autotune.size_class(1 << 22) == 22 and autotune.size_class(3_000_000) == 22
    assert autotune.size_class(1 << 19) in (18, 20)
    assert {b for _, b in autotune.traversal_candidates("sssp")} == set(autotune.TUNE_BUDGETS)
    assert {b for _, b in autotune.traversal_candidates("bfs")} == {0}
    t = {"rows": [{"graph": "rmat18", "class": "skewed", "log2v": 18, "algo": "sssp", "blocks_per_sm": 4,
                   "budget": 1 << 20},
                  {"graph": "rmat22", "class": "skewed", "log2v": 22, "algo": "sssp", "blocks_per_sm": 8,
                   "budget": 1 << 22}]}
    p = tmp_path / "t.json"
    p.write_text(json.dumps(t))
    info = {"degcv": 4.0, "avgdeg": 30.0, "nodes": 1 << 21}
    assert autotune.lookup(info, "sssp", p)["budget"] == 1 << 22  # size 22 is the nearest class
    assert autotune.lookup(dict(info, nodes=1 << 17), "sssp", p)["budget"] == 1 << 20
    assert autotune.lookup(dict(info, degcv=0.1), "sssp", p) is None
    assert autotune.lookup(info, "bfs", p) is None
    assert autotune.lookup(info, "sssp", tmp_path / "missing.json") is None
    if autotune.TRAVERSAL_TABLE.exists():
        table = json.loads(autotune.TRAVERSAL_TABLE.read_text())
        assert len(table["rows"]) > 1
        for r in table["rows"]:  # every committed choice is its row's fastest candidate
            best = min(r["candidates"], key=lambda c: c["ms"])
            assert (best["blocks_per_sm"], best["budget"]) == (r["blocks_per_sm"], r["budget"])
        # and it measurably beats the default on at least one shape
        assert any(r["ms"] < 0.9 * r["default_ms"] for r in table["rows"])


def test_selector_parameters_match_their_recorded_training():
    """The committed parameters name the command and sweep that made them, and
    the committed sweep is the one whose hash they record."""
    import hashlib
    import json

    from indigo2suite_b200 import selector as S

    meta = json.loads(S.PARAMS_PATH.with_suffix(".json").read_text())
    p = np.fromfile(S.PARAMS_PATH, np.float32)
    assert p.size == i2.mlp_param_count()
    assert hashlib.sha256(p.tobytes()).hexdigest() == meta["params_sha256"]
    z = np.load(S.PARAMS_PATH.with_name("selector_sweep.npz"))
    assert z["X"].shape == (meta["rows"], 16)
    h = hashlib.sha256(z["X"].tobytes() + z["T"].tobytes() + z["M"].tobytes()).hexdigest()
    assert h == meta["sweep_sha256"]
    assert "selector train" in meta["command"] and "--data" in meta["command"]
