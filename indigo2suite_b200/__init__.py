"""indigo2suite_b200 — B200 engine for the Indigo2 BFS/SSSP/CC relaxation path.

Python host side of the C ABI in include/i2b200.h. It mirrors the reference's
interface for this path:

* ``ECLGraph`` / ``read_eclgraph`` / ``write_eclgraph``: the CSR layout and file
  format of include/ECLgraph.h:44-106 (nodes, edges, nindex, nlist, eweight).
* ``GPUbfs_vertex``, ``GPUbfs_edge``, ``GPUsssp_vertex``, ``GPUsssp_edge``,
  ``GPUcc_vertex``, ``GPUcc_edge``: same arguments and meaning as the
  reference's per-variant host drivers (include/bfs_vertex_cuda.h:61,
  include/bfs_edge_cuda.h:61, include/sssp_vertex_cuda.h:60,
  include/sssp_edge_cuda.h:60, include/cc_vertex_cuda.h:57,
  include/cc_edge_cuda.h:57): fill ``dist``/``label`` (host int32 arrays of
  ``nodes``) and return the device time in seconds. Errors raise ``I2Error``
  instead of exiting the process.

All compute runs in the CUDA library; nothing here computes results on the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi as capi
from ._capi import (I2_SSSP_BUDGET_AUTO, I2_AUTO_HEURISTIC, I2_AUTO_LEARNED, I2_BFS, I2_CC, I2_LOOP_GRAPH, I2_LOOP_HOST, I2_LOOP_RELAUNCH,
                    I2_MIS, MIS_IN, MIS_OUT,
                    I2_NUM_VARIANTS, I2_SSSP, VARIANTS)

lib = capi.load()

__all__ = [
    "I2Error", "ECLGraph", "DeviceGraph", "Batch", "read_eclgraph", "write_eclgraph", "gen_er", "gen_rmat",
    "gen_grid", "gen_rmat_n", "synth_weights", "build_sp", "VARIANTS", "variant_id", "GPUbfs_vertex", "GPUbfs_edge",
    "GPUsssp_vertex", "GPUsssp_edge", "GPUcc_vertex", "GPUcc_edge", "mlp_param_count", "mlp_loss_grad",
    "mlp_train", "mlp_predict", "mlp_set_params", "device_count", "I2_BFS", "I2_SSSP", "I2_CC", "I2_MIS",
    "MIS_IN", "MIS_OUT", "GPUmis_vertex", "GPUmis_edge", "mis_priority",
    "I2_AUTO_HEURISTIC", "I2_AUTO_LEARNED", "I2_SSSP_BUDGET_AUTO", "I2_NUM_VARIANTS", "I2_LOOP_GRAPH", "I2_LOOP_HOST", "I2_LOOP_RELAUNCH",
]

INF = np.iinfo(np.int32).max


class I2Error(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib.i2_status_string(status).decode()
        super().__init__(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


def _check(status: int, what: str) -> int:
    if status != capi.I2_OK:
        raise I2Error(status, what)
    return status


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def device_count() -> int:
    return int(lib.i2_device_count())


def trim_device_memory() -> None:
    """Hand the device memory that freed graphs left reserved in the engine's
    pool (current device) back to the driver."""
    _check(lib.i2_trim_device_memory(), "trim device memory")


def variant_id(v) -> int:
    if isinstance(v, (int, np.integer)):
        return int(v)
    if v in ("auto", "heuristic", "auto_heuristic"):
        return I2_AUTO_HEURISTIC
    if v in ("learned", "auto_learned"):
        return I2_AUTO_LEARNED
    return VARIANTS.index(v)


@dataclass
class ECLGraph:
    """Host CSR graph (include/ECLgraph.h:44-50). Arrays are int32."""

    nodes: int
    edges: int
    nindex: np.ndarray
    nlist: np.ndarray
    eweight: np.ndarray | None = None
    _keep: list = field(default_factory=list, repr=False)

    def as_c(self) -> capi.EclGraphC:
        for name in ("nindex", "nlist", "eweight"):
            a = getattr(self, name)
            if a is not None and (a.dtype != np.int32 or not a.flags.c_contiguous):
                setattr(self, name, np.ascontiguousarray(a, dtype=np.int32))
        w = self.eweight
        return capi.EclGraphC(self.nodes, self.edges, _iptr(self.nindex), _iptr(self.nlist),
                              _iptr(w) if w is not None else C.POINTER(C.c_int)())

    @classmethod
    def _from_c(cls, cg: capi.EclGraphC) -> "ECLGraph":
        n, e = cg.nodes, cg.edges
        nindex = np.ctypeslib.as_array(cg.nindex, shape=(n + 1,)).copy()
        nlist = np.ctypeslib.as_array(cg.nlist, shape=(e,)).copy() if e else np.zeros(0, np.int32)
        w = None
        if bool(cg.eweight):
            w = np.ctypeslib.as_array(cg.eweight, shape=(e,)).copy() if e else np.zeros(0, np.int32)
        lib.i2_free_eclgraph(C.byref(cg))
        return cls(n, e, nindex, nlist, w)

    def degrees(self) -> np.ndarray:
        return np.diff(self.nindex.astype(np.int64))


def read_eclgraph(path: str) -> ECLGraph:
    cg = capi.EclGraphC()
    _check(lib.i2_read_eclgraph(str(path).encode(), C.byref(cg)), f"read {path}")
    return ECLGraph._from_c(cg)


def write_eclgraph(g: ECLGraph, path: str) -> None:
    cg = g.as_c()
    _check(lib.i2_write_eclgraph(C.byref(cg), str(path).encode()), f"write {path}")


def synth_weights(g: ECLGraph) -> ECLGraph:
    """Reference synthetic SSSP weights (include/sssp_vertex_cuda.h:127-137), computed by the library."""
    w = np.empty(g.edges + 4, np.int32)
    cg = capi.EclGraphC(g.nodes, g.edges, _iptr(g.nindex), _iptr(g.nlist), _iptr(w))
    _check(lib.i2_synth_weights(C.byref(cg)), "synth_weights")
    return ECLGraph(g.nodes, g.edges, g.nindex, g.nlist, w[: g.edges].copy())


def build_sp(g: ECLGraph) -> np.ndarray:
    """Starting-point array of include/bfs_edge_cuda.h:140-146."""
    sp = np.empty(max(g.edges, 1), np.int32)
    cg = g.as_c()
    _check(lib.i2_build_sp(C.byref(cg), _iptr(sp)), "build_sp")
    return sp[: g.edges]


def gen_er(n: int, m: int, seed: int, weighted: bool = True) -> ECLGraph:
    cg = capi.EclGraphC()
    _check(lib.i2_gen_er(n, m, seed, int(weighted), C.byref(cg)), "gen_er")
    return ECLGraph._from_c(cg)


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1, weighted: bool = True) -> ECLGraph:
    cg = capi.EclGraphC()
    _check(lib.i2_gen_rmat(scale, edge_factor, a, b, c, seed, int(weighted), C.byref(cg)), "gen_rmat")
    return ECLGraph._from_c(cg)


def gen_rmat_n(n: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
               seed: int = 1, weighted: bool = True) -> ECLGraph:
    cg = capi.EclGraphC()
    _check(lib.i2_gen_rmat_n(n, edge_factor, a, b, c, seed, int(weighted), C.byref(cg)), "gen_rmat_n")
    return ECLGraph._from_c(cg)


def gen_grid(side: int, remove_frac: float = 0.05, add_frac: float = 0.001, seed: int = 1,
             weighted: bool = True) -> ECLGraph:
    cg = capi.EclGraphC()
    _check(lib.i2_gen_grid(side, remove_frac, add_frac, seed, int(weighted), C.byref(cg)), "gen_grid")
    return ECLGraph._from_c(cg)


@dataclass
class Report:
    seconds: float
    relax_seconds: float
    iterations: int
    variant_hist: list
    reached_vertices: int
    reached_edges: int
    status: int = 0


def _opts(variant, loop, iter_cap, record, stream, delta: int = 0, then_variant=None, then_at: int = 0,
          budget: int = 0) -> capi.Opts:
    """delta: SSSP near/far threshold step for the vp_cta style (<= 0 off, > 0 this step).
    budget: SSSP budgeted near/far ordering for the vp_cta style when delta <= 0 (0 off,
    > 0 frontier edges per near set, I2_SSSP_BUDGET_AUTO the engine's default).
    then_variant/then_at: switch to then_variant from iteration then_at on."""
    tv = variant_id(then_variant) if then_variant is not None else 0
    return capi.Opts(variant_id(variant), int(loop), int(iter_cap), int(record),
                     C.c_void_p(stream) if stream else None, int(delta), int(then_at) if then_variant is not None else 0,
                     tv, int(budget))


def _report(r: capi.Report, status: int) -> Report:
    return Report(r.seconds, r.relax_seconds, r.iterations, list(r.variant_hist)[:I2_NUM_VARIANTS],
                  r.reached_vertices, r.reached_edges, status)


class DeviceGraph:
    """A CSR graph resident in device memory (the reference harness's ``d_g``)."""

    def __init__(self, handle: C.c_void_p, host: ECLGraph | None = None):
        self._h = handle
        self.host = host
        n, e = C.c_int(), C.c_int()
        _check(lib.i2_graph_size(self._h, C.byref(n), C.byref(e)), "graph size")
        self.nodes, self.edges = n.value, e.value

    def degree(self, v: int) -> int:
        d = C.c_int()
        _check(lib.i2_graph_degree(self._h, v, C.byref(d)), "degree")
        return d.value

    @property
    def info(self) -> dict:
        """Graph statistics (the first query also checks symmetry on the device)."""
        info = capi.GraphInfo()
        _check(lib.i2_graph_info_get(self._h, C.byref(info)), "graph info")
        return {k: getattr(info, k) for k, _ in capi.GraphInfo._fields_}

    @classmethod
    def upload(cls, g: ECLGraph) -> "DeviceGraph":
        h = C.c_void_p()
        cg = g.as_c()
        _check(lib.i2_graph_upload(C.byref(cg), C.byref(h)), "graph upload")
        return cls(h, g)

    @classmethod
    def wrap_device(cls, nodes: int, edges: int, nindex_ptr: int, nlist_ptr: int, eweight_ptr: int = 0):
        """Wrap CSR arrays already in device memory (e.g. torch tensors' data_ptr())."""
        cg = capi.EclGraphC(nodes, edges, C.cast(C.c_void_p(nindex_ptr), C.POINTER(C.c_int)),
                            C.cast(C.c_void_p(nlist_ptr), C.POINTER(C.c_int)),
                            C.cast(C.c_void_p(eweight_ptr), C.POINTER(C.c_int)) if eweight_ptr
                            else C.POINTER(C.c_int)())
        h = C.c_void_p()
        _check(lib.i2_graph_wrap_device(C.byref(cg), C.byref(h)), "graph wrap")
        return cls(h)

    @classmethod
    def generate_rmat(cls, scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
                      c: float = 0.19, seed: int = 1, weighted: bool = True) -> "DeviceGraph":
        h = C.c_void_p()
        _check(lib.i2_graph_generate_rmat(scale, edge_factor, a, b, c, seed, int(weighted), C.byref(h)),
               "device rmat")
        return cls(h)

    @classmethod
    def generate_rmat_n(cls, n: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                        seed: int = 1, weighted: bool = True) -> "DeviceGraph":
        """RMAT on n vertices built on the device: the same CSR as gen_rmat_n."""
        h = C.c_void_p()
        _check(lib.i2_graph_generate_rmat_n(n, edge_factor, a, b, c, seed, int(weighted), C.byref(h)),
               "device rmat_n")
        return cls(h)

    @classmethod
    def generate_er(cls, n: int, m: int, seed: int = 1, weighted: bool = True) -> "DeviceGraph":
        """G(n, m) built on the device: the same CSR as gen_er."""
        h = C.c_void_p()
        _check(lib.i2_graph_generate_er(n, m, seed, int(weighted), C.byref(h)), "device er")
        return cls(h)

    @classmethod
    def generate_grid(cls, side: int, remove_frac: float = 0.05, add_frac: float = 0.001, seed: int = 1,
                      weighted: bool = True) -> "DeviceGraph":
        """The grid graph built on the device: the same CSR as gen_grid."""
        h = C.c_void_p()
        _check(lib.i2_graph_generate_grid(side, remove_frac, add_frac, seed, int(weighted), C.byref(h)),
               "device grid")
        return cls(h)

    @classmethod
    def from_coo_device(cls, nodes: int, m: int, src_ptr: int, dst_ptr: int, w_ptr: int = 0,
                        symmetrize: bool = False) -> "DeviceGraph":
        """CSR built on the device from m (src, dst[, w]) pairs already in device
        memory (e.g. torch tensors' data_ptr()): self-loops dropped, duplicates
        merged keeping the smallest weight, adjacency sorted."""
        h = C.c_void_p()
        _check(lib.i2_graph_from_coo_device(nodes, m, C.c_void_p(src_ptr), C.c_void_p(dst_ptr),
                                            C.c_void_p(w_ptr) if w_ptr else None, int(symmetrize), C.byref(h)),
               "coo to csr")
        return cls(h)

    def hub(self) -> int:
        """The highest-degree vertex (lowest ID on ties)."""
        v = C.c_int()
        _check(lib.i2_graph_hub(self._h, C.byref(v)), "hub")
        return v.value

    def sp(self) -> np.ndarray:
        """The starting-point array sp[e] (source vertex of CSR entry e), built on the device."""
        out = np.empty(max(1, self.edges), np.int32)
        dp = C.c_void_p()
        _check(lib.i2_graph_sp(self._h, C.byref(dp), _iptr(out)), "sp")
        return out[: self.edges]

    def download(self) -> ECLGraph:
        cg = capi.EclGraphC()
        _check(lib.i2_graph_download(self._h, C.byref(cg)), "graph download")
        return ECLGraph._from_c(cg)

    def tune(self, heavy_threshold: int = 0, blocks_per_sm: int = 0, smem_carveout: int = -1) -> None:
        _check(lib.i2_graph_tune(self._h, heavy_threshold, blocks_per_sm, smem_carveout), "tune")

    def reorder(self, order: str = "degree") -> None:
        """Run BFS and SSSP on a copy of the graph renumbered by descending
        degree ("degree"), or drop that copy ("none"). Results stay in the
        original IDs and equal the original CSR's."""
        code = {"none": capi.I2_ORDER_NONE, "degree": capi.I2_ORDER_DEGREE}[order]
        _check(lib.i2_graph_reorder(self._h, code), "reorder")

    def synth_weights(self) -> None:
        _check(lib.i2_graph_synth_weights(self._h), "synth weights")

    def free(self) -> None:
        if self._h:
            lib.i2_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # -- traversals ---------------------------------------------------------
    def _run(self, algo: int, src: int, variant, loop, iter_cap, record, stream, out=None, delta=0,
             then_variant=None, then_at=0, budget=0):
        dist = out if out is not None else np.empty(self.nodes, np.int32)
        assert dist.dtype == np.int32 and dist.size >= self.nodes and dist.flags.c_contiguous
        o = _opts(variant, loop, iter_cap, record, stream, delta, then_variant, then_at, budget)
        r = capi.Report()
        if algo == I2_BFS:
            st = lib.i2_bfs(self._h, src, _iptr(dist), C.byref(o), C.byref(r))
        elif algo == I2_SSSP:
            st = lib.i2_sssp(self._h, src, _iptr(dist), C.byref(o), C.byref(r))
        elif algo == I2_CC:
            st = lib.i2_cc(self._h, _iptr(dist), C.byref(o), C.byref(r))
        else:
            st = lib.i2_mis(self._h, _iptr(dist), C.byref(o), C.byref(r))
        if st not in (capi.I2_OK,):
            raise I2Error(st, ["bfs", "sssp", "cc", "mis"][algo])
        return dist, _report(r, st)

    def bfs(self, src: int, variant="vp_cta", loop=I2_LOOP_GRAPH, iter_cap=0, record=False, stream=None, out=None,
            then_variant=None, then_at: int = 0):
        return self._run(I2_BFS, src, variant, loop, iter_cap, record, stream, out, 0, then_variant, then_at)

    def sssp(self, src: int, variant="vp_cta", loop=I2_LOOP_GRAPH, iter_cap=0, record=False, stream=None, out=None,
             delta: int = 0, then_variant=None, then_at: int = 0, budget: int = 0):
        return self._run(I2_SSSP, src, variant, loop, iter_cap, record, stream, out, delta, then_variant, then_at,
                         budget)

    def cc(self, variant="vp_cta", loop=I2_LOOP_GRAPH, iter_cap=0, record=False, stream=None, out=None,
           then_variant=None, then_at: int = 0):
        return self._run(I2_CC, 0, variant, loop, iter_cap, record, stream, out, 0, then_variant, then_at)

    def mis(self, loop=I2_LOOP_GRAPH, iter_cap=0, record=False, stream=None, out=None):
        """Maximal independent set: status per vertex, MIS_IN (1) or MIS_OUT (2)."""
        return self._run(I2_MIS, 0, "vp_warp", loop, iter_cap, record, stream, out)

    def run_device(self, algo: int, src: int = 0, out_ptr: int = 0, variant="vp_cta", loop=I2_LOOP_GRAPH,
                   iter_cap=0, record=False, stream=None, report: bool = True, delta: int = 0,
                   budget: int = 0) -> Report | None:
        """Traversal with the result left in device memory (copied to out_ptr if given).
        With report=False and the graph loop the call is asynchronous on `stream`."""
        o = _opts(variant, loop, iter_cap, record, stream, delta, budget=budget)
        r = capi.Report()
        st = lib.i2_run_device(self._h, algo, src, C.c_void_p(out_ptr) if out_ptr else None, C.byref(o),
                               C.byref(r) if report else None)
        if st != capi.I2_OK:
            raise I2Error(st, "run_device")
        return _report(r, st) if report else None

    def records(self, cap: int = 1 << 16) -> list[dict]:
        buf = (capi.IterRecord * cap)()
        n = C.c_int()
        _check(lib.i2_get_records(self._h, buf, cap, C.byref(n)), "records")
        return [_rec(buf[i]) for i in range(n.value)]

    def sweep(self, algo: int, src: int = 0, follow: int = -1, reps: int = 1, cap: int = 4096):
        """Per-iteration times (ns) of every variant along one trajectory; -1 where not allowed."""
        recs = (capi.IterRecord * cap)()
        times = np.full(cap * I2_NUM_VARIANTS, -1.0, np.float32)
        n = C.c_int()
        _check(lib.i2_sweep(self._h, algo, src, follow, reps, recs, _fptr(times), cap, C.byref(n)), "sweep")
        return [_rec(recs[i]) for i in range(n.value)], times[: n.value * I2_NUM_VARIANTS].reshape(
            n.value, I2_NUM_VARIANTS)


def _rec(r: capi.IterRecord) -> dict:
    return {"iter": r.iter, "variant": r.variant, "size": r.size, "hsize": r.hsize, "edges": r.edges,
            "maxdeg": r.maxdeg, "mindist": r.mindist, "visited": r.visited, "t_ns": r.t_ns, "kind": r.kind,
            "threshold": r.threshold, "pile": r.pile,
            "feat": np.array(list(r.feat), np.float32)}


class Batch:
    """Many graphs traversed together as one disjoint-union CSR: from host
    graphs (ECLGraph, uploaded) or from device graphs (DeviceGraph, copied on
    the device)."""

    def __init__(self, graphs: list):
        self.graphs = graphs
        self._h = C.c_void_p()
        if graphs and isinstance(graphs[0], DeviceGraph):
            arr = (C.c_void_p * len(graphs))(*[g._h for g in graphs])
            _check(lib.i2_batch_from_device(arr, len(graphs), C.byref(self._h)), "batch from device")
        else:
            arr = (capi.EclGraphC * len(graphs))(*[g.as_c() for g in graphs])
            _check(lib.i2_batch_upload(arr, len(graphs), C.byref(self._h)), "batch upload")
        voff = (C.c_longlong * (len(graphs) + 1))()
        _check(lib.i2_batch_offsets(self._h, voff), "batch offsets")
        self.voff = np.array(list(voff), np.int64)
        self.nodes = int(self.voff[-1])

    def run(self, algo: int, srcs=None, variant="vp_cta", loop=I2_LOOP_GRAPH, stream=None):
        dist = np.empty(self.nodes, np.int32)
        o = _opts(variant, loop, 0, 0, stream)
        r = capi.Report()
        s = None
        if algo != I2_CC:
            s = np.ascontiguousarray(srcs, dtype=np.int32)
        st = lib.i2_batch_run(self._h, algo, _iptr(s) if s is not None else None, _iptr(dist), C.byref(o),
                              C.byref(r))
        if st != capi.I2_OK:
            raise I2Error(st, "batch run")
        return [dist[self.voff[k]:self.voff[k + 1]] for k in range(len(self.graphs))], _report(r, st)

    def tune(self, heavy_threshold: int = 0, blocks_per_sm: int = 0, smem_carveout: int = -1) -> None:
        _check(lib.i2_batch_tune(self._h, heavy_threshold, blocks_per_sm, smem_carveout), "batch tune")

    def run_device(self, algo: int, srcs=None, variant="vp_cta", loop=I2_LOOP_GRAPH, stream=None,
                   report: bool = True):
        """Traversal of every graph with results left on the device."""
        o = _opts(variant, loop, 0, 0, stream)
        r = capi.Report()
        self._srcs = np.ascontiguousarray(srcs, dtype=np.int32) if algo != I2_CC else None
        st = lib.i2_batch_run_device(self._h, algo, _iptr(self._srcs) if self._srcs is not None else None,
                                     C.byref(o), C.byref(r) if report else None)
        if st != capi.I2_OK:
            raise I2Error(st, "batch run")
        return _report(r, st) if report else None

    def result(self, stream=None):
        dist = np.empty(self.nodes, np.int32)
        o = _opts("vp_cta", I2_LOOP_GRAPH, 0, 0, stream)
        _check(lib.i2_batch_result(self._h, _iptr(dist), C.byref(o)), "batch result")
        return [dist[self.voff[k]:self.voff[k + 1]] for k in range(len(self.graphs))]

    def free(self):
        if self._h:
            lib.i2_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Reference-interface mirror (include/*_cuda.h). ``g`` is a DeviceGraph, like
# the reference's d_g; dist/label are host int32 arrays of g.nodes.

DEFAULT_VARIANT = I2_AUTO_HEURISTIC


def _mirror(algo, src, g: DeviceGraph, out: np.ndarray, variant) -> float:
    _, rep = g._run(algo, src, DEFAULT_VARIANT if variant is None else variant, I2_LOOP_GRAPH, 0, False, None,
                    out)
    return rep.seconds


def GPUbfs_vertex(src: int, g: DeviceGraph, dist: np.ndarray, variant=None) -> float:
    return _mirror(I2_BFS, src, g, dist, variant)


def GPUbfs_edge(src: int, g: DeviceGraph, dist: np.ndarray, sp: np.ndarray | None = None, variant=None) -> float:
    # sp (the host starting-point array) is accepted for signature parity; the
    # engine builds its own on the device when an edge-centric variant needs it.
    return _mirror(I2_BFS, src, g, dist, "edge_topo" if variant is None else variant)


def GPUsssp_vertex(src: int, g: DeviceGraph, dist: np.ndarray, variant=None) -> float:
    return _mirror(I2_SSSP, src, g, dist, variant)


def GPUsssp_edge(src: int, g: DeviceGraph, dist: np.ndarray, sp: np.ndarray | None = None, variant=None) -> float:
    return _mirror(I2_SSSP, src, g, dist, "vp_cta" if variant is None else variant)


def GPUcc_vertex(g: DeviceGraph, label: np.ndarray, variant=None) -> float:
    return _mirror(I2_CC, 0, g, label, variant)


def GPUcc_edge(g: DeviceGraph, label: np.ndarray, sp: np.ndarray | None = None, variant=None) -> float:
    return _mirror(I2_CC, 0, g, label, "edge_topo" if variant is None else variant)


def mis_priority(v: np.ndarray) -> np.ndarray:
    """Priorities the reference's CUDA MIS codes give vertices (int32)."""
    x = (np.asarray(v, np.uint64) + 712313887) & 0xFFFFFFFF
    for _ in range(2):
        x = (((x >> 16) ^ x) * 0x45D9F3B) & 0xFFFFFFFF
    x = (x >> 16) ^ x
    return x.astype(np.uint32).view(np.int32)


def GPUmis_vertex(g: DeviceGraph, priority: np.ndarray, status: np.ndarray) -> float:
    """Mirror of the reference's GPUmis_vertex(g, priority, status): fills both
    host arrays (priority as the reference computes it) and returns seconds."""
    priority[: g.nodes] = mis_priority(np.arange(g.nodes))
    _, rep = g._run(I2_MIS, 0, "vp_warp", I2_LOOP_GRAPH, 0, False, None, status)
    return rep.seconds


def GPUmis_edge(g: DeviceGraph, sp, priority: np.ndarray, status: np.ndarray) -> float:
    """Mirror of GPUmis_edge(g, sp, priority, status); sp is accepted for
    signature parity (the engine needs none for MIS)."""
    return GPUmis_vertex(g, priority, status)


# ---------------------------------------------------------------------------
# Learned selector.

def mlp_param_count() -> int:
    return int(lib.i2_mlp_param_count())


def mlp_set_params(params: np.ndarray) -> None:
    p = np.ascontiguousarray(params, np.float32)
    _check(lib.i2_mlp_set_params(_fptr(p), p.size), "mlp set params")


def mlp_loss_grad(params, X, T, M):
    p = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    M = np.ascontiguousarray(M, np.float32)
    loss = np.zeros(1, np.float32)
    grad = np.zeros(p.size, np.float32)
    _check(lib.i2_mlp_loss_grad(_fptr(p), _fptr(X), _fptr(T), _fptr(M), X.shape[0], _fptr(loss), _fptr(grad)),
           "mlp loss/grad")
    return float(loss[0]), grad


def mlp_train(params, X, T, M, epochs=200, batch=256, lr=3e-3, seed=1):
    p = np.ascontiguousarray(params, np.float32).copy()
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    M = np.ascontiguousarray(M, np.float32)
    loss = np.zeros(1, np.float32)
    _check(lib.i2_mlp_train(_fptr(p), _fptr(X), _fptr(T), _fptr(M), X.shape[0], epochs, batch, lr, seed,
                            _fptr(loss)), "mlp train")
    return p, float(loss[0])


def mlp_predict(params, X, allowed_mask: int = (1 << I2_NUM_VARIANTS) - 1) -> np.ndarray:
    p = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    out = np.empty(X.shape[0], np.int32)
    _check(lib.i2_mlp_predict(_fptr(p), _fptr(X), X.shape[0], allowed_mask, _iptr(out)), "mlp predict")
    return out
