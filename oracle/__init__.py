"""ORACLE — test infrastructure only.

Checker for the engine's results: ctypes access to the C restatement in
oracle.c (liboracle.so) and helpers that run the reference's own programs built
by oracle/Makefile into oracle/_ref/ (the reference's serial Dijkstra, its
OpenMP harness used as a verifier of injected results, its CPU programs and a
few of its CUDA programs). Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg may use this package; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"

_lib = None


def build(ref: bool = True) -> None:
    """Build liboracle.so, and the _ref/ programs when the reference tree is present."""
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-j", str(min(16, os.cpu_count() or 1)), "-C", str(HERE), target], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build(ref=False)
        _lib = C.CDLL(str(path))
        P = C.POINTER(C.c_int)
        _lib.oracle_bfs.argtypes = [C.c_int, P, P, C.c_int, P]
        _lib.oracle_sssp.argtypes = [C.c_int, P, P, P, C.c_int, P]
        _lib.oracle_cc_minlabel.argtypes = [C.c_int, P, P, P]
        _lib.oracle_cc_check.argtypes = [C.c_int, P, P, P]
        _lib.oracle_synth_weights.argtypes = [C.c_int, P, P, P]
        _lib.oracle_sp.argtypes = [C.c_int, P, P]
        _lib.oracle_mis.argtypes = [C.c_int, P, P, C.c_int, P]
        _lib.oracle_mis_priority.argtypes = [C.c_int]
        _lib.oracle_synth_weights.restype = None
        _lib.oracle_sp.restype = None
        PP = C.POINTER(P)
        _lib.oracle_gen_rmat.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                         C.c_int, P, P, PP, PP, PP]
        _lib.oracle_graph_free.argtypes = [P, P, P]
        _lib.oracle_graph_free.restype = None
        _lib.oracle_certify_distances.argtypes = [C.c_int, P, P, P, C.c_int, P]
        _lib.oracle_certify_cc.argtypes = [C.c_int, P, P, P]
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _csr(g):
    return np.ascontiguousarray(g.nindex, np.int32), np.ascontiguousarray(g.nlist, np.int32)


class Graph:
    """A host CSR in the ECLgraph layout (nodes, edges, nindex, nlist, eweight)."""

    def __init__(self, nodes: int, edges: int, nindex: np.ndarray, nlist: np.ndarray, eweight):
        self.nodes, self.edges = nodes, edges
        self.nindex, self.nlist, self.eweight = nindex, nlist, eweight

    def degrees(self) -> np.ndarray:
        return np.diff(self.nindex)


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1, weighted: bool = True) -> Graph:
    """The seeded RMAT graph of graphgen.c (the same CSR as the engine's host
    and device RMAT generators, built without the engine library)."""
    P = C.POINTER(C.c_int)
    n, e = C.c_int(), C.c_int()
    ni, nl, ew = P(), P(), P()
    rc = lib().oracle_gen_rmat(scale, edge_factor, a, b, c, seed, int(weighted), C.byref(n), C.byref(e),
                               C.byref(ni), C.byref(nl), C.byref(ew))
    if rc != 0:
        raise ValueError(f"oracle_gen_rmat failed ({rc})")
    try:
        nindex = np.ctypeslib.as_array(ni, (n.value + 1,)).copy()
        nlist = np.ctypeslib.as_array(nl, (e.value,)).copy() if e.value else np.zeros(0, np.int32)
        eweight = (np.ctypeslib.as_array(ew, (e.value,)).copy() if e.value else np.zeros(0, np.int32)) \
            if weighted else None
    finally:
        lib().oracle_graph_free(ni, nl, ew)
    return Graph(n.value, e.value, nindex, nlist, eweight)


def bfs(g, src: int) -> np.ndarray:
    ni, nl = _csr(g)
    out = np.empty(g.nodes, np.int32)
    rc = lib().oracle_bfs(g.nodes, _p(ni), _p(nl), src, _p(out))
    assert rc == 0, rc
    return out


def sssp(g, src: int) -> np.ndarray:
    ni, nl = _csr(g)
    w = np.ascontiguousarray(g.eweight, np.int32)
    out = np.empty(g.nodes, np.int32)
    rc = lib().oracle_sssp(g.nodes, _p(ni), _p(nl), _p(w), src, _p(out))
    assert rc == 0, rc
    return out


def cc(g) -> np.ndarray:
    ni, nl = _csr(g)
    out = np.empty(g.nodes, np.int32)
    rc = lib().oracle_cc_minlabel(g.nodes, _p(ni), _p(nl), _p(out))
    assert rc == 0, rc
    return out


def mis(g, unsigned_priority: bool = False) -> np.ndarray:
    """Status per vertex: 1 in the maximal independent set, 2 excluded. The
    reference's CUDA MIS codes compare priorities as int (the default here),
    its CPU codes as unsigned int."""
    ni, nl = _csr(g)
    out = np.empty(g.nodes, np.int32)
    rc = lib().oracle_mis(g.nodes, _p(ni), _p(nl), int(unsigned_priority), _p(out))
    assert rc == 0, rc
    return out


def ref_cuda_mis(g) -> np.ndarray:
    """The status array of the reference's CUDA MIS variant
    (MIS_CUDA_V_Data_Pull_Determ_..._Thread.cu via _ref/libref_cuda_mis.so);
    needs a GPU."""
    L = C.CDLL(str(REF_OUT / "libref_cuda_mis.so"))
    P = C.POINTER(C.c_int)
    L.ref_cuda_mis.argtypes = [C.c_int, C.c_int, P, P, P]
    L.ref_cuda_mis.restype = C.c_double
    ni, nl = _csr(g)
    out = np.empty(g.nodes, np.int32)
    import sys

    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)  # the reference driver prints its iteration count
    try:
        t = L.ref_cuda_mis(g.nodes, g.edges, _p(ni), _p(nl), _p(out))
        C.CDLL(None).fflush(None)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    if t < 0:
        raise RuntimeError("reference CUDA MIS could not allocate")
    return out


def mis_priority(v: int) -> int:
    return int(lib().oracle_mis_priority(int(v)))


def cc_check(g, label: np.ndarray) -> int:
    ni, nl = _csr(g)
    return int(lib().oracle_cc_check(g.nodes, _p(ni), _p(nl), _p(np.ascontiguousarray(label, np.int32))))


def synth_weights(g) -> np.ndarray:
    ni, nl = _csr(g)
    w = np.empty(max(g.edges, 1), np.int32)
    lib().oracle_synth_weights(g.nodes, _p(ni), _p(nl), _p(w))
    return w[: g.edges]


def sp(g) -> np.ndarray:
    ni, _ = _csr(g)
    out = np.empty(max(g.edges, 1), np.int32)
    lib().oracle_sp(g.nodes, _p(ni), _p(out))
    return out[: g.edges]


# ---------------------------------------------------------------------------
# The reference's own programs (oracle/_ref).

def have_ref() -> bool:
    return (REF_OUT / "libref_serial_bfs.so").exists()


_serial = {}


def ref_serial(kind: str, g, src: int) -> np.ndarray:
    """The reference's CPUserialDijkstra from harness `kind` in {bfs, sssp_vertex, sssp_edge}."""
    if kind not in _serial:
        L = C.CDLL(str(REF_OUT / f"libref_serial_{kind}.so"))
        P = C.POINTER(C.c_int)
        L.ref_serial.argtypes = [C.c_int, C.c_int, P, P, P, C.c_int, P]
        _serial[kind] = L
    ni, nl = _csr(g)
    w = np.ascontiguousarray(g.eweight, np.int32) if g.eweight is not None else None
    out = np.empty(g.nodes, np.int32)
    _serial[kind].ref_serial(g.nodes, g.edges, _p(ni), _p(nl), _p(w) if w is not None else None, src, _p(out))
    return out


def write_egr(g, path: str) -> None:
    """ECLgraph file (include/ECLgraph.h:82-96 layout), written by numpy."""
    with open(path, "wb") as f:
        np.array([g.nodes, g.edges], np.int32).tofile(f)
        np.ascontiguousarray(g.nindex, np.int32).tofile(f)
        np.ascontiguousarray(g.nlist, np.int32).tofile(f)
        if g.eweight is not None:
            np.ascontiguousarray(g.eweight, np.int32).tofile(f)


def ref_verify(kind: str, egr_path: str, values: np.ndarray, src: int | None = 0, timeout: float = 600) -> tuple[bool, str]:
    """Run the reference harness `inject_<kind>` on the graph file with `values`
    as the variant's result; True when the reference verifier passes."""
    exe = REF_OUT / f"inject_{kind}"
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        np.ascontiguousarray(values, np.int32).tofile(f)
        rpath = f.name
    try:
        args = [str(exe), str(egr_path)] + ([str(src)] if src is not None else []) + ["1"]
        env = dict(os.environ, I2_RESULT=rpath, OMP_NUM_THREADS="1")
        p = subprocess.run(args, capture_output=True, text=True, env=env, timeout=timeout)
        out = p.stdout + p.stderr
        return (p.returncode == 0 and "verification passed" in out), out
    finally:
        os.unlink(rpath)


def run_ref_program(name: str, args: list[str], threads: int | None = None, timeout: float = 900) -> dict:
    """Run a reference program from _ref/ and parse its printed runtime/throughput."""
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    p = subprocess.run([str(REF_OUT / name), *args], capture_output=True, text=True, env=env, timeout=timeout)
    out = p.stdout + p.stderr
    rt = re.findall(r"runtime:\s*([0-9.eE+-]+)\s*s", out)
    tp = re.findall(r"Throughput:\s*([0-9.eE+-]+)\s*gigaedges/s", out)
    return {"rc": p.returncode, "out": out, "runtime": float(rt[-1]) if rt else None,
            "gteps": float(tp[-1]) if tp else None, "verified": "verification passed" in out}


def bfs_programs() -> list[tuple[str, str]]:
    """(model, program) of every reference OpenMP and C++-threads BFS program
    built unchanged into _ref/bfs_omp and _ref/bfs_cpp."""
    out = []
    for model in ("omp", "cpp"):
        d = REF_OUT / f"bfs_{model}"
        if d.is_dir():
            out += [(model, p.name) for p in sorted(d.iterdir()) if os.access(p, os.X_OK)]
    return out


def run_bfs_program(model: str, name: str, egr_path: str, src: int, threads: int, timeout: float = 600) -> dict:
    """One run of a reference CPU BFS program through its own main(): the
    median of its runs as it prints it, and its own verifier's verdict
    (OpenMP programs take the thread count from OMP_NUM_THREADS, C++-threads
    programs as an argument, include/bfs_vertex_cpp.h:91-110)."""
    exe = REF_OUT / f"bfs_{model}" / name
    args = [str(exe), egr_path, str(src), "1"]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    if model == "cpp":
        args += ["3", str(threads)]
    p = subprocess.run(args, capture_output=True, text=True, env=env, timeout=timeout)
    out = p.stdout + p.stderr
    rt = re.findall(r"runtime:\s*([0-9.eE+-]+)\s*s", out)
    return {"rc": p.returncode, "runtime": float(rt[-1]) if rt else None, "verified": "verification passed" in out}


# ---------------------------------------------------------------------------
# Size-independent certificates (certify.c, parallel C), for sizes where
# running the serial oracle is too slow.

_DIST_FAIL = {1: "dist[src] != 0", 2: "negative value", 3: "unreached neighbour of a reached vertex",
              4: "relaxable edge", 5: "reached vertex without a tight in-edge", 6: "weight below 1",
              -1: "out of memory", -2: "bad arguments"}
_CC_FAIL = {1: "adjacent labels differ", 2: "label above its vertex id", 3: "label is not its own label",
            4: "vertex not connected to its label", -1: "out of memory", -2: "bad arguments"}


def certify_distances(g, src: int, dist: np.ndarray, weighted: bool) -> str | None:
    """Shortest-path certificate (weights >= 1): dist[src] == 0; dist[v] <=
    dist[u] + w(u, v) on every edge out of a reached vertex, whose neighbours
    are all reached; every other reached vertex has a tight in-edge. Returns
    None when it holds, else what failed."""
    ni, nl = _csr(g)
    w = _p(np.ascontiguousarray(g.eweight, np.int32)) if weighted else None
    d = np.ascontiguousarray(dist, np.int32)
    rc = lib().oracle_certify_distances(g.nodes, _p(ni), _p(nl), w, int(src), _p(d))
    return None if rc == 0 else _DIST_FAIL.get(rc, f"code {rc}")


def certify_cc(g, label: np.ndarray) -> str | None:
    """Minimum-label certificate on a symmetric graph: labels equal across every
    edge, 0 <= label[v] <= v, label[label[v]] == label[v], and every vertex
    connected to the vertex its label names. Returns None when it holds."""
    ni, nl = _csr(g)
    lab = np.ascontiguousarray(label, np.int32)
    rc = lib().oracle_certify_cc(g.nodes, _p(ni), _p(nl), _p(lab))
    return None if rc == 0 else _CC_FAIL.get(rc, f"code {rc}")


def certify_mis(g, status: np.ndarray) -> str | None:
    """The checks of the reference MIS harness's verifier
    (include/mis_vertex_cuda.h:80-98): every vertex decided, no two adjacent
    vertices in the set, and every excluded vertex has a neighbour in the set.
    Returns None when they hold."""
    st = np.asarray(status)
    if not np.isin(st, (1, 2)).all():
        return "undecided vertex"
    deg = np.diff(np.asarray(g.nindex, np.int64))
    u = np.repeat(np.arange(g.nodes, dtype=np.int64), deg)
    inn = st == 1
    nbr_in = inn[np.asarray(g.nlist, np.int64)]
    if (inn[u] & nbr_in).any():
        return "adjacent vertices in the set"
    covered = np.zeros(g.nodes, bool)
    covered[u[nbr_in]] = True
    if not (inn | covered).all():
        return "set is not maximal"
    return None


# ---------------------------------------------------------------------------
# One call of a reference CPU host driver (oracle/_ref/libref_cpu_<name>.so).

_cpu = {}


def ref_cpu_run(name: str, g, src: int, threads: int, sp: np.ndarray | None = None) -> tuple[float, np.ndarray]:
    """Run the reference CPU program `name` (sssp_edge_cpp, sssp_vertex_cpp,
    sssp_edge_omp, bfs_cpp, bfs_omp, cc_cpp, cc_omp, mis_cpp) once; returns its own
    measured runtime in seconds and the result."""
    if name not in _cpu:
        L = C.CDLL(str(REF_OUT / f"libref_cpu_{name}.so"))
        P = C.POINTER(C.c_int)
        L.ref_cpu_run.argtypes = [C.c_int, C.c_int, P, P, P, C.c_int, P, P, C.c_int]
        L.ref_cpu_run.restype = C.c_double
        _cpu[name] = L
    ni, nl = _csr(g)
    w = np.ascontiguousarray(g.eweight, np.int32) if g.eweight is not None else None
    if sp is None and "edge" in name:
        sp = globals()["sp"](g)
    out = np.empty(g.nodes, np.int32)
    # the reference program prints progress on stdout; keep the caller's stdout clean
    import sys

    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        t = _cpu[name].ref_cpu_run(g.nodes, g.edges, _p(ni), _p(nl), _p(w) if w is not None else None, src,
                                   _p(out), _p(sp) if sp is not None else None, threads)
        C.CDLL(None).fflush(None)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    return float(t), out
