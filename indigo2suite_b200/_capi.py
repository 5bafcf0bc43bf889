"""ctypes declarations of the C ABI in include/i2b200.h.

The library is loaded from this package directory (libi2b200.so, built in-tree
by indigo2suite_b200/build.py). There is no fallback: if the library is missing
or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# I2B200_LIB selects another build of the library (e.g. one with other tuning constants)
LIB_PATH = Path(os.environ.get("I2B200_LIB") or Path(__file__).resolve().parent / "libi2b200.so")

I2_OK = 0
I2_ERR_ARG = 1
I2_ERR_IO = 2
I2_ERR_FORMAT = 3
I2_ERR_NOMEM = 4
I2_ERR_CUDA = 5
I2_ERR_NO_DEVICE = 6
I2_ERR_UNSUPPORTED = 7
I2_ERR_ITER_CAP = 8
I2_ERR_OVERFLOW = 9
I2_ERR_CAPACITY = 10
I2_ERR_STALL = 11

I2_BFS, I2_SSSP, I2_CC, I2_MIS = 0, 1, 2, 3
MIS_IN, MIS_OUT = 1, 2  # status values of i2_mis (the reference's included / excluded)

I2_AUTO_HEURISTIC = -1
I2_AUTO_LEARNED = -2
I2_SSSP_BUDGET_AUTO = -1
I2_ORDER_NONE = 0
I2_ORDER_DEGREE = 1
VARIANTS = ["vp_thread", "vp_warp", "vp_cta", "vp_block", "pull_frontier", "pull_topo", "edge_topo", "push_topo",
            "union_find"]
I2_NUM_VARIANTS = len(VARIANTS)
I2_LOOP_GRAPH, I2_LOOP_HOST, I2_LOOP_RELAUNCH = 0, 1, 2

NUM_FEATURES = 16


class EclGraphC(C.Structure):
    _fields_ = [("nodes", C.c_int), ("edges", C.c_int), ("nindex", C.POINTER(C.c_int)),
                ("nlist", C.POINTER(C.c_int)), ("eweight", C.POINTER(C.c_int))]


class Opts(C.Structure):
    _fields_ = [("variant", C.c_int), ("loop_mode", C.c_int), ("iter_cap", C.c_int),
                ("record_iters", C.c_int), ("stream", C.c_void_p), ("sssp_delta", C.c_int),
                ("then_at", C.c_int), ("then_variant", C.c_int), ("sssp_budget", C.c_int)]


class Report(C.Structure):
    _fields_ = [("seconds", C.c_double), ("relax_seconds", C.c_double), ("iterations", C.c_int),
                ("variant_hist", C.c_int * 16), ("reached_vertices", C.c_longlong),
                ("reached_edges", C.c_longlong)]


class IterRecord(C.Structure):
    _fields_ = [("iter", C.c_int), ("variant", C.c_int), ("size", C.c_int), ("hsize", C.c_int),
                ("edges", C.c_ulonglong), ("maxdeg", C.c_int), ("mindist", C.c_int),
                ("visited", C.c_longlong), ("t_ns", C.c_ulonglong), ("feat", C.c_float * NUM_FEATURES),
                ("kind", C.c_int), ("threshold", C.c_int), ("pile", C.c_uint), ("pad", C.c_int)]


class GraphInfo(C.Structure):
    _fields_ = [("nodes", C.c_int), ("edges", C.c_int), ("maxdeg", C.c_int), ("nheavy", C.c_int),
                ("wmin", C.c_int), ("symmetric", C.c_int), ("has_weights", C.c_int),
                ("avgdeg", C.c_float), ("degcv", C.c_float)]


_P = C.c_void_p
_I = C.c_int
_PI = C.POINTER(C.c_int)
_PF = C.POINTER(C.c_float)
_PG = C.POINTER(EclGraphC)

# name -> (restype, argtypes)
SIGNATURES = {
    "i2_status_string": (C.c_char_p, [_I]),
    "i2_variant_name": (C.c_char_p, [_I]),
    "i2_version": (_I, []),
    "i2_device_count": (_I, []),
    "i2_read_eclgraph": (_I, [C.c_char_p, _PG]),
    "i2_write_eclgraph": (_I, [_PG, C.c_char_p]),
    "i2_free_eclgraph": (None, [_PG]),
    "i2_alloc_eclgraph": (_I, [_I, _I, _I, _PG]),
    "i2_synth_weights": (_I, [_PG]),
    "i2_build_sp": (_I, [_PG, _PI]),
    "i2_gen_er": (_I, [_I, C.c_longlong, C.c_uint64, _I, _PG]),
    "i2_gen_rmat": (_I, [_I, _I, C.c_double, C.c_double, C.c_double, C.c_uint64, _I, _PG]),
    "i2_gen_grid": (_I, [_I, C.c_double, C.c_double, C.c_uint64, _I, _PG]),
    "i2_graph_upload": (_I, [_PG, C.POINTER(_P)]),
    "i2_graph_wrap_device": (_I, [_PG, C.POINTER(_P)]),
    "i2_graph_generate_rmat_n": (_I, [_I, _I, C.c_double, C.c_double, C.c_double, C.c_uint64, _I,
                                      C.POINTER(C.c_void_p)]),
    "i2_batch_from_device": (_I, [C.POINTER(C.c_void_p), _I, C.POINTER(C.c_void_p)]),
    "i2_graph_generate_er": (_I, [_I, C.c_longlong, C.c_uint64, _I, C.POINTER(C.c_void_p)]),
    "i2_graph_generate_grid": (_I, [_I, C.c_double, C.c_double, C.c_uint64, _I, C.POINTER(C.c_void_p)]),
    "i2_graph_from_coo_device": (_I, [_I, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, _I,
                                      C.POINTER(C.c_void_p)]),
    "i2_graph_sp": (_I, [C.c_void_p, C.POINTER(C.c_void_p), _PI]),
    "i2_graph_hub": (_I, [C.c_void_p, _PI]),
    "i2_graph_generate_rmat": (_I, [_I, _I, C.c_double, C.c_double, C.c_double, C.c_uint64, _I,
                                    C.POINTER(_P)]),
    "i2_graph_size": (_I, [_P, _PI, _PI]),
    "i2_graph_degree": (_I, [_P, _I, _PI]),
    "i2_graph_info_get": (_I, [_P, C.POINTER(GraphInfo)]),
    "i2_graph_download": (_I, [_P, _PG]),
    "i2_graph_synth_weights": (_I, [_P]),
    "i2_graph_tune": (_I, [_P, _I, _I, _I]),
    "i2_graph_reorder": (_I, [_P, _I]),
    "i2_gen_rmat_n": (_I, [_I, _I, C.c_double, C.c_double, C.c_double, C.c_uint64, _I, _PG]),
    "i2_graph_free": (_I, [_P]),
    "i2_trim_device_memory": (_I, []),
    "i2_bfs": (_I, [_P, _I, _PI, C.POINTER(Opts), C.POINTER(Report)]),
    "i2_sssp": (_I, [_P, _I, _PI, C.POINTER(Opts), C.POINTER(Report)]),
    "i2_cc": (_I, [_P, _PI, C.POINTER(Opts), C.POINTER(Report)]),
    "i2_mis": (_I, [_P, _PI, C.POINTER(Opts), C.POINTER(Report)]),
    "i2_run_device": (_I, [_P, _I, _I, C.c_void_p, C.POINTER(Opts), C.POINTER(Report)]),
    "i2_get_records": (_I, [_P, C.POINTER(IterRecord), _I, _PI]),
    "i2_sweep": (_I, [_P, _I, _I, _I, _I, C.POINTER(IterRecord), _PF, _I, _PI]),
    "i2_mlp_param_count": (_I, []),
    "i2_mlp_set_params": (_I, [_PF, _I]),
    "i2_mlp_loss_grad": (_I, [_PF, _PF, _PF, _PF, _I, _PF, _PF]),
    "i2_mlp_train": (_I, [_PF, _PF, _PF, _PF, _I, _I, _I, C.c_float, C.c_uint64, _PF]),
    "i2_mlp_predict": (_I, [_PF, _PF, _I, _I, _PI]),
    "i2_run_noalloc": (_I, [_I, _PG, _I, C.c_void_p, C.c_void_p, _PI]),
    "i2_batch_upload": (_I, [_PG, _I, C.POINTER(_P)]),
    "i2_batch_run": (_I, [_P, _I, _PI, _PI, C.POINTER(Opts), C.POINTER(Report)]),
    "i2_batch_offsets": (_I, [_P, C.POINTER(C.c_longlong)]),
    "i2_batch_run_device": (_I, [_P, _I, _PI, C.POINTER(Opts), C.POINTER(Report)]),
    "i2_batch_result": (_I, [_P, _PI, C.POINTER(Opts)]),
    "i2_batch_tune": (_I, [_P, _I, _I, _I]),
    "i2_batch_free": (_I, [_P]),
}


def load(path: Path | str = LIB_PATH) -> C.CDLL:
    path = Path(path)
    if not path.exists():
        raise ImportError(f"{path} is not built; run indigo2suite_b200/build.py (or __graft_entry__.build())")
    lib = C.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
