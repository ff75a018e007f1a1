"""ctypes binding of libmg_subiso.so (declarations in include/mg_subiso.h).

The library is built in-tree by ``matrixgraph_b200.build``; importing this
module without it raises immediately — there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmg_subiso.so")

MG_OK = 0
MG_E_IO = -1
MG_E_FORMAT = -2
MG_E_OOM = -3
MG_E_CAPACITY = -4
MG_E_TIMEOUT = -5
MG_E_CUDA = -6
MG_E_ARG = -7
MG_E_LIMIT = -8

MG_MAX_QUERY_VERTICES = 16
MG_MAX_LABELS = 256

MG_ORDER_REFERENCE = 0
MG_ORDER_STRONG = 1
MG_ORDER_LEARNED = 2
MG_ORDER_GIVEN = 3

MG_LANES_SHARED = 0xFFFFFFFF

MG_FILTER_DEGREE = 1
MG_FILTER_NLB = 2
MG_FILTER_ALL = 3

MG_BUILD_SYMMETRIZE = 1
MG_BUILD_NO_SELF = 2
MG_BUILD_DEDUP = 4

ERROR_NAMES = {
    MG_E_IO: "MG_E_IO", MG_E_FORMAT: "MG_E_FORMAT", MG_E_OOM: "MG_E_OOM",
    MG_E_CAPACITY: "MG_E_CAPACITY", MG_E_TIMEOUT: "MG_E_TIMEOUT", MG_E_CUDA: "MG_E_CUDA",
    MG_E_ARG: "MG_E_ARG", MG_E_LIMIT: "MG_E_LIMIT",
}

P32 = C.POINTER(C.c_uint32)


class CsrView(C.Structure):
    _fields_ = [("n", C.c_uint32), ("max_vid", C.c_uint32), ("min_vid", C.c_uint32),
                ("m_in", C.c_uint32), ("m_out", C.c_uint32), ("_pad", C.c_uint32),
                ("globalid", P32), ("indeg", P32), ("outdeg", P32), ("in_off", P32),
                ("out_off", P32), ("in_edges", P32), ("out_edges", P32),
                ("edges_globalid_by_localid", P32), ("localid_by_globalid", P32),
                ("labels", P32)]


class Opts(C.Structure):
    _fields_ = [("order", C.c_int32), ("filters", C.c_uint32), ("given_order", P32),
                ("model", C.c_void_p), ("chunk_rows", C.c_uint64), ("grab", C.c_uint32),
                ("root_step", C.c_uint32), ("probe_min", C.c_uint32),
                ("kernel_events", C.c_uint32), ("mem_budget_bytes", C.c_uint64),
                ("root_begin", C.c_uint64), ("root_end", C.c_uint64),
                ("no_tail", C.c_uint32), ("lanes", C.c_uint32),
                ("max_elements", C.c_uint64), ("matrix_filter", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("k", C.c_uint32), ("order", C.c_uint32 * MG_MAX_QUERY_VERTICES),
                ("level_rows", C.c_uint64 * (MG_MAX_QUERY_VERTICES + 1)),
                ("balg_bytes", C.c_uint64), ("balg_count_bytes", C.c_uint64),
                ("device_ms", C.c_double), ("launches", C.c_uint64), ("chunks", C.c_uint64),
                ("elements", C.c_uint64), ("expand_ms", C.c_double),
                ("expand_launches", C.c_uint64)]


class GraphInfo(C.Structure):
    _fields_ = [("n", C.c_uint32), ("n_labels", C.c_uint32), ("m_out", C.c_uint64),
                ("m_in", C.c_uint64), ("symmetric", C.c_uint32), ("device", C.c_uint32),
                ("device_bytes", C.c_uint64), ("max_degree", C.c_uint32),
                ("nlb_words", C.c_uint32), ("hubs", C.c_uint32),
                ("hub_min_degree", C.c_uint32), ("hub_bytes", C.c_uint64)]


MG_HUB_AUTO = 2 ** 64 - 1


class UploadOpts(C.Structure):
    _fields_ = [("hub_bytes", C.c_uint64), ("hub_min_degree", C.c_uint32),
                ("_reserved", C.c_uint32)]


class MGError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is not built; run python -m matrixgraph_b200.build")

lib = C.CDLL(LIB_PATH)

_VP = C.c_void_p
_PVP = C.POINTER(C.c_void_p)
_PV = C.POINTER(CsrView)
_PU64 = C.POINTER(C.c_uint64)
_SIGS = {
    "mg_last_error": (C.c_char_p, []),
    "mg_version": (C.c_char_p, []),
    "mg_opts_default": (None, [C.POINTER(Opts)]),
    "mg_csr_dir_open": (C.c_int, [C.c_char_p, _PV, _PVP]),
    "mg_csr_dir_close": (None, [_VP]),
    "mg_csr_dir_write": (C.c_int, [C.c_char_p, _PV]),
    "mg_csr_from_edges": (C.c_int, [C.c_uint32, P32, P32, C.c_uint64, P32, C.c_uint32, _PV,
                                    _PVP]),
    "mg_csr_from_csv": (C.c_int, [C.c_char_p, C.c_uint32, _PV, _PVP]),
    "mg_gen_chung_lu": (C.c_int, [C.c_uint32, C.c_double, C.c_double, C.c_uint64, C.c_uint32,
                                  C.POINTER(P32), C.POINTER(P32), _PU64]),
    "mg_gen_rmat": (C.c_int, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                              C.c_uint64, C.c_uint32, C.POINTER(P32), C.POINTER(P32), _PU64]),
    "mg_free_buffer": (None, [_VP]),
    "mg_gen_labels": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_double, C.c_uint64,
                                P32]),
    "mg_gen_query_walk": (C.c_int, [_PV, C.c_uint32, P32, P32, C.c_uint32, C.c_uint64, _PV,
                                    _PVP]),
    "mg_gen_query_random": (C.c_int, [_PV, C.c_uint32, C.c_double, C.c_uint64, _PV, _PVP]),
    "mg_query_from_edges": (C.c_int, [C.c_uint32, P32, P32, C.c_uint32, P32, C.c_int, _PV,
                                      _PVP]),
    "mg_plan_order": (C.c_int, [_VP, _PV, C.POINTER(Opts), P32, P32]),
    "mg_graph_upload": (C.c_int, [_PV, C.c_int, _PVP]),
    "mg_graph_free": (None, [_VP]),
    "mg_graph_get_info": (C.c_int, [_VP, C.POINTER(GraphInfo)]),
    "mg_graph_upload_ex": (C.c_int, [_PV, C.c_int, C.POINTER(UploadOpts), _PVP]),
    "mg_selftest_wait_timeout": (C.c_int, [_VP, _PV, C.c_uint32, C.POINTER(C.c_int)]),
    "mg_plan_orders": (C.c_int, [_VP, C.POINTER(_PV), C.c_uint32, C.POINTER(Opts), P32]),
    "mg_matrix_filter_load": (C.c_int, [C.POINTER(C.c_char_p), C.c_int, C.POINTER(C.c_void_p)]),
    "mg_matrix_filter_free": (None, [_VP]),
    "mg_matrix_filter_keep": (C.c_int, [_VP, C.c_uint32, P32, C.c_uint64,
                                        C.POINTER(C.c_uint8)]),
    "mg_subiso_count": (C.c_int, [_VP, _PV, C.POINTER(Opts), _PU64]),
    "mg_subiso_count_ex": (C.c_int, [_VP, _PV, C.POINTER(Opts), _PU64, C.POINTER(Stats)]),
    "mg_subiso_emit": (C.c_int, [_VP, _PV, C.POINTER(Opts), P32, C.c_uint64, _PU64]),
    "mg_subiso_emit_ex": (C.c_int, [_VP, _PV, C.POINTER(Opts), P32, C.c_uint64, _PU64,
                                    C.POINTER(Stats)]),
    "mg_subiso_batch_count": (C.c_int, [_VP, C.POINTER(_PV), C.c_uint32, C.POINTER(Opts),
                                        _PU64]),
    "mg_subiso_batch_count_ex": (C.c_int, [_VP, C.POINTER(_PV), C.c_uint32, C.POINTER(Opts),
                                           _PU64, C.POINTER(Stats)]),
    "mg_subiso_count_noalloc": (C.c_int, [_VP, _PV, C.POINTER(Opts), _PU64]),
    "mg_subiso_batch_count_orders": (C.c_int, [_VP, C.POINTER(_PV), C.c_uint32, P32,
                                               C.POINTER(Opts), _PU64, _PU64,
                                               C.POINTER(Stats)]),
    "mg_order_model_create": (C.c_int, [C.c_int, C.c_uint64, _PVP]),
    "mg_order_model_load": (C.c_int, [C.c_char_p, C.c_int, _PVP]),
    "mg_order_model_save": (C.c_int, [_VP, C.c_char_p]),
    "mg_order_model_free": (None, [_VP]),
    "mg_order_model_num_params": (C.c_int, []),
    "mg_order_model_get_params": (C.c_int, [_VP, C.POINTER(C.c_float)]),
    "mg_order_model_set_params": (C.c_int, [_VP, C.POINTER(C.c_float)]),
    "mg_order_model_train": (C.c_int, [_VP, _VP, C.POINTER(_PV), C.c_uint32, P32, P32,
                                       C.POINTER(C.c_float), C.c_uint32, C.c_uint32,
                                       C.c_uint32, C.c_float, C.c_uint64,
                                       C.POINTER(C.c_float)]),
    "mg_order_model_grad": (C.c_int, [_VP, _VP, C.POINTER(_PV), C.c_uint32, P32, P32,
                                      C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_float),
                                      C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "mg_order_model_predict": (C.c_int, [_VP, _VP, C.POINTER(_PV), C.c_uint32, P32, P32,
                                         C.c_uint32, C.POINTER(C.c_float)]),
    "mg_order_model_features": (C.c_int, [_VP, _PV, C.POINTER(C.c_float),
                                          C.POINTER(C.c_float), P32]),
}

# include/mg_gar_match.h
_PI32 = C.POINTER(C.c_int32)
_PI = C.POINTER(C.c_int)
_GAR_ARGS = [P32, _PI32, C.c_int, P32, P32, P32, _PI32, C.c_int,        # data graph
             _PI32, C.c_int, _PI32, _PI32, _PI32, C.c_int,              # pattern
             _PI, P32, _PI32, _PI32, _PI32, _PI32, C.c_int, _PI,         # rows
             P32, C.c_int, _PI]                                          # matched ids
_SIGS["matrixgraph_gar_match"] = (C.c_int, list(_GAR_ARGS))
_SIGS["mg_gar_match_ex"] = (C.c_int, list(_GAR_ARGS) + [C.POINTER(Opts), _PU64])
_SIGS["mg_gar_instance"] = (C.c_int, [P32, _PI32, C.c_int, P32, P32, _PI32, C.c_int,
                                      _PI32, C.c_int, _PI32, _PI32, _PI32, C.c_int,
                                      _PV, _PVP, _PV, _PVP])
_SIGS["mg_gar_flatten"] = (C.c_int, [P32, C.c_uint64, C.c_uint32, C.c_uint32, P32, C.c_int]
                           + list(_GAR_ARGS[14:]))

EXPORTED = tuple(_SIGS)

for _name, (_res, _args) in _SIGS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def check(rc: int) -> int:
    """Raises MGError for a negative status, returns the status otherwise."""
    if rc != MG_OK:
        raise MGError(rc, (lib.mg_last_error() or b"").decode())
    return rc


def default_opts(**kw) -> Opts:
    o = Opts()
    lib.mg_opts_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o
