"""ctypes binding of libsubgraph_b200.so (the C ABI in include/sg_api.h).

The library is loaded from this package directory; a missing library is an
error (there is no fallback implementation).
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsubgraph_b200.so")

SG_OK = 0
SG_ERR_INVALID = 1
SG_ERR_OOM = 2
SG_ERR_CUDA = 3
SG_ERR_TIMEOUT = 4
SG_ERR_IO = 5
SG_ERR_UNSUPPORTED = 6

MODE_REFERENCE = 0
MODE_FP64 = 1
MODE_ORIGINAL = 2
MODE_ORIGINAL_CSR = 3

# every symbol include/sg_api.h declares
EXPORTS = [
    "sg_last_error", "sg_version", "sg_free",
    "sg_edgelist_read", "sg_edgelist_write", "sg_csc_build", "sg_csr_build",
    "sg_graph_data_write", "sg_graph_data_read", "sg_graph_data_encode", "sg_graph_data_decode",
    "sg_rmat_generate",
    "sg_plan_create", "sg_plan_read", "sg_plan_destroy", "sg_plan_info", "sg_plan_sub", "sg_plan_shared_tables",
    "sg_plan_tables", "sg_plan_automorphisms", "sg_plan_sub_edges",
    "sg_graph_create", "sg_graph_destroy", "sg_graph_info", "sg_graph_create_edges", "sg_graph_create_text",
    "sg_graph_create_rmat", "sg_graph_download_csc",
    "sg_count_opts_default", "sg_count", "sg_count_jobs", "sg_estimate",
    "sg_colors", "sg_debug_sub_table", "sg_debug_root", "sg_debug_count_unsatisfiable_wait",
    "sg_colors_noalloc",
    "sg_countmat_create", "sg_countmat_destroy", "sg_countmat_initialization",
    "sg_countmat_set_seed", "sg_countmat_compute", "sg_countmat_raw",
]


class SGError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[sg status {code}] {msg}")
        self.code = code


class CountOpts(ctypes.Structure):
    _fields_ = [("n_colorings", ctypes.c_int32), ("seed_base", ctypes.c_uint32), ("mode", ctypes.c_int32),
                ("batch", ctypes.c_int32), ("hub_threshold", ctypes.c_int32), ("profile", ctypes.c_int32),
                ("no_autotune", ctypes.c_int32), ("exact", ctypes.c_int32), ("wait_limit_ms", ctypes.c_int32),
                ("no_blocked", ctypes.c_int32),
                ("persistent", ctypes.c_int32), ("no_rooted", ctypes.c_int32),
                ("no_flat", ctypes.c_int32)]


class CountStats(ctypes.Structure):
    _fields_ = [("device_ms", ctypes.c_double), ("kernel_launches", ctypes.c_int64), ("table_bytes", ctypes.c_int64),
                ("fused_ms", ctypes.c_double), ("fused_launches", ctypes.c_int64), ("fused_alg_bytes", ctypes.c_double),
                ("fused_gather_bytes", ctypes.c_double), ("hub_ms", ctypes.c_double), ("top_sub", ctypes.c_int32),
                ("top_launches", ctypes.c_int64), ("top_ms", ctypes.c_double), ("top_alg_bytes", ctypes.c_double)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                          "or `python subgraph_b200/build.py` (there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, u32, u64, d = (ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32,
                                 ctypes.c_uint64, ctypes.c_double)
    P = ctypes.POINTER
    pp = P(ctypes.c_void_p)
    sigs = {
        "sg_last_error": ([], ctypes.c_char_p),
        "sg_version": ([], ctypes.c_char_p),
        "sg_free": ([vp], None),
        "sg_edgelist_read": ([ctypes.c_char_p, P(i32), P(i64), pp, pp], i32),
        "sg_edgelist_write": ([ctypes.c_char_p, i32, i64, vp, vp], i32),
        "sg_csc_build": ([i32, i64, vp, vp, pp, pp, pp], i32),
        "sg_csr_build": ([i32, i64, vp, vp, pp, pp, pp], i32),
        "sg_graph_data_write": ([ctypes.c_char_p, i32, i32, vp, vp, vp], i32),
        "sg_graph_data_read": ([ctypes.c_char_p, P(i32), P(i32), pp, pp, pp], i32),
        "sg_graph_data_encode": ([i32, i32, vp, vp, vp, pp, P(i64)], i32),
        "sg_graph_data_decode": ([vp, i64, P(i32), P(i32), pp, pp, pp], i32),
        "sg_rmat_generate": ([i32, i32, d, d, d, u64, P(i32), P(i64), pp, pp], i32),
        "sg_plan_create": ([i32, i32, vp, vp, pp], i32),
        "sg_plan_read": ([ctypes.c_char_p, pp], i32),
        "sg_plan_destroy": ([vp], None),
        "sg_plan_info": ([vp, P(i32), P(i32), P(i32), P(i64)], i32),
        "sg_plan_sub": ([vp, i32, vp], i32),
        "sg_plan_shared_tables": ([vp, vp], i32),
        "sg_plan_tables": ([vp, i32, vp, vp, vp], i32),
        "sg_plan_automorphisms": ([vp, P(i32)], i32),
        "sg_plan_sub_edges": ([vp, i32, P(i32), vp, vp], i32),
        "sg_graph_create": ([vp, vp, i32, i64, i32, pp], i32),
        "sg_graph_destroy": ([vp], None),
        "sg_graph_info": ([vp, P(i32), P(i64), P(i32)], i32),
        "sg_graph_create_edges": ([i32, vp, vp, i64, i32, pp], i32),
        "sg_graph_create_text": ([ctypes.c_char_p, i32, pp], i32),
        "sg_graph_create_rmat": ([i32, i32, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_uint64, i32,
                                  pp], i32),
        "sg_graph_download_csc": ([vp, vp, vp], i32),
        "sg_count_opts_default": ([P(CountOpts)], None),
        "sg_count": ([vp, vp, P(CountOpts), vp, P(CountStats)], i32),
        "sg_count_jobs": ([vp, i32, vp, vp, P(CountOpts), vp, vp, P(CountStats)], i32),
        "sg_estimate": ([vp, i32, i32, i32, P(d)], i32),
        "sg_colors": ([vp, i32, u32, vp], i32),
        "sg_debug_sub_table": ([vp, vp, u32, i32, i32, i32, vp], i32),
        "sg_debug_root": ([vp, vp, u32, i32, i32, vp, P(d)], i32),
        "sg_debug_count_unsatisfiable_wait": ([vp, vp, P(CountOpts), vp], i32),
        "sg_colors_noalloc": ([i32, i32, u32, vp, vp], i32),
        "sg_countmat_create": ([pp], i32),
        "sg_countmat_destroy": ([vp], None),
        "sg_countmat_initialization": ([vp, vp, vp, i32, i32, i32, i32, i32, i32], i32),
        "sg_countmat_set_seed": ([vp, u32], i32),
        "sg_countmat_compute": ([vp, vp, i32, i32, P(d)], i32),
        "sg_countmat_raw": ([vp, vp], i32),
    }
    for name, (args, res) in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(status: int) -> None:
    if status != SG_OK:
        msg = lib().sg_last_error()
        raise SGError(status, msg.decode() if msg else "")
