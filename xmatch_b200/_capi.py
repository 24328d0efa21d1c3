"""ctypes declarations of include/xmatch.h (libxmatch_b200.so).

The shared library is built in-tree (``python xmatch_b200/build.py``).  There
is no fallback: if the library is missing or cannot be loaded, import of
this module raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxmatch_b200.so")

XM_OK = 0
XM_ERR_INVALID = 1
XM_ERR_CUDA = 2
XM_ERR_NOMEM = 3
XM_ERR_CAPACITY = 4
XM_ERR_MISMATCH = 5
XM_ERR_NODEVICE = 6
XM_ERR_IO = 7
XM_ERR_BUSY = 8
XM_ERR_TIMEOUT = 9
XM_ERR_TOO_LARGE = 10
XM_NOALLOC_MAX_OBJS = 1 << 20

XM_FILTER32 = 0
XM_PLAIN64 = 1 << 0
XM_COUNT_CAND = 1 << 1
XM_NO_DIST = 1 << 2
XM_NO_GRAPH = 1 << 3


class XmObj(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int64), ("ra_deg", ctypes.c_double), ("dec_deg", ctypes.c_double)]


class XmPairs(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_void_p), ("dist", ctypes.c_void_p),
                ("capacity", ctypes.c_uint64), ("count", ctypes.c_uint64)]


class XmStats(ctypes.Structure):
    _fields_ = [("n_tested", ctypes.c_uint64), ("n_cand", ctypes.c_uint64),
                ("n_border", ctypes.c_uint64), ("n_exact", ctypes.c_uint64),
                ("n_match", ctypes.c_uint64), ("n_tiles", ctypes.c_uint64),
                ("n_launches", ctypes.c_uint32), ("n_retries", ctypes.c_uint32),
                ("ms_total", ctypes.c_float), ("ms_match", ctypes.c_float),
                ("ms_build", ctypes.c_float), ("ms_h2d", ctypes.c_float),
                ("ms_d2h", ctypes.c_float), ("ms_zb_count", ctypes.c_float),
                ("ms_zb_scan", ctypes.c_float), ("ms_zb_scatter", ctypes.c_float),
                ("ms_zb_sort", ctypes.c_float), ("ms_plan", ctypes.c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class XmTuning(ctypes.Structure):
    _fields_ = [("tile", ctypes.c_uint32), ("chunk", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_uint32),
                ("zones", ctypes.c_uint32)]


class XmServeCfg(ctypes.Structure):
    _fields_ = [("mem_budget", ctypes.c_uint64), ("max_batch", ctypes.c_uint32), ("flags", ctypes.c_uint32)]


class XmServeInfo(ctypes.Structure):
    _fields_ = [("t_submit_ms", ctypes.c_double), ("t_admit_ms", ctypes.c_double), ("t_built_ms", ctypes.c_double),
                ("t_batch_ms", ctypes.c_double), ("t_matched_ms", ctypes.c_double), ("t_done_ms", ctypes.c_double),
                ("batch", ctypes.c_uint32), ("batch_size", ctypes.c_uint32), ("count", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class XmJob(ctypes.Structure):
    _fields_ = [("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("sr_deg", ctypes.c_double)]


P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I32 = ctypes.c_int32
D = ctypes.c_double
PP = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes); every function declared in include/xmatch.h
SIGNATURES = {
    "xm_ctx_create": (ctypes.c_int, [ctypes.c_int, PP]),
    "xm_ctx_destroy": (ctypes.c_int, [P]),
    "xm_status_str": (ctypes.c_char_p, [ctypes.c_int]),
    "xm_last_error": (ctypes.c_char_p, [P]),
    "xm_ctx_info": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(U64), ctypes.POINTER(U64)]),
    "xm_ctx_synchronize": (ctypes.c_int, [P]),
    "xm_ctx_stream": (ctypes.c_int, [P, PP]),
    "xm_segment_build": (ctypes.c_int, [P, U32, P, U64, D, PP, ctypes.POINTER(XmStats)]),
    "xm_segment_build_device": (ctypes.c_int, [P, U32, P, U64, D, PP, ctypes.POINTER(XmStats)]),
    "xm_segment_rebuild_device": (ctypes.c_int, [P, P, U64, ctypes.POINTER(XmStats)]),
    "xm_segment_free": (ctypes.c_int, [P]),
    "xm_segment_offload": (ctypes.c_int, [P]),
    "xm_segment_page_in": (ctypes.c_int, [P]),
    "xm_segment_page_out": (ctypes.c_int, [P]),
    "xm_segment_resident": (ctypes.c_int, [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(U64)]),
    "xm_segment_info": (ctypes.c_int, [P, ctypes.POINTER(U32), ctypes.POINTER(U64), ctypes.POINTER(I32),
                                       ctypes.POINTER(D)]),
    "xm_segment_export": (ctypes.c_int, [P, P, P, P, P]),
    "xm_match": (ctypes.c_int, [P, P, P, D, U32, ctypes.POINTER(XmPairs), ctypes.POINTER(XmStats)]),
    "xm_fetch_pairs": (ctypes.c_int, [P, ctypes.POINTER(XmPairs)]),
    "xm_match_batch": (ctypes.c_int, [P, ctypes.POINTER(XmJob), U32, U32, ctypes.POINTER(XmTuning),
                                      ctypes.POINTER(XmPairs), ctypes.POINTER(U64), ctypes.POINTER(XmStats)]),
    "xm_autotune_batch": (ctypes.c_int, [P, ctypes.POINTER(XmJob), U32, U32, ctypes.POINTER(XmTuning),
                                         ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "xm_idradec_count": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(U64)]),
    "xm_idradec_read": (ctypes.c_int, [ctypes.c_char_p, U64, U64, P]),
    "xm_idradec_write": (ctypes.c_int, [ctypes.c_char_p, P, U64]),
    "xm_pairs_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(XmPairs), ctypes.c_int, ctypes.c_int]),
    "xm_unit_vectors": (ctypes.c_int, [P, P, P, U64, P]),
    "xm_segment_build_noalloc": (ctypes.c_int, [ctypes.c_int, P, P, U64, D, P, P, P, P, U64,
                                                ctypes.POINTER(U64)]),
    "xm_alpha_table": (ctypes.c_int, [D, D, P, I32]),
    "xm_filter_bounds": (ctypes.c_int, [D, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]),
    "xm_crossmatch": (ctypes.c_int, [P, P, U64, P, U64, D, D, U32, ctypes.POINTER(XmPairs), ctypes.POINTER(XmStats)]),
    "xm_serve_open": (ctypes.c_int, [P, P, ctypes.POINTER(XmServeCfg), PP]),
    "xm_serve_submit": (ctypes.c_int, [P, P, U64, D, ctypes.POINTER(U64)]),
    "xm_serve_poll": (ctypes.c_int, [P, U64, ctypes.c_int, ctypes.POINTER(XmPairs), ctypes.POINTER(XmServeInfo)]),
    "xm_serve_last_error": (ctypes.c_int, [P, ctypes.c_char_p, U64]),
    "xm_serve_close": (ctypes.c_int, [P]),
}


def load(path=LIB_PATH):
    if not os.path.exists(path):
        raise ImportError("libxmatch_b200.so not built: run `python xmatch_b200/build.py` (%s)" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()
