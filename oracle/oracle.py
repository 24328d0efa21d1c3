"""ctypes binding of ``xm_oracle.c`` (TEST INFRASTRUCTURE ONLY).

The C file restates the reference's zone algorithm (BoostXmatch/Sorter.cu,
Common.cu, Worker.cu); see its header for the line-by-line citations.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

OBJ_DTYPE = np.dtype([("id", "<i8"), ("ra", "<f8"), ("dec", "<f8")])  # Obj.h:21-25

MODE_ALLPAIRS = 0
MODE_ALLPAIRS_SINCOS = 1
MODE_WINDOWED = 2


class OrStats(ctypes.Structure):
    _fields_ = [("n_tested", ctypes.c_uint64), ("n_cand", ctypes.c_uint64),
                ("n_match", ctypes.c_uint64), ("nA_kept", ctypes.c_uint64),
                ("nB_kept", ctypes.c_uint64), ("n_zones", ctypes.c_int64),
                ("nz", ctypes.c_int32), ("sr_rad", ctypes.c_double),
                ("sr_dist2", ctypes.c_double)]


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.or_xmatch.restype = ctypes.c_int64
        L.or_xmatch.argtypes = [P, ctypes.c_int64, P, ctypes.c_int64, ctypes.c_double,
                                ctypes.c_double, ctypes.c_int, ctypes.c_int, P, P,
                                ctypes.c_uint64, ctypes.POINTER(OrStats)]
        L.or_sincos_batch.argtypes = [P, ctypes.c_int64, P, P]
        L.or_unit_vectors.argtypes = [P, P, ctypes.c_int64, P]
        L.or_alpha_table.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int64, P]
        L.or_calc_alpha.restype = ctypes.c_double
        L.or_calc_alpha.argtypes = [ctypes.c_double, ctypes.c_double]
        L.or_build_export.restype = ctypes.c_int64
        L.or_build_export.argtypes = [P, ctypes.c_int64, ctypes.c_double, P, P, P, P, ctypes.c_int64]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def as_objs(a):
    a = np.ascontiguousarray(a)
    if a.dtype != OBJ_DTYPE:
        raise TypeError("expected .idradec records")
    return a


def xmatch(A, B, sr_deg, zh_deg=None, mode=MODE_WINDOWED, nthreads=None, with_dist=True):
    """Return (pairs[n,2] int64, dist[n] float64, stats) of the full crossmatch."""
    A = as_objs(A)
    B = as_objs(B)
    if zh_deg is None:
        zh_deg = sr_deg
    if nthreads is None:
        nthreads = os.cpu_count() or 1
    st = OrStats()
    L = lib()
    cap = max(16, 2 * max(len(A), len(B)))
    while True:
        pairs = np.empty((cap, 2), np.int64)
        dist = np.empty(cap, np.float64) if with_dist else None
        n = L.or_xmatch(_ptr(A), len(A), _ptr(B), len(B), sr_deg, zh_deg, mode, nthreads,
                        _ptr(pairs), _ptr(dist), cap, ctypes.byref(st))
        if n < 0:
            raise RuntimeError("oracle failed (%d)" % n)
        if n <= cap:
            return pairs[:n], (dist[:n] if with_dist else None), st
        cap = int(n)


def sincos(x):
    x = np.ascontiguousarray(x, np.float64)
    s = np.empty_like(x)
    c = np.empty_like(x)
    lib().or_sincos_batch(_ptr(x), len(x), _ptr(s), _ptr(c))
    return s, c


def unit_vectors(ra_deg, dec_deg):
    ra = np.ascontiguousarray(ra_deg, np.float64)
    de = np.ascontiguousarray(dec_deg, np.float64)
    out = np.empty((len(ra), 3), np.float64)
    lib().or_unit_vectors(_ptr(ra), _ptr(de), len(ra), _ptr(out))
    return out


def alpha_table(sr_deg, zh_deg):
    n_zones = int(np.ceil(180 / zh_deg))
    out = np.empty(n_zones, np.float64)
    lib().or_alpha_table(sr_deg, zh_deg, n_zones, _ptr(out))
    return out


def calc_alpha(theta, abs_dec):
    return lib().or_calc_alpha(theta, abs_dec)


def build_export(A, zh_deg):
    """Sorted segment as the reference's Sorter produces it: (id, radec_rad[n,2], zbeg, zend)."""
    A = as_objs(A)
    n_zones = int(np.ceil(180 / zh_deg))
    ids = np.empty(max(1, len(A)), np.int64)
    radec = np.empty((max(1, len(A)), 2), np.float64)
    zb = np.empty(n_zones, np.int64)
    ze = np.empty(n_zones, np.int64)
    m = lib().or_build_export(_ptr(A), len(A), zh_deg, _ptr(ids), _ptr(radec), _ptr(zb), _ptr(ze), n_zones)
    return ids[:m], radec[:m], zb, ze
