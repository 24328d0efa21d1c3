"""ctypes binding of oracle/_ref/libref_kernel.so -- the reference's own pair
kernel (BoostXmatch/Worker.cu, Common.cu) compiled unmodified for sm_100a and
driven by oracle/ref_harness.cu.  TEST INFRASTRUCTURE ONLY.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_kernel.so")
RAD2DEG = 57.295779513082323   # Common.h:9

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.ref_xmatch.restype = ctypes.c_longlong
        L.ref_xmatch.argtypes = [P, ctypes.c_longlong, P, P, P, ctypes.c_longlong, P, P, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_double, P, ctypes.c_uint, ctypes.POINTER(ctypes.c_int),
                                 ctypes.c_int, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_float)]
        _lib = L
    return _lib


def _zone_layout(objs, zh_deg, n_zones):
    """Group by zone as Sorter.cu does (zone = floor((dec+90)/zh), Sorter.cu:20-24;
    objects outside [0, n_zones) are left out, as the reference's lower/upper
    bound search leaves them outside every zone)."""
    zone = np.floor((objs["dec"] + 90.0) / zh_deg)
    ok = (zone >= 0) & (zone < n_zones)
    idx = np.nonzero(ok)[0]
    z = zone[idx].astype(np.int64)
    order = np.lexsort((objs["ra"][idx], z))
    idx = idx[order]
    z = z[order]
    radec = np.empty((len(idx), 2), np.float64)
    radec[:, 0] = objs["ra"][idx] / RAD2DEG     # Sorter.cu:52-62, division
    radec[:, 1] = objs["dec"][idx] / RAD2DEG
    zb = np.searchsorted(z, np.arange(n_zones), "left").astype(np.int32)
    ze = np.searchsorted(z, np.arange(n_zones), "right").astype(np.int32)
    return idx, np.ascontiguousarray(radec), zb, ze


def xmatch(A, B, sr_deg, zh_deg=None, validate=True, pad=True):
    """Pairs (idA, idB) the reference kernel appends; returns (pairs, n_outside, launches).

    pad=True launches whole 16x16 blocks only (the compaction of Worker.cu:
    157-233 is unsound in partial blocks) and keeps the pairs inside the true
    zone ranges: the reference predicate evaluated by its own kernel.
    pad=False uses the reference launch geometry as is."""
    if zh_deg is None:
        zh_deg = sr_deg
    n_zones = int(np.ceil(180 / zh_deg))       # Sorter.cu:156
    ia, ra, zba, zea = _zone_layout(A, zh_deg, n_zones)
    ib, rb, zbb, zeb = _zone_layout(B, zh_deg, n_zones)
    cap = max(1 << 16, 4 * (len(ia) + len(ib)))
    L = lib()
    while True:
        out = np.empty((cap, 2), np.uint32)
        launches = ctypes.c_int()
        outside = ctypes.c_longlong()
        n = L.ref_xmatch(ra.ctypes.data, len(ia), zba.ctypes.data, zea.ctypes.data, rb.ctypes.data, len(ib),
                         zbb.ctypes.data, zeb.ctypes.data, n_zones, sr_deg, zh_deg, out.ctypes.data, cap,
                         ctypes.byref(launches), 1 if (validate or pad) else 0, ctypes.byref(outside),
                         1 if pad else 0, None)
        if n < 0:
            if cap >= 1 << 30:
                raise RuntimeError("reference kernel harness failed")
            cap *= 4
            continue
        if n > cap:
            cap = int(n) + 1024
            continue
        p = out[:n].astype(np.int64)
        pairs = np.stack([A["id"][ia[p[:, 0]]], B["id"][ib[p[:, 1]]]], 1)
        return pairs, int(outside.value), launches.value


def time_zone_loop(A, B, sr_deg, zh_deg=None):
    """Device time of the reference's zone loop (Worker.cu:330-366) exactly as it
    launches: its geometry, no per-launch synchronisation; inputs are copied to
    the device before the clock starts.  Returns (seconds, launches, count)."""
    if zh_deg is None:
        zh_deg = sr_deg
    n_zones = int(np.ceil(180 / zh_deg))
    ia, ra, zba, zea = _zone_layout(A, zh_deg, n_zones)
    ib, rb, zbb, zeb = _zone_layout(B, zh_deg, n_zones)
    cap = max(1 << 16, 4 * (len(ia) + len(ib)))
    out = np.empty((cap, 2), np.uint32)
    launches = ctypes.c_int()
    outside = ctypes.c_longlong()
    ms = ctypes.c_float()
    n = lib().ref_xmatch(ra.ctypes.data, len(ia), zba.ctypes.data, zea.ctypes.data, rb.ctypes.data, len(ib),
                         zbb.ctypes.data, zeb.ctypes.data, n_zones, sr_deg, zh_deg, out.ctypes.data, cap,
                         ctypes.byref(launches), 0, ctypes.byref(outside), 0, ctypes.byref(ms))
    if n < 0:
        raise RuntimeError("reference kernel harness failed")
    return ms.value * 1e-3, launches.value, int(n)
