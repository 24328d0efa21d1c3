"""xmatch_b200 -- zone-algorithm catalog crossmatch on one B200.

Python access to libxmatch_b200.so (include/xmatch.h).  The compute path is
the CUDA library; this module only moves arrays across the C ABI.  Names
follow the reference (matthiaslee/Xmatch, BoostXmatch): catalogs are split
into segments, a segment is zone-sorted by the builder (Sorter::Sort), a job
is a pair of segments and a radius (Job), and matching a job
(Worker::Match) yields (idA, idB) pairs plus the distance in radians.
"""
import ctypes

import numpy as np

from . import _capi
from ._capi import (XM_COUNT_CAND, XM_FILTER32, XM_NO_DIST, XM_NO_GRAPH, XM_OK, XM_PLAIN64,  # noqa: F401
                    XmJob, XmPairs, XmStats, XmTuning)

OBJ_DTYPE = np.dtype([("id", "<i8"), ("ra", "<f8"), ("dec", "<f8")])   # Obj.h:21-25, 24 bytes
PAIR_DTYPE = np.dtype([("idA", "<i8"), ("idB", "<i8")])                 # Worker.cu:413-417, 16 bytes

_lib = _capi.lib


class XmatchError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        text = _lib.xm_status_str(status).decode()
        super().__init__("%s (%d)%s" % (text, status, (": " + msg) if msg else ""))


def _check(status, ctx=None):
    if status != XM_OK:
        msg = _lib.xm_last_error(ctx).decode(errors="replace") if ctx else ""
        raise XmatchError(status, msg)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def as_objs(a):
    """View a structured array / bytes as contiguous .idradec records."""
    if isinstance(a, (bytes, bytearray, memoryview)):
        a = np.frombuffer(a, OBJ_DTYPE)
    a = np.ascontiguousarray(a)
    if a.dtype != OBJ_DTYPE:
        if a.dtype.names == ("id", "ra", "dec"):
            a = a.astype(OBJ_DTYPE)
        else:
            raise TypeError("expected records with fields (id int64, ra f64, dec f64)")
    return a


def read_idradec(path, first=0, count=None):
    """Read a headerless .idradec file (Segment::Load, Segment.cpp:14-22)."""
    n = ctypes.c_uint64()
    _check(_lib.xm_idradec_count(path.encode(), ctypes.byref(n)))
    total = n.value
    if count is None:
        count = total - first
    out = np.empty(max(0, count), OBJ_DTYPE)
    _check(_lib.xm_idradec_read(path.encode(), first, count, _ptr(out)))
    return out


def write_idradec(path, objs):
    objs = as_objs(objs)
    _check(_lib.xm_idradec_write(path.encode(), _ptr(objs), len(objs)))


def write_pairs(path, pairs, dist=None, mode=16, append=False):
    """Write matches: mode 16 = reference {idA, idB}, 24 = with distance, 0 = ASCII."""
    pairs = np.ascontiguousarray(pairs, np.int64).reshape(-1, 2)
    d = np.ascontiguousarray(dist, np.float64) if dist is not None else None
    p = XmPairs(_ptr(pairs), _ptr(d), len(pairs), len(pairs))
    _check(_lib.xm_pairs_write(path.encode(), ctypes.byref(p), mode, 1 if append else 0))


def alpha_table(sr_deg, zh_deg):
    n = int(np.ceil(180 / zh_deg))
    out = np.empty(n, np.float64)
    _check(_lib.xm_alpha_table(sr_deg, zh_deg, _ptr(out), n))
    return out


def filter_bounds(sr_deg):
    """(thr_hi, thr_lo) of the FP32 chord^2 filter at radius sr_deg (float32 values)."""
    hi, lo = ctypes.c_float(), ctypes.c_float()
    _check(_lib.xm_filter_bounds(sr_deg, ctypes.byref(hi), ctypes.byref(lo)))
    return np.float32(hi.value), np.float32(lo.value)


class DeviceSegment:
    """A zone-sorted segment resident on the GPU (Segment, Segment.h:22-41)."""

    def __init__(self, ctx, handle):
        self._ctx = ctx
        self._h = handle

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("segment was freed")
        return self._h

    def info(self):
        sid, n, nz, zh = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_int32(), ctypes.c_double()
        _check(_lib.xm_segment_info(self.handle, ctypes.byref(sid), ctypes.byref(n), ctypes.byref(nz),
                                    ctypes.byref(zh)))
        return {"seg_id": sid.value, "n": n.value, "n_zones": nz.value, "zh_deg": zh.value}

    def __len__(self):
        return self.info()["n"]

    def export(self):
        """(id[n], radec_rad[n,2], zone_begin[n_zones], zone_end[n_zones]) -- Sorter.cu:178-182."""
        inf = self.info()
        n, nz = inf["n"], inf["n_zones"]
        ids = np.empty(max(n, 1), np.int64)
        radec = np.empty((max(n, 1), 2), np.float64)
        zb = np.empty(nz, np.int32)
        ze = np.empty(nz, np.int32)
        _check(_lib.xm_segment_export(self.handle, _ptr(ids), _ptr(radec), _ptr(zb), _ptr(ze)), self._ctx._h)
        return ids[:n], radec[:n], zb, ze

    def rebuild_device(self, dev_ptr, n, stats=None):
        _check(_lib.xm_segment_rebuild_device(self.handle, ctypes.c_void_p(dev_ptr), n,
                                              ctypes.byref(stats) if stats is not None else None), self._ctx._h)

    # ---- host-resident segments (catalogs larger than device memory) ----
    def offload(self):
        """Move the sorted arrays to pinned host memory and free the device copy."""
        _check(_lib.xm_segment_offload(self.handle), self._ctx._h)

    def page_in(self):
        """Queue the copy back to the device (returns at once; later work waits for it)."""
        _check(_lib.xm_segment_page_in(self.handle), self._ctx._h)

    def page_out(self):
        """Free the device copy, keeping the host copy."""
        _check(_lib.xm_segment_page_out(self.handle), self._ctx._h)

    def resident(self):
        """(arrays in device memory, their bytes)."""
        on, nb = ctypes.c_int(), ctypes.c_uint64()
        _check(_lib.xm_segment_resident(self.handle, ctypes.byref(on), ctypes.byref(nb)))
        return bool(on.value), nb.value

    def free(self):
        if self._h is not None:
            _lib.xm_segment_free(self._h)
            self._h = None

    def __del__(self):
        try:
            if self._ctx._h is not None:
                self.free()
        except Exception:
            pass


class Server:
    """A resident catalog answering query catalogs (xm_serve_*): submit() queues a
    query and returns a ticket, poll() returns (pairs, dist, info) once it is done.
    The context is the server's until close()."""

    def __init__(self, ctx, catalog, mem_budget=0, max_batch=0, flags=XM_FILTER32):
        self.ctx = ctx
        self.catalog = catalog
        self.with_dist = (flags & XM_NO_DIST) == 0
        cfg = _capi.XmServeCfg(mem_budget, max_batch, flags)
        h = ctypes.c_void_p()
        _check(_lib.xm_serve_open(ctx._h, catalog.handle, ctypes.byref(cfg), ctypes.byref(h)), ctx._h)
        self._h = h

    def _check(self, status):
        if status != XM_OK:
            buf = ctypes.create_string_buffer(1024)
            _lib.xm_serve_last_error(self._h, buf, len(buf))
            raise XmatchError(status, buf.value.decode(errors="replace"))

    def submit(self, objs, sr_deg):
        objs = as_objs(objs)
        t = ctypes.c_uint64()
        self._check(_lib.xm_serve_submit(self._h, _ptr(objs), len(objs), sr_deg, ctypes.byref(t)))
        return t.value

    def poll(self, ticket, wait=True):
        """(pairs, dist, info dict), or None if not ready and wait is False."""
        info = _capi.XmServeInfo()
        p = XmPairs(None, None, 0, 0)
        rc = _lib.xm_serve_poll(self._h, ticket, 1 if wait else 0, ctypes.byref(p), ctypes.byref(info))
        if rc == _capi.XM_ERR_BUSY:
            return None
        self._check(rc)
        n = p.count
        pairs = np.empty((max(n, 1), 2), np.int64)
        dist = np.empty(max(n, 1), np.float64) if self.with_dist else None
        p = XmPairs(_ptr(pairs), _ptr(dist), n, 0)
        self._check(_lib.xm_serve_poll(self._h, ticket, 1, ctypes.byref(p), ctypes.byref(info)))
        return pairs[:n], (dist[:n] if self.with_dist else None), info.as_dict()

    def close(self):
        if self._h:
            _check(_lib.xm_serve_close(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Context:
    """One GPU (replaces CudaManager/CudaContext)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        _check(_lib.xm_ctx_create(device, ctypes.byref(h)))
        self._h = h
        self.device = device

    def close(self):
        if self._h is not None:
            _lib.xm_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        dev, sm, free, total = ctypes.c_int(), ctypes.c_int(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(_lib.xm_ctx_info(self._h, ctypes.byref(dev), ctypes.byref(sm), ctypes.byref(free),
                                ctypes.byref(total)))
        return {"device": dev.value, "sm_count": sm.value, "free": free.value, "total": total.value}

    def synchronize(self):
        _check(_lib.xm_ctx_synchronize(self._h), self._h)

    # ---- zone builder (Sorter::Sort) ----
    def build(self, objs, zh_deg, seg_id=0, stats=None):
        """Zone-build host records on the GPU; `stats` (XmStats) accumulates timings."""
        objs = as_objs(objs)
        h = ctypes.c_void_p()
        _check(_lib.xm_segment_build(self._h, seg_id, _ptr(objs), len(objs), zh_deg, ctypes.byref(h),
                                     ctypes.byref(stats) if stats is not None else None), self._h)
        return DeviceSegment(self, h)

    def build_device(self, dev_ptr, n, zh_deg, seg_id=0, stats=None):
        """Build from n records already in this GPU's memory (e.g. a torch tensor's data_ptr())."""
        h = ctypes.c_void_p()
        _check(_lib.xm_segment_build_device(self._h, seg_id, ctypes.c_void_p(dev_ptr), n, zh_deg,
                                            ctypes.byref(h), ctypes.byref(stats) if stats is not None else None),
               self._h)
        return DeviceSegment(self, h)

    def stream(self):
        """The context's cudaStream_t as an integer (e.g. for torch.cuda.ExternalStream)."""
        s = ctypes.c_void_p()
        _check(_lib.xm_ctx_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    # ---- matching (Worker::Match) ----
    def match(self, A, B, sr_deg, flags=XM_FILTER32, fetch=True, with_dist=True, out=None):
        """Crossmatch segment A against B.  Returns (pairs[n,2] int64, dist[n] or None, stats dict).

        With fetch=False the pairs stay on the GPU and (None, None, stats) is returned.
        `out` may supply preallocated host arrays (pairs, dist) of sufficient capacity."""
        st = XmStats()
        if not with_dist:
            flags |= XM_NO_DIST
        if not fetch:
            p = XmPairs(None, None, 0, 0)
            _check(_lib.xm_match(self._h, A.handle, B.handle, sr_deg, flags, ctypes.byref(p), ctypes.byref(st)),
                   self._h)
            return None, None, st.as_dict()
        if out is not None:
            pairs, dist = out
        else:
            cap = 2 * max(len(A), len(B), 8)
            pairs = np.empty((cap, 2), np.int64)
            dist = np.empty(cap, np.float64) if with_dist else None
        p = XmPairs(_ptr(pairs), _ptr(dist) if with_dist else None, len(pairs), 0)
        rc = _lib.xm_match(self._h, A.handle, B.handle, sr_deg, flags, ctypes.byref(p), ctypes.byref(st))
        if rc == _capi.XM_ERR_CAPACITY and out is None:
            n = p.count
            pairs = np.empty((n, 2), np.int64)
            dist = np.empty(n, np.float64) if with_dist else None
            p = XmPairs(_ptr(pairs), _ptr(dist) if with_dist else None, n, 0)
            rc = _lib.xm_fetch_pairs(self._h, ctypes.byref(p))
        _check(rc, self._h)
        n = p.count
        return pairs[:n], (dist[:n] if with_dist else None), st.as_dict()

    def fetch(self, n, with_dist=True):
        pairs = np.empty((n, 2), np.int64)
        dist = np.empty(n, np.float64) if with_dist else None
        p = XmPairs(_ptr(pairs), _ptr(dist), n, 0)
        _check(_lib.xm_fetch_pairs(self._h, ctypes.byref(p)), self._h)
        return pairs[:p.count], (dist[:p.count] if with_dist else None)

    def _jobs(self, jobs):
        arr = (XmJob * len(jobs))()
        for k, (a, b, r) in enumerate(jobs):
            arr[k] = XmJob(a.handle, b.handle, r)
        return arr

    def match_batch(self, jobs, flags=XM_FILTER32, tuning=None, fetch=True, with_dist=True):
        """jobs: list of (A, B, sr_deg).  Returns (list of (pairs, dist), counts, stats)."""
        arr = self._jobs(jobs)
        nj = len(jobs)
        if not with_dist:
            flags |= XM_NO_DIST
        t = XmTuning(*tuning) if tuning else None
        counts = (ctypes.c_uint64 * max(nj, 1))()
        st = XmStats()
        _check(_lib.xm_match_batch(self._h, arr, nj, flags, ctypes.byref(t) if t else None, None, counts,
                                   ctypes.byref(st)), self._h)
        cnt = [counts[k] for k in range(nj)]
        if not fetch:
            return None, cnt, st.as_dict()
        pairs, dist = self.fetch(sum(cnt), with_dist)
        res, o = [], 0
        for c in cnt:
            res.append((pairs[o:o + c], dist[o:o + c] if with_dist else None))
            o += c
        return res, cnt, st.as_dict()

    def autotune(self, jobs, flags=XM_FILTER32):
        arr = self._jobs(jobs)
        best = XmTuning()
        bms, fms = ctypes.c_float(), ctypes.c_float()
        _check(_lib.xm_autotune_batch(self._h, arr, len(jobs), flags, ctypes.byref(best), ctypes.byref(bms),
                                      ctypes.byref(fms)), self._h)
        return (best.tile, best.chunk, best.blocks_per_sm, best.zones), bms.value, fms.value

    def crossmatch(self, A, B, sr_deg, zh_deg=None, flags=XM_FILTER32, with_dist=True, out=None):
        """Both catalogs from host records to matches (xm_crossmatch): (pairs, dist, stats).
        `out` = (pairs[n,2] int64, dist[n] or None); pinned arrays (e.g. from torch's
        pin_memory) are written by the pair kernel directly."""
        A, B = as_objs(A), as_objs(B)
        if not with_dist:
            flags |= XM_NO_DIST
        if out is not None:
            pairs, dist = out
        else:
            cap = 2 * max(len(A), len(B), 8)
            pairs = np.empty((cap, 2), np.int64)
            dist = np.empty(cap, np.float64) if with_dist else None
        st = XmStats()
        p = XmPairs(_ptr(pairs), _ptr(dist) if with_dist else None, len(pairs), 0)
        rc = _lib.xm_crossmatch(self._h, _ptr(A), len(A), _ptr(B), len(B), sr_deg, zh_deg or sr_deg, flags,
                                ctypes.byref(p), ctypes.byref(st))
        if rc == _capi.XM_ERR_CAPACITY and out is None:
            n = p.count
            pairs = np.empty((n, 2), np.int64)
            dist = np.empty(n, np.float64) if with_dist else None
            p = XmPairs(_ptr(pairs), _ptr(dist) if with_dist else None, n, 0)
            rc = _lib.xm_fetch_pairs(self._h, ctypes.byref(p))
        _check(rc, self._h)
        n = p.count
        return pairs[:n], (dist[:n] if with_dist else None), st.as_dict()

    def unit_vectors(self, ra_deg, dec_deg):
        ra = np.ascontiguousarray(ra_deg, np.float64)
        de = np.ascontiguousarray(dec_deg, np.float64)
        out = np.empty((len(ra), 3), np.float64)
        _check(_lib.xm_unit_vectors(self._h, _ptr(ra), _ptr(de), len(ra), _ptr(out)), self._h)
        return out


def crossmatch(A, B, r_arcsec, zh_arcsec=None, device=0, flags=XM_FILTER32, ctx=None):
    """One-shot crossmatch of two catalogs (arcsec, as the reference CLI)."""
    zh = (zh_arcsec or r_arcsec) / 3600.0
    own = ctx is None
    ctx = ctx or Context(device)
    try:
        return ctx.crossmatch(A, B, r_arcsec / 3600.0, zh, flags)
    finally:
        if own:
            ctx.close()
