"""The allocation-free zone build (xm_segment_build_noalloc) against the
regular one.

Some callers cannot allocate device memory once running -- a serving process
that reserved its HBM budget at start-up, or a host application whose device
memory belongs to another allocator.  They pass device input and output
arrays; the sort scratch is a fixed array inside the library.  This checks,
through the C ABI, that two calls in a row (different catalogs, so the second
call starts from the first call's leftovers in the shared scratch) give the
same segments as xm_segment_build + xm_segment_export.  Collected last on
purpose: the file name sorts after every other test file.
"""
import ctypes

import numpy as np
import pytest

import oracle
from oracle import OBJ_DTYPE

pytestmark = pytest.mark.gpu

ARCSEC = 1.0 / 3600.0


def _catalog(seed, n):
    rng = np.random.default_rng(seed)
    o = np.empty(n, OBJ_DTYPE)
    o["id"] = rng.permutation(n).astype(np.int64) + 7_000_000_000 * seed
    o["ra"] = rng.uniform(0, 360, n)
    o["dec"] = np.degrees(np.arcsin(rng.uniform(-1, 1, n)))
    o["ra"][:50] = np.nan          # dropped
    o["dec"][50:100] = 91.0        # dropped
    o["dec"][100:120] = 90.0       # kept in the last zone
    o["ra"][120:200] = 123.456     # ties in the sort key
    o["dec"][120:200] = -33.3
    return o


def _noalloc(objs, zh_deg):
    import torch
    import xmatch_b200 as xm
    n = len(objs)
    n_zones = int(np.ceil(180 / zh_deg))
    dev = torch.device("cuda", 0)
    d_in = torch.from_numpy(objs.view(np.uint8).copy()).to(dev)
    d_id = torch.empty(max(n, 1), dtype=torch.int64, device=dev)
    d_radec = torch.empty(2 * max(n, 1), dtype=torch.float64, device=dev)
    d_xyz = torch.empty(4 * max(n, 1), dtype=torch.float32, device=dev)
    d_zoff = torch.empty(n_zones + 1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize(dev)
    kept = ctypes.c_uint64()
    rc = xm._lib.xm_segment_build_noalloc(0, None, ctypes.c_void_p(d_in.data_ptr()), n, zh_deg,
                                          ctypes.c_void_p(d_id.data_ptr()), ctypes.c_void_p(d_radec.data_ptr()),
                                          ctypes.c_void_p(d_xyz.data_ptr()), ctypes.c_void_p(d_zoff.data_ptr()),
                                          n_zones + 1, ctypes.byref(kept))
    assert rc == 0, xm._lib.xm_status_str(rc)
    m = kept.value
    zoff = d_zoff.cpu().numpy().view(np.uint32).astype(np.int64)
    return (d_id[:m].cpu().numpy(), d_radec[:2 * m].cpu().numpy().reshape(-1, 2),
            d_xyz[:4 * m].cpu().numpy().reshape(-1, 4), zoff)


def test_noalloc_matches_regular_build(ctx):
    cases = [(_catalog(1, 300_000), 1.0 * ARCSEC), (_catalog(2, 120_000), 5.0 * ARCSEC)]
    for objs, zh in cases:   # two calls in a row through the shared scratch
        ids, radec, xyz, zoff = _noalloc(objs, zh)
        seg = ctx.build(objs, zh)
        rid, rradec, zb, ze = seg.export()
        seg.free()
        assert np.array_equal(ids, rid)
        assert radec.tobytes() == rradec.tobytes()          # FP64 bits
        assert np.array_equal(zoff[:-1], zb) and np.array_equal(zoff[1:], ze)
        oid, _, _, _ = oracle.build_export(objs, zh)
        assert np.array_equal(ids, oid)
        # FP32 unit vectors: the oracle's FP64 ones (same degree inputs) rounded to nearest
        order = {v: k for k, v in enumerate(objs["id"])}
        src = objs[[order[i] for i in ids]]
        ref = oracle.unit_vectors(src["ra"], src["dec"]).astype(np.float32)
        assert np.array_equal(xyz[:, :3], ref)


def test_noalloc_at_capacity(ctx):
    """Exactly XM_NOALLOC_MAX_OBJS records: the fixed scratch is full."""
    import xmatch_b200 as xm
    n = xm._capi.XM_NOALLOC_MAX_OBJS
    objs = _catalog(3, n)
    zh = 2.0 * ARCSEC
    ids, radec, xyz, zoff = _noalloc(objs, zh)
    seg = ctx.build(objs, zh)
    rid, rradec, zb, ze = seg.export()
    seg.free()
    assert len(ids) == n - 100        # 50 NaN ra and 50 dec = 91 dropped
    assert np.array_equal(ids, rid) and radec.tobytes() == rradec.tobytes()
    assert np.array_equal(zoff[:-1], zb) and np.array_equal(zoff[1:], ze)


def test_noalloc_empty_and_all_dropped(ctx):
    """n = 0, and an input whose every record is dropped: nothing kept, every
    zone offset 0."""
    zh = 5.0 * ARCSEC
    n_zones = int(np.ceil(180 / zh))
    ids, radec, xyz, zoff = _noalloc(np.empty(0, OBJ_DTYPE), zh)
    assert len(ids) == 0 and len(zoff) == n_zones + 1 and not zoff.any()
    bad = _catalog(4, 5000)
    bad["dec"] = 95.0
    ids, radec, xyz, zoff = _noalloc(bad, zh)
    assert len(ids) == 0 and not zoff.any()
    # and a regular call after them still agrees with the regular build
    objs = _catalog(5, 20_000)
    ids, radec, xyz, zoff = _noalloc(objs, zh)
    seg = ctx.build(objs, zh)
    rid, rradec, zb, ze = seg.export()
    seg.free()
    assert np.array_equal(ids, rid) and radec.tobytes() == rradec.tobytes()


def test_noalloc_rejects_small_zone_array_and_keeps_device(ctx):
    import torch
    import xmatch_b200 as xm
    zh = 5.0 * ARCSEC
    n_zones = int(np.ceil(180 / zh))
    objs = _catalog(6, 1000)
    dev = torch.device("cuda", 0)
    d_in = torch.from_numpy(objs.view(np.uint8).copy()).to(dev)
    out = [torch.empty(k * len(objs), dtype=t, device=dev)
           for k, t in ((1, torch.int64), (2, torch.float64), (4, torch.float32))]
    d_zoff = torch.empty(n_zones, dtype=torch.int32, device=dev)     # one entry short
    torch.cuda.synchronize(dev)
    kept = ctypes.c_uint64(12345)
    before = torch.cuda.current_device()
    rc = xm._lib.xm_segment_build_noalloc(0, None, ctypes.c_void_p(d_in.data_ptr()), len(objs), zh,
                                          *[ctypes.c_void_p(t.data_ptr()) for t in out],
                                          ctypes.c_void_p(d_zoff.data_ptr()), n_zones, ctypes.byref(kept))
    assert rc == xm._capi.XM_ERR_INVALID
    assert kept.value == 12345          # rejected before any work
    assert torch.cuda.current_device() == before


def test_noalloc_rejects_oversize(ctx):
    import xmatch_b200 as xm
    kept = ctypes.c_uint64()
    # null buffers: the size check comes first, and a null pointer is rejected before any launch
    rc = xm._lib.xm_segment_build_noalloc(0, None, None, xm._capi.XM_NOALLOC_MAX_OBJS + 1, 1.0,
                                          None, None, None, None, 8, ctypes.byref(kept))
    assert rc == xm._capi.XM_ERR_TOO_LARGE
    assert b"capacity" in xm._lib.xm_status_str(rc)
