"""GPU parity: every result of the CUDA path (through the C ABI) against the
oracle on the same inputs.  Pair sets and sorted segments must be
bit-identical; distances within 1e-12 rad."""
import os

import numpy as np
import pytest

import oracle
from oracle import OBJ_DTYPE

pytestmark = pytest.mark.gpu

ARCSEC = 1.0 / 3600.0
DIST_TOL = 1e-12   # radians


def sp(p, d=None):
    o = np.lexsort((p[:, 1], p[:, 0]))
    return (p[o], d[o]) if d is not None else p[o]


def objs(ids, ra, dec):
    o = np.empty(len(ids), OBJ_DTYPE)
    o["id"], o["ra"], o["dec"] = ids, ra, dec
    return o


def run_gpu(ctx, A, B, r_arcsec, zh_arcsec=None, flags=0, tuning=None):
    import xmatch_b200 as xm
    zh = (zh_arcsec or r_arcsec) * ARCSEC
    sa = ctx.build(A, zh, 0)
    sb = ctx.build(B, zh, 1)
    if tuning is None:
        p, d, st = ctx.match(sa, sb, r_arcsec * ARCSEC, flags | xm.XM_COUNT_CAND)
    else:
        res, cnt, st = ctx.match_batch([(sa, sb, r_arcsec * ARCSEC)], flags | xm.XM_COUNT_CAND, tuning=tuning)
        p, d = res[0]
    sa.free()
    sb.free()
    return p, d, st


def check_parity(ctx, A, B, r_arcsec, zh_arcsec=None, variants=(0, 1), tuning=None):
    po, do, so = oracle.xmatch(A, B, r_arcsec * ARCSEC, (zh_arcsec or r_arcsec) * ARCSEC)
    po, do = sp(po, do)
    for flags in variants:
        p, d, st = run_gpu(ctx, A, B, r_arcsec, zh_arcsec, flags, tuning)
        p, d = sp(p, d)
        assert len(p) == len(po), (flags, len(p), len(po))
        assert np.array_equal(p, po), flags
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL
        assert st["n_cand"] == so.n_cand, (flags, st["n_cand"], so.n_cand)
        assert st["n_match"] == len(po)
    return po, so


def test_unit_vectors_bit_exact(ctx):
    rng = np.random.default_rng(11)
    ra = np.concatenate([rng.uniform(0, 360, 100_000), [0.0, -0.0, 90.0, 180.0, 270.0, 359.9999999, 1e-300]])
    dec = np.concatenate([rng.uniform(-90, 90, 100_000), [0.0, 0.0, 90.0, -90.0, 45.0, -1e-12, 0.0]])
    g = ctx.unit_vectors(ra, dec)
    o = oracle.unit_vectors(ra, dec)
    assert g.tobytes() == o.tobytes()


@pytest.mark.parametrize("zh_arcsec", [1, 5, 30])
def test_segment_build_matches_oracle(ctx, fixtures, zh_arcsec):
    a, _ = fixtures
    seg = ctx.build(a, zh_arcsec * ARCSEC)
    ids, radec, zb, ze = seg.export()
    oid, ordec, ozb, oze = oracle.build_export(a, zh_arcsec * ARCSEC)
    assert np.array_equal(ids, oid)
    assert radec.tobytes() == ordec.tobytes()
    assert np.array_equal(zb, ozb) and np.array_equal(ze, oze)
    seg.free()


@pytest.mark.parametrize("r", [1, 5, 30])
def test_fixture_self_match(ctx, fixtures, golden_dir, r):
    a, _ = fixtures
    po, _ = check_parity(ctx, a, a, r)
    f = os.path.join(golden_dir, "pairs_test_x_test_r%d.npz" % r)
    if os.path.exists(f):
        assert np.array_equal(po, np.load(f)["pairs"])


@pytest.mark.parametrize("r", [1, 5, 30])
def test_fixture_cross_match(ctx, fixtures, r):
    a, a2 = fixtures
    check_parity(ctx, a2, a, r)
    check_parity(ctx, a, a2, r)


def test_config0_shape_small(ctx):
    from xmatch_b200 import synth
    A, B = synth.config0(n_a=50_000, n_b=50_000, seed=5)
    check_parity(ctx, A, B, 3)


def test_wrap_and_pole_dense(ctx):
    rng = np.random.default_rng(12)
    n = 20_000
    ra = np.concatenate([rng.uniform(0, 0.01, n), rng.uniform(359.99, 360, n), rng.uniform(0, 360, n)])
    ra = np.where(ra >= 360, 0.0, ra)
    dec = np.concatenate([rng.uniform(-1, 1, 2 * n), rng.uniform(89.9, 90.0, n)])
    A = objs(np.arange(3 * n), ra, dec)
    B = objs(np.arange(3 * n) + 10 ** 9, (ra + rng.normal(0, 1e-4, 3 * n)) % 360.0,
             np.clip(dec + rng.normal(0, 1e-4, 3 * n), -90, 90))
    for r in (1, 10):
        check_parity(ctx, A, B, r)


def test_south_pole_and_full_ring_zones(ctx):
    rng = np.random.default_rng(13)
    n = 5000
    A = objs(np.arange(n), rng.uniform(0, 360, n), -90 + rng.uniform(0, 0.02, n))
    B = objs(np.arange(n) + 10 ** 6, rng.uniform(0, 360, n), -90 + rng.uniform(0, 0.02, n))
    check_parity(ctx, A, B, 20)


def test_zone_height_differs_from_radius(ctx, fixtures):
    a, a2 = fixtures
    check_parity(ctx, a2, a, 5, zh_arcsec=2)      # nz = 3
    check_parity(ctx, a2, a, 5, zh_arcsec=7.5)    # nz = 1, zones taller than r


def test_oversize_zones(ctx):
    # every source in one 10" zone: zones far larger than the shared-memory sort chunk
    rng = np.random.default_rng(14)
    n = 30_000
    A = objs(np.arange(n), rng.uniform(0, 2, n), rng.uniform(0, 0.0027, n))
    B = objs(np.arange(n) + 10 ** 6, rng.uniform(0, 2, n), rng.uniform(0, 0.0027, n))
    check_parity(ctx, A, B, 10, variants=(0,))
    seg = ctx.build(A, 10 * ARCSEC)
    ids, radec, zb, ze = seg.export()
    oid, ordec, ozb, oze = oracle.build_export(A, 10 * ARCSEC)
    assert np.array_equal(ids, oid) and radec.tobytes() == ordec.tobytes()
    seg.free()


def _zone_mix(rng):
    # zones of 1 .. 300 objects (warp path), one of 5000 (block path), and input
    # in dec order so that neighbouring records share a zone
    zh = 2 * ARCSEC
    sizes = np.concatenate([np.arange(1, 301), [5000]])
    zone = np.repeat(np.arange(len(sizes)) * 3 + 20_000, sizes)
    dec = -90 + (zone + rng.uniform(0.1, 0.9, len(zone))) * zh
    ra = rng.uniform(0, 360, len(zone))
    ra[: len(ra) // 7] = 180.0            # ties in ra inside a zone
    return objs(np.arange(len(zone)), ra, dec), zh


@pytest.mark.parametrize("case", ["mix_sorted", "mix_shuffled", "one_zone_8192", "one_zone_8193"])
def test_build_paths_match_oracle_export(ctx, case):
    rng = np.random.default_rng(21)
    if case.startswith("mix"):
        A, zh = _zone_mix(rng)
        if case == "mix_shuffled":
            A = A[rng.permutation(len(A))]
    else:
        n = int(case.rsplit("_", 1)[1])   # 8192 = largest zone of the block sort
        zh = 10 * ARCSEC
        A = objs(np.arange(n), rng.uniform(0, 360, n), rng.uniform(0, 0.0027, n))
    seg = ctx.build(A, zh)
    ids, radec, zb, ze = seg.export()
    oid, ordec, ozb, oze = oracle.build_export(A, zh)
    assert np.array_equal(ids, oid) and radec.tobytes() == ordec.tobytes()
    assert np.array_equal(zb, ozb) and np.array_equal(ze, oze)
    seg.free()
    check_parity(ctx, A, A, zh / ARCSEC, variants=(0,))


def test_empty_single_and_dropped(ctx):
    E = np.empty(0, OBJ_DTYPE)
    one = objs([7], [10.0], [10.0])
    bad = objs([1, 2, 3, 4, 5], [0.0, 0.0, np.nan, 5.0, np.inf], [90.0, 91.0, 0.0, np.nan, 1.0])
    north = objs([9], [200.0], [90.0])
    for x, y in ((E, E), (E, one), (one, E), (one, one), (bad, north), (bad, bad)):
        check_parity(ctx, x, y, 1)


def test_duplicate_coordinates(ctx):
    # identical (ra, dec) for many ids: ties in the sort key, zero distances
    n = 3000
    A = objs(np.arange(n), np.full(n, 123.456), np.full(n, -33.3))
    check_parity(ctx, A, A, 1, variants=(0,))


@pytest.mark.parametrize("tile,chunk,zones", [(64, 1, 1), (128, 16, 16), (256, 32, 64)])
def test_tuning_does_not_change_results(ctx, fixtures, tile, chunk, zones):
    a, _ = fixtures
    check_parity(ctx, a, a, 5, variants=(0,), tuning=(tile, chunk, 0, zones))


def test_output_growth_never_truncates():
    # 2,500 sources inside 20": every pair matches at r = 60" (6.25 M pairs,
    # far beyond the initial 2 * max(nA, nB) buffer of a fresh context)
    import xmatch_b200 as xm
    rng = np.random.default_rng(15)
    n = 2500
    A = objs(np.arange(n), 100 + rng.uniform(0, 20 * ARCSEC, n), 20 + rng.uniform(0, 20 * ARCSEC, n))
    with xm.Context(0) as fresh:
        p, d, st = run_gpu(fresh, A, A, 60)
    assert len(p) == n * n
    assert st["n_retries"] >= 1
    po, do, _ = oracle.xmatch(A, A, 60 * ARCSEC)
    assert np.array_equal(sp(p), sp(po))


def test_capacity_error_reports_count(ctx, fixtures):
    import ctypes
    import xmatch_b200 as xm
    a, _ = fixtures
    sa = ctx.build(a, 5 * ARCSEC)
    small = np.empty((10, 2), np.int64)
    p = xm.XmPairs(small.ctypes.data, None, 10, 0)
    rc = xm._lib.xm_match(ctx._h, sa.handle, sa.handle, 5 * ARCSEC, 0, ctypes.byref(p), None)
    assert rc == xm._capi.XM_ERR_CAPACITY and p.count == 10980
    pairs, dist = ctx.fetch(p.count)     # the result is still on the device
    assert len(pairs) == 10980
    sa.free()


def test_mismatched_zone_heights_rejected(ctx, fixtures):
    import xmatch_b200 as xm
    a, _ = fixtures
    s1 = ctx.build(a, 1 * ARCSEC)
    s2 = ctx.build(a, 2 * ARCSEC)
    with pytest.raises(xm.XmatchError) as e:
        ctx.match(s1, s2, ARCSEC)
    assert e.value.status == xm._capi.XM_ERR_MISMATCH
    s1.free()
    s2.free()


def test_batch_equals_single_jobs(ctx, fixtures):
    from xmatch_b200 import synth
    jobs = synth.config2_jobs(n_jobs=12, seed=3, scale=0.1)
    segs = []
    for A, B, r in jobs:
        zh = r * ARCSEC
        segs.append((ctx.build(A, zh), ctx.build(B, zh), r * ARCSEC))
    res, cnt, st = ctx.match_batch(segs)
    for k, (A, B, r) in enumerate(jobs):
        po, do, _ = oracle.xmatch(A, B, r * ARCSEC)
        p, d = res[k]
        assert cnt[k] == len(po)
        p, d = sp(p, d)
        po, do = sp(po, do)
        assert np.array_equal(p, po)
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL
    for a, b, _ in segs:
        a.free()
        b.free()


def test_graph_and_direct_launches_agree(ctx, fixtures):
    # the match sequence runs as the context's CUDA graph unless XM_NO_GRAPH; a
    # second shape (other radius) exercises the graph update
    import xmatch_b200 as xm
    a, a2 = fixtures
    for r in (5, 20, 5):
        pg, dg, sg = run_gpu(ctx, a2, a, r, flags=0)
        pd, dd, sd = run_gpu(ctx, a2, a, r, flags=xm.XM_NO_GRAPH)
        pg, dg = sp(pg, dg)
        pd, dd = sp(pd, dd)
        assert np.array_equal(pg, pd) and dg.tobytes() == dd.tobytes()
        assert sg["n_cand"] == sd["n_cand"] and sg["n_tested"] == sd["n_tested"]


def test_batch_of_many_radii(ctx):
    # 200 jobs, each with its own radius and zone height: one alpha table per
    # job's zone range, one launch
    from xmatch_b200 import synth
    jobs = synth.config2_jobs(n_jobs=200, seed=11, scale=0.02)
    segs = [(ctx.build(A, r * ARCSEC), ctx.build(B, r * ARCSEC), r * ARCSEC) for A, B, r in jobs]
    res, cnt, st = ctx.match_batch(segs)
    for k, (A, B, r) in enumerate(jobs):
        po, do, _ = oracle.xmatch(A, B, r * ARCSEC)
        p, d = sp(*res[k])
        po, do = sp(po, do)
        assert cnt[k] == len(po) and np.array_equal(p, po), k
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL
    for x, y, _ in segs:
        x.free()
        y.free()


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("with_dist", [True, False])
def test_crossmatch_one_call(ctx, fixtures, pinned, with_dist):
    # host records in, matches out; pinned output buffers are written by the pair kernel directly
    import torch
    import xmatch_b200 as xm
    a, a2 = fixtures
    r = 5 * ARCSEC
    po, do, _ = oracle.xmatch(a2, a, r)
    po, do = sp(po, do)
    cap = len(po) + 100
    if pinned:
        P = torch.empty(cap * 2, dtype=torch.int64, pin_memory=True).numpy().reshape(-1, 2)
        D = torch.empty(cap, dtype=torch.float64, pin_memory=True).numpy() if with_dist else None
    else:
        P = np.empty((cap, 2), np.int64)
        D = np.empty(cap, np.float64) if with_dist else None
    p, d, st = ctx.crossmatch(a2, a, r, flags=xm.XM_FILTER32, with_dist=with_dist, out=(P, D))
    if with_dist:
        p, d = sp(p, d)
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL
    else:
        p = sp(p)
    assert np.array_equal(p, po)
    assert st["n_match"] == len(po)
    # output too small: the count is reported and the matches wait on the device
    small = np.empty((10, 2), np.int64)
    with pytest.raises(xm.XmatchError) as e:
        ctx.crossmatch(a2, a, r, with_dist=False, out=(small, None))
    assert e.value.status == xm._capi.XM_ERR_CAPACITY
    q, _ = ctx.fetch(len(po), with_dist=False)
    assert np.array_equal(sp(q), po)


def test_crossmatch_streams_a_in_chunks(ctx, fixtures, monkeypatch):
    # 2,000-object chunks: A (10,000) streamed in 5 chunks through 2 staging slots
    import torch
    monkeypatch.setenv("XMATCH_CHUNK_OBJS", "2000")
    a, a2 = fixtures
    r = 5 * ARCSEC
    po, do, _ = oracle.xmatch(a, a2, r)
    po, do = sp(po, do)
    cap = len(po) + 10
    P = torch.empty(cap * 2, dtype=torch.int64, pin_memory=True).numpy().reshape(-1, 2)
    D = torch.empty(cap, dtype=torch.float64, pin_memory=True).numpy()
    for _ in range(2):
        p, d, st = ctx.crossmatch(a, a2, r, out=(P, D))
        p, d = sp(p, d)
        assert np.array_equal(p, po) and np.max(np.abs(d - do), initial=0) <= DIST_TOL
    # explicit schedules: the largest chunk not the first (the staging slots take
    # the largest), a chunk of one object, an empty chunk; rings of 2, 3 and 5 slots
    for w, slots in (("1,3,1", "2"), ("9997,1,2", "3"), ("1,0.00001,1", "2"), ("5,1,4,2,3,1,1", "3"),
                     ("1,1,1,1,1", "5")):
        monkeypatch.setenv("XMATCH_CHUNK_WEIGHTS", w)
        monkeypatch.setenv("XMATCH_CHUNK_SLOTS", slots)
        p, d, st = ctx.crossmatch(a, a2, r, out=(P, D))
        p, d = sp(p, d)
        assert np.array_equal(p, po) and np.max(np.abs(d - do), initial=0) <= DIST_TOL
    monkeypatch.delenv("XMATCH_CHUNK_WEIGHTS")
    monkeypatch.delenv("XMATCH_CHUNK_SLOTS")
    # room for fewer than all: the whole match reruns into device buffers, the count is reported
    import xmatch_b200 as xm
    with pytest.raises(xm.XmatchError) as e:
        ctx.crossmatch(a, a2, r, out=(P[: len(po) // 2], D[: len(po) // 2]))
    assert e.value.status == xm._capi.XM_ERR_CAPACITY
    q, dq = ctx.fetch(len(po))
    q, dq = sp(q, dq)
    assert np.array_equal(q, po)


def test_crossmatch_dense_chunks(ctx, monkeypatch):
    # a dense patch streamed in 4,000-object chunks of A with about 9 matches per
    # object: each chunk's ~36,000 matches written into the caller's pinned buffers
    # after those of the chunks before it
    import torch
    from xmatch_b200 import synth
    monkeypatch.setenv("XMATCH_CHUNK_OBJS", "4000")
    rng = np.random.default_rng(41)
    n = 20_000
    A = synth.make_objs(np.arange(n, dtype=np.int64), rng.uniform(10.0, 10.2, n), rng.uniform(-0.1, 0.1, n))
    B = synth.make_objs(np.arange(n, dtype=np.int64) + 10**9, rng.uniform(10.0, 10.2, n), rng.uniform(-0.1, 0.1, n))
    r = 30 * ARCSEC
    po, do, _ = oracle.xmatch(A, B, r)
    po, do = sp(po, do)
    assert len(po) > 5 * (2 * 4000 + 1024)
    cap = len(po) + 10
    P = torch.empty(cap * 2, dtype=torch.int64, pin_memory=True).numpy().reshape(-1, 2)
    D = torch.empty(cap, dtype=torch.float64, pin_memory=True).numpy()
    p, d, st = ctx.crossmatch(A, B, r, out=(P, D))
    p, d = sp(p, d)
    assert np.array_equal(p, po) and np.max(np.abs(d - do), initial=0) <= DIST_TOL
    assert st["n_match"] == len(po)


def test_crossmatch_config1_mixture_4M(ctx):
    # one call from pinned host records to pinned host pairs, 4.5M objects a side of
    # the config-1 mixture (clusters, wrap and polar sources)
    import torch
    from xmatch_b200 import synth
    A, B = synth.config1(n=4_500_000, seed=23)
    r = ARCSEC
    po, _, _ = oracle.xmatch(A, B, r, r)
    po = sp(po)
    cap = len(po) + 10
    P = torch.empty(cap * 2, dtype=torch.int64, pin_memory=True).numpy().reshape(-1, 2)
    p, _, st = ctx.crossmatch(A, B, r, zh_deg=r, with_dist=False, out=(P, None))
    assert np.array_equal(sp(p), po)
    assert st["n_match"] == len(po)


def test_segmentation_invariance(ctx, fixtures):
    a, _ = fixtures
    whole, _, _ = oracle.xmatch(a, a, 5 * ARCSEC)
    zh = 5 * ARCSEC
    segs = [ctx.build(a[s:s + 2020], zh, k) for k, s in enumerate(range(0, len(a), 2020))]
    jobs = [(x, y, 5 * ARCSEC) for x in segs for y in segs]
    res, cnt, _ = ctx.match_batch(jobs)
    allp = np.concatenate([r[0] for r in res])
    assert np.array_equal(sp(allp), sp(whole))
    for s in segs:
        s.free()


def test_offloaded_segments_page_in_per_job(ctx, fixtures):
    """Segments moved to pinned host memory and paged back in (the next one's copy
    queued while the current job matches) give the pairs of resident segments;
    an offloaded segment is refused by the match and still exports."""
    import xmatch_b200 as xm
    a, a2 = fixtures
    zh = 5 * ARCSEC
    segs = [ctx.build(a[s:s + 2500], zh, k) for k, s in enumerate(range(0, len(a), 2500))]
    B = ctx.build(a2, zh, 9)
    want = [sp(ctx.match(s, B, zh, with_dist=False)[0]) for s in segs]
    ids0 = segs[0].export()
    for s in segs:
        s.offload()
        assert s.resident()[0] is False
    assert np.array_equal(segs[0].export()[0], ids0[0])     # from the host copy
    with pytest.raises(xm.XmatchError):
        ctx.match(segs[0], B, zh)
    for rep in range(2):
        segs[0].page_in()
        for k, s in enumerate(segs):
            if k + 1 < len(segs):
                segs[k + 1].page_in()
            p = sp(ctx.match(s, B, zh, with_dist=False)[0])
            assert np.array_equal(p, want[k]), (rep, k)
            s.page_out()
    for s in segs:
        s.free()
    B.free()


@pytest.mark.parametrize("zh_arcsec", [15, 30, 60])
def test_bin_index_dense_zones(ctx, zh_arcsec):
    """Segments dense enough for the per-zone bin index (8, 16 and 32 bins per zone at
    these zone heights): the window search that starts inside the bin of the window's
    lower end gives the oracle's pairs, wraparound and polar zones included."""
    from xmatch_b200 import synth
    rng = np.random.default_rng(16)
    n = 800_000
    ra, dec = synth.uniform_sphere(rng, n)
    A = objs(np.arange(n), ra, dec)
    k = n // 2
    pra, pdec = synth.perturb(rng, ra[:k], dec[:k], 10 * ARCSEC)
    rra, rdec = synth.uniform_sphere(rng, n - k)
    B = objs(np.arange(n) + 10 ** 9, np.concatenate([pra, rra]), np.concatenate([pdec, rdec]))
    check_parity(ctx, A, B, zh_arcsec)


@pytest.mark.parametrize("zh_arcsec,r_arcsec", [(15, 60), (10, 120)])
def test_bin_index_radius_spanning_zones(ctx, zh_arcsec, r_arcsec):
    """Radius of several zone heights over segments with a bin index: windows in 9 and
    25 zones per object, searched in staged bands and (at 120") in global memory through
    the segment's bin rows, against the oracle."""
    from xmatch_b200 import synth
    rng = np.random.default_rng(17)
    n = 2_000_000
    ra, dec = synth.uniform_sphere(rng, n)
    A = objs(np.arange(n), ra, dec)
    k = n // 2
    pra, pdec = synth.perturb(rng, ra[:k], dec[:k], r_arcsec / 2 * ARCSEC)
    rra, rdec = synth.uniform_sphere(rng, n - k)
    B = objs(np.arange(n) + 10 ** 9, np.concatenate([pra, rra]), np.concatenate([pdec, rdec]))
    check_parity(ctx, A, B, r_arcsec, zh_arcsec=zh_arcsec, variants=(0,))
