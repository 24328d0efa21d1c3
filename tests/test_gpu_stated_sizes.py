"""Parity at the sizes the benchmark configurations state, on the GPU.

* config 0 at its full 200,000 x 200,000 (r = zh = 3"): the CUDA path (both
  kernel variants) against the oracle, and the reference's own kernel
  (Worker.cu, whole 16 x 16 blocks over the zone loop of Worker.cu:330-366)
  against the oracle;
* config 3 at its full 10M x 10M + 1M planted pairs, r = 0.1" and 60";
* config 1 at 2M x 2M pair for pair, and at its full 50M x 50M against the
  digest of the oracle's pair set (tests/golden/config1_pairset.json);
* config 2's 4,096 uneven jobs in one batch, every job pair for pair;
* the autotuner on an uneven batch.
Pair sets bit for bit, distances within 1e-12 rad.
"""
import json
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

ARCSEC = 1.0 / 3600.0
DIST_TOL = 1e-12   # radians
TWO_PI = 6.2831853071795864769252867665590057683943387987502116419498   # Worker.cu:23
RAD2DEG = 57.295779513082323                                              # Common.h:9
HERE = os.path.dirname(os.path.abspath(__file__))


def sp(p, d=None):
    o = np.lexsort((p[:, 1], p[:, 0]))
    return (p[o], d[o]) if d is not None else p[o]


def gpu_pairs(ctx, A, B, r, zh, flags):
    import xmatch_b200 as xm
    sa, sb = ctx.build(A, zh, 0), ctx.build(B, zh, 1)
    p, d, st = ctx.match(sa, sb, r, flags | xm.XM_COUNT_CAND, with_dist=not (flags & xm.XM_NO_DIST))
    sa.free()
    sb.free()
    return p, d, st


def assert_branch3_artefacts(A, B, only, r):
    """Pairs the reference kernel reports and the oracle does not must all come
    from the sign error of its wraparound branch 3 (Worker.cu:110-121): A near
    ra = 0, B near 2 pi, a true chord outside r that |y_b| brings inside."""
    if len(only) == 0:
        return
    ia = {v: k for k, v in enumerate(A["id"])}
    ib = {v: k for k, v in enumerate(B["id"])}
    a = A[[ia[x] for x in only[:, 0]]]
    b = B[[ib[x] for x in only[:, 1]]]
    ra1, de1 = a["ra"] / RAD2DEG, a["dec"] / RAD2DEG
    ra2, de2 = b["ra"] / RAD2DEG, b["dec"] / RAD2DEG
    x1, y1, z1 = np.cos(de1) * np.cos(ra1), np.cos(de1) * np.sin(ra1), np.sin(de1)
    x2, y2, z2 = np.cos(de2) * np.cos(ra2 + TWO_PI), np.cos(de2) * np.sin(ra2 + TWO_PI), np.sin(de2)
    d = 2 * np.sin(np.radians(r) / 2)
    T = d * d
    assert np.all(np.abs(ra1 - ra2 + TWO_PI) < np.radians(1.0))  # across ra = 0, A on the low side
    assert np.all((x1 - x2) ** 2 + (y1 - y2) ** 2 + (z1 - z2) ** 2 >= T * (1 - 1e-9))
    assert np.all((x1 - x2) ** 2 + (y1 - np.abs(y2)) ** 2 + (z1 - z2) ** 2 < T * (1 + 1e-9))


def test_config0_full_size(ctx):
    """200k x 200k, dec +-10 deg, r = zh = 3": bit-exact against the oracle and
    the reference's own kernel."""
    from oracle import ref_kernel
    from xmatch_b200 import synth
    A, B = synth.config0()
    assert len(A) == len(B) == 200_000
    r = 3 * ARCSEC
    po, do, so = oracle.xmatch(A, B, r, r)
    po, do = sp(po, do)
    assert len(po) > 100_000
    for flags in (0, 1):   # FILTER32, PLAIN64
        p, d, st = gpu_pairs(ctx, A, B, r, r, flags)
        p, d = sp(p, d)
        assert np.array_equal(p, po), (flags, len(p), len(po))
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL
        assert st["n_cand"] == so.n_cand
    if not ref_kernel.available():
        pytest.skip("oracle/_ref/libref_kernel.so not built (needs the reference tree at build time)")
    pr, _, _ = ref_kernel.xmatch(A, B, r, pad=True)
    sr = set(map(tuple, pr.tolist()))
    so_ = set(map(tuple, po.tolist()))
    assert so_ <= sr, "the reference kernel misses an oracle pair"
    only = np.array(sorted(sr - so_), np.int64).reshape(-1, 2)
    assert_branch3_artefacts(A, B, only, r)


@pytest.mark.parametrize("r_arcsec", [0.1, 60.0])
def test_config3_full_size(ctx, r_arcsec):
    """10M x 10M uniform + 1M planted pairs at r (1 +- k 1e-9): both variants equal
    the oracle; every planted pair whose offset is resolvable in FP64 (k 1e-9 r
    >= 1e-13 rad) is found exactly when it lies inside r."""
    import xmatch_b200 as xm
    from xmatch_b200 import synth
    n, npl = 10_000_000, 1_000_000
    A, B, sign, k = synth.config3(n=n, n_planted=npl, r_arcsec=r_arcsec)
    r = r_arcsec * ARCSEC
    po, do, so = oracle.xmatch(A, B, r, r)
    po, do = sp(po, do)
    resolvable = k * 1e-9 * np.radians(r) >= 1e-13
    sa, sb = ctx.build(A, r), ctx.build(B, r)
    got = {}
    for flags in (xm.XM_FILTER32, xm.XM_PLAIN64):
        p, d, st = ctx.match(sa, sb, r, flags | xm.XM_COUNT_CAND)
        p, d = sp(p, d)
        assert np.array_equal(p, po), (flags, len(p), len(po))
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL
        assert st["n_cand"] == so.n_cand
        hit = np.zeros(npl, bool)
        pl = (p[:, 0] >= n) & (p[:, 1] - 100_000_000_000 == p[:, 0])
        hit[p[pl, 0] - n] = True
        assert not np.any(resolvable & (hit != (sign < 0))), "a resolvable planted pair decided wrongly"
        got[flags] = p
    assert np.array_equal(got[xm.XM_FILTER32], got[xm.XM_PLAIN64])
    sa.free()
    sb.free()


def test_config1_mixture_2M(ctx):
    """The config-1 mixture (clusters, wrap and polar sources) at 2M x 2M, r = zh = 1",
    pair for pair against the oracle."""
    from xmatch_b200 import synth
    A, B = synth.config1(n=2_000_000, seed=7)
    r = ARCSEC
    po, do, so = oracle.xmatch(A, B, r, r)
    po, do = sp(po, do)
    for flags in (0, 1):
        p, d, st = gpu_pairs(ctx, A, B, r, r, flags)
        p, d = sp(p, d)
        assert np.array_equal(p, po), (flags, len(p), len(po))
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL
        assert st["n_cand"] == so.n_cand


@pytest.mark.slow
def test_config1_full_size_digest(ctx):
    """The headline 50M x 50M crossmatch: the GPU pair set's order-independent
    digest equals the one of the oracle's pair set recorded by
    tests/golden/make_config1_pairset.py."""
    import xmatch_b200 as xm
    from xmatch_b200 import pairhash, synth
    with open(os.path.join(HERE, "golden", "config1_pairset.json")) as f:
        g = json.load(f)
    A, B = synth.config1(n=g["n"], seed=g["seed"])
    if pairhash.inputs_fingerprint(A) != g["inputs"]["A"] or pairhash.inputs_fingerprint(B) != g["inputs"]["B"]:
        pytest.skip("the random generator no longer reproduces the recorded catalogs")
    r = g["r_arcsec"] * ARCSEC
    p, _, st = gpu_pairs(ctx, A, B, r, g["zh_arcsec"] * ARCSEC, xm.XM_NO_DIST)
    assert st["n_cand"] == g["candidates"]
    assert pairhash.pairset_digest(p) == g["digest"]


def oracle_jobs(jobs):
    """The oracle's result of every job, jobs spread over the host threads (one
    oracle thread each; the ctypes call releases the interpreter lock)."""
    from concurrent.futures import ThreadPoolExecutor

    def one(job):
        A, B, r = job
        po, do, _ = oracle.xmatch(A, B, r * ARCSEC, nthreads=1)
        return sp(po, do)
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        return list(ex.map(one, jobs))


def test_batch_4096_jobs_pair_for_pair(ctx):
    """4,096 uneven jobs (config 2's LogNormal sizes at a tenth of their scale,
    own dec band and radius each) in one batch: every job's pairs and distances
    equal the oracle's."""
    from xmatch_b200 import synth
    jobs = synth.config2_jobs(n_jobs=4096, scale=0.1)
    segs = [(ctx.build(A, r * ARCSEC), ctx.build(B, r * ARCSEC), r * ARCSEC) for A, B, r in jobs]
    res, cnt, st = ctx.match_batch(segs)
    assert len(res) == 4096
    for k, (po, do) in enumerate(oracle_jobs(jobs)):
        p, d = sp(*res[k])
        assert cnt[k] == len(po) and np.array_equal(p, po), k
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL, k
    for a, b, _ in segs:
        a.free()
        b.free()


def test_autotuner(ctx):
    """xm_autotune_batch on an uneven batch: the tuning it returns is no slower
    than the fixed one as it measured them, and gives the oracle's pair sets."""
    from xmatch_b200 import synth
    jobs = synth.config2_jobs(n_jobs=96, seed=17, scale=0.05)
    segs = [(ctx.build(A, r * ARCSEC), ctx.build(B, r * ARCSEC), r * ARCSEC) for A, B, r in jobs]
    tuning, best_ms, fixed_ms = ctx.autotune(segs)
    assert tuning[0] in (64, 128, 256) and 1 <= tuning[1] <= 32 and 1 <= tuning[3] <= 64
    assert 0 < best_ms <= fixed_ms
    res, cnt, _ = ctx.match_batch(segs, tuning=tuning)
    for k, (po, do) in enumerate(oracle_jobs(jobs)):
        p, d = sp(*res[k])
        assert np.array_equal(p, po), k
        assert np.max(np.abs(d - do), initial=0) <= DIST_TOL
    for a, b, _ in segs:
        a.free()
        b.free()
