"""Serving (xm_serve_*): a resident catalog answers query catalogs submitted
while others are in flight.  Each query's result in the mix must equal its
result alone (xm_match of the query segment against the catalog) and the
oracle's, bit for bit in the pair set and within 1e-12 rad in distance."""
import threading

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

ARCSEC = 1.0 / 3600.0
ZH = 2 * ARCSEC


def sp(p, d):
    o = np.lexsort((p[:, 1], p[:, 0]))
    return p[o], d[o]


def make_queries(cat, k, seed):
    from xmatch_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for j in range(k):
        n = int(np.exp(rng.uniform(np.log(50), np.log(20_000))))
        src = rng.integers(0, len(cat), n)
        ra, dec = synth.perturb(rng, cat["ra"][src], cat["dec"][src], rng.uniform(0.2, 2.0) * ARCSEC)
        q = np.empty(n, cat.dtype)
        q["id"] = np.arange(n) + 1_000_000 * (j + 1)
        q["ra"], q["dec"] = ra, dec
        out.append((q, rng.uniform(0.5, 5.0) * ARCSEC))
    return out


@pytest.fixture(scope="module")
def catalog():
    from xmatch_b200 import synth
    A, _ = synth.config0(n_a=200_000, n_b=1000, seed=77)
    return A


def alone(ctx, cat_seg, queries):
    res = []
    for q, r in queries:
        s = ctx.build(q, ZH, 9)
        p, d, _ = ctx.match(s, cat_seg, r)
        s.free()
        res.append(sp(p, d))
    return res


@pytest.mark.parametrize("budget", [0, 4 << 20])
def test_mix_equals_alone(catalog, budget):
    import xmatch_b200 as xm
    queries = make_queries(catalog, 24, seed=5)
    with xm.Context(0) as ctx:
        cat = ctx.build(catalog, ZH, 0)
        ref = alone(ctx, cat, queries)
        srv = xm.Server(ctx, cat, mem_budget=budget)
        tickets = [srv.submit(q, r) for q, r in queries]
        got = [srv.poll(t) for t in tickets]
        srv.close()
        cat.free()
    sizes = []
    for (p, d, info), (pr, dr) in zip(got, ref):
        p, d = sp(p, d)
        assert np.array_equal(p, pr) and d.tobytes() == dr.tobytes()
        assert info["count"] == len(p)
        assert info["t_submit_ms"] <= info["t_admit_ms"] <= info["t_done_ms"]
        sizes.append(info["batch_size"])
    if budget == 0:
        assert max(sizes) > 1     # a burst is batched
    for (q, r), (pr, dr) in zip(queries[:6], ref[:6]):
        po, do, _ = oracle.xmatch(q, catalog, r, ZH)
        po, do = sp(po, do)
        assert np.array_equal(po, pr) and np.max(np.abs(do - dr), initial=0) <= 1e-12


def test_concurrent_submitters_and_nonblocking_poll(catalog):
    import xmatch_b200 as xm
    queries = make_queries(catalog, 40, seed=9)
    with xm.Context(0) as ctx:
        cat = ctx.build(catalog, ZH, 0)
        ref = alone(ctx, cat, queries)
        srv = xm.Server(ctx, cat, max_batch=8)
        tickets = [None] * len(queries)

        def submit(part):
            for k in part:
                tickets[k] = srv.submit(*queries[k])
        th = [threading.Thread(target=submit, args=(range(s, len(queries), 2),)) for s in (0, 1)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        got = {}
        while len(got) < len(queries):
            for k, t in enumerate(tickets):
                if k not in got:
                    r = srv.poll(t, wait=False)
                    if r is not None:
                        got[k] = r
        srv.close()
        cat.free()
    for k, (pr, dr) in enumerate(ref):
        p, d = sp(got[k][0], got[k][1])
        assert np.array_equal(p, pr) and d.tobytes() == dr.tobytes()
        assert got[k][2]["batch_size"] <= 8


def test_query_larger_than_budget_is_refused(catalog):
    import xmatch_b200 as xm
    q, r = make_queries(catalog, 1, seed=3)[0]
    with xm.Context(0) as ctx:
        cat = ctx.build(catalog, ZH, 0)
        srv = xm.Server(ctx, cat, mem_budget=1024)
        with pytest.raises(xm.XmatchError):
            srv.submit(q, r)
        srv.close()
        cat.free()
