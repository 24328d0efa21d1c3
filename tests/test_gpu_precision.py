"""Precision stress (config 3 shape): uniform catalogs plus planted pairs at
separation r (1 +- k 1e-9), k in 1..100.  The FP32-filter path and the plain
FP64 path must both return exactly the oracle's pair set, with distances
within 1e-12 rad.  Where the planted offset k 1e-9 r is at least 1e-13 rad
(all pairs at 60", none at 0.1", whose offsets of 5e-16 .. 5e-14 rad are at
the FP64 spacing of coordinates stored in degrees), every planted pair inside
r is found and none outside; below that the stored doubles decide, as in the
oracle."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

ARCSEC = 1.0 / 3600.0


def sp(p, d):
    o = np.lexsort((p[:, 1], p[:, 0]))
    return p[o], d[o]


@pytest.mark.parametrize("r_arcsec", [0.1, 60.0])
def test_planted_pairs_exact(ctx, r_arcsec):
    import xmatch_b200 as xm
    from xmatch_b200 import synth
    n, npl = 1_000_000, 100_000
    A, B, sign, k = synth.config3(n=n, n_planted=npl, r_arcsec=r_arcsec, seed=31)
    resolvable = k * 1e-9 * np.radians(r_arcsec * ARCSEC) >= 1e-13
    r = r_arcsec * ARCSEC
    po, do, so = oracle.xmatch(A, B, r, r)
    po, do = sp(po, do)
    sa, sb = ctx.build(A, r), ctx.build(B, r)
    for flags in (xm.XM_FILTER32, xm.XM_PLAIN64):
        p, d, st = ctx.match(sa, sb, r, flags | xm.XM_COUNT_CAND)
        p, d = sp(p, d)
        assert np.array_equal(p, po), (flags, len(p), len(po))
        assert np.max(np.abs(d - do), initial=0) <= 1e-12
        assert st["n_cand"] == so.n_cand
        hit = np.zeros(npl, bool)
        pl = (p[:, 0] >= n) & (p[:, 1] - 100_000_000_000 == p[:, 0])
        hit[p[pl, 0] - n] = True
        assert not np.any(hit & (sign > 0) & resolvable), "a planted pair outside r was matched"
        assert np.all(hit[(sign < 0) & resolvable]), "a planted pair inside r was missed"
        if flags == xm.XM_FILTER32:
            assert st["n_border"] > 0   # the planted pairs sit in the FP32 margin band
    sa.free()
    sb.free()
