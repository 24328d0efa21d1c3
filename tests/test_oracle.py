"""CPU tests of the oracle (the checker) against known answers and an
independent brute-force evaluation.  No GPU needed."""
import json
import os

import numpy as np
import pytest

import oracle
from oracle import OBJ_DTYPE

ARCSEC = 1.0 / 3600.0

# Match counts of the reference's two fixture catalogs computed independently
# of the oracle (a numpy restatement and a brute-force all-pairs FP64 chord
# test), self-pairs included, zh = r.
KNOWN_COUNTS = {
    ("test_x_test", 1): 10004, ("test_x_test", 5): 10980, ("test_x_test", 30): 41166,
    ("test2_x_test", 1): 1002, ("test2_x_test", 5): 1082, ("test2_x_test", 30): 4777,
    ("test2_x_test2", 1): 1002, ("test2_x_test2", 5): 1074, ("test2_x_test2", 30): 2748,
}


def _cases(fixtures):
    a, a2 = fixtures
    return {"test_x_test": (a, a), "test2_x_test": (a2, a), "test2_x_test2": (a2, a2)}


def sorted_pairs(p, d=None):
    o = np.lexsort((p[:, 1], p[:, 0]))
    return (p[o], d[o]) if d is not None else p[o]


def brute_force(A, B, r_deg):
    """All pairs, no zones: chord^2 of numpy unit vectors against (2 sin(r/2))^2."""
    def xyz(o):
        ra, de = np.radians(o["ra"]), np.radians(o["dec"])
        return np.stack([np.cos(de) * np.cos(ra), np.cos(de) * np.sin(ra), np.sin(de)], 1)
    xa, xb = xyz(A), xyz(B)
    t = (2 * np.sin(np.radians(r_deg) / 2)) ** 2
    out, near = [], 0
    for s in range(0, len(A), 512):
        d = xa[s:s + 512, None, :] - xb[None, :, :]
        c = (d * d).sum(-1)
        i, j = np.nonzero(c < t)
        out.append(np.stack([A["id"][s + i], B["id"][j]], 1))
        near += int(np.count_nonzero(np.abs(c / t - 1) < 1e-9))
    return np.concatenate(out), near


@pytest.mark.parametrize("name,r", sorted(KNOWN_COUNTS))
def test_known_counts_all_modes(fixtures, name, r):
    a, b = _cases(fixtures)[name]
    res = []
    for mode in (oracle.MODE_ALLPAIRS, oracle.MODE_ALLPAIRS_SINCOS, oracle.MODE_WINDOWED):
        p, d, st = oracle.xmatch(a, b, r * ARCSEC, mode=mode, nthreads=4)
        assert len(p) == KNOWN_COUNTS[(name, r)]
        res.append((sorted_pairs(p, d), st.n_cand))
    for k in (1, 2):
        assert np.array_equal(res[0][0][0], res[k][0][0])
        assert np.array_equal(res[0][0][1], res[k][0][1])   # identical FP64 bits
        assert res[0][1] == res[k][1]


def test_golden_counts_and_pairs(fixtures, golden_dir):
    cases = _cases(fixtures)
    with open(os.path.join(golden_dir, "known_counts.json")) as f:
        known = json.load(f)
    for key, v in known.items():
        name, r = key.rsplit("_r", 1)
        a, b = cases[name]
        p, d, st = oracle.xmatch(a, b, int(r) * ARCSEC)
        assert len(p) == v["matches"] and st.n_cand == v["candidates"]
        f = os.path.join(golden_dir, "pairs_%s.npz" % key)
        if os.path.exists(f):
            g = np.load(f)
            sp, sd = sorted_pairs(p, d)
            assert np.array_equal(sp, g["pairs"])
            assert np.array_equal(sd, g["dist"])


@pytest.mark.parametrize("r", [1, 5, 30])
def test_against_brute_force(fixtures, r):
    a, _ = fixtures
    p, _, _ = oracle.xmatch(a, a, r * ARCSEC)
    bf, near = brute_force(a, a, r * ARCSEC)
    assert near == 0   # no pair within 1e-9 of the threshold: both decisions must agree
    assert np.array_equal(sorted_pairs(p), sorted_pairs(bf))


def test_sincos_within_one_ulp():
    rng = np.random.default_rng(7)
    x = np.concatenate([rng.uniform(-7, 7, 200_000), rng.uniform(-1e-6, 1e-6, 1000),
                        np.arange(-8, 9) * np.pi / 4, [0.0, 1e-300, np.pi, 2 * np.pi]])
    s, c = oracle.sincos(x)
    for got, ref in ((s, np.sin(x)), (c, np.cos(x))):
        ulp = np.abs(got - ref) / np.spacing(np.maximum(np.abs(got), np.abs(ref)))
        assert ulp.max() <= 1.0


def test_unit_vectors_normalised():
    rng = np.random.default_rng(3)
    ra = rng.uniform(0, 360, 10000)
    dec = rng.uniform(-90, 90, 10000)
    v = oracle.unit_vectors(ra, dec)
    assert np.abs(np.linalg.norm(v, axis=1) - 1).max() < 4e-16


def test_alpha_formula():
    """calc_alpha of Common.cu:7-23: 180 sentinel above 89.99 deg, else
    atan(sin t)/sqrt(|cos(d-t) cos(d+t)|) with 1 % overshoot of t."""
    t = 5 * ARCSEC
    assert oracle.calc_alpha(t, 89.99) == 180
    d = 45.0
    want = abs(np.arctan(np.sin(np.radians(t))) / np.sqrt(abs(np.cos(np.radians(d - t)) * np.cos(np.radians(d + t)))))
    assert oracle.calc_alpha(t, d) == pytest.approx(want, rel=1e-15)
    tab = oracle.alpha_table(t, t)
    assert len(tab) == 129600
    # never smaller than the exact RA half-width of a circle of radius t at the zone edge
    z = np.arange(len(tab))
    dmax = np.maximum(np.abs(z * t - 90), np.abs((z + 1) * t - 90))
    ok = dmax + t < 89.99
    exact = np.arctan(np.sin(np.radians(t)) / np.sqrt(np.cos(np.radians(dmax[ok] - t)) * np.cos(np.radians(dmax[ok] + t))))
    assert np.all(tab[ok] >= exact)
    assert np.all(tab[~ok] == 180)


def _objs(ids, ra, dec):
    o = np.empty(len(ids), OBJ_DTYPE)
    o["id"], o["ra"], o["dec"] = ids, ra, dec
    return o


def test_wrap_pairs_and_branch3_fix():
    # across ra = 0: 0.0001 deg and 359.9995 deg on the equator are 2.16" apart
    A = _objs([1], [0.0001], [0.0])
    B = _objs([2], [359.9995], [0.0])
    for r, want in ((2.0, 0), (2.2, 1)):
        p, d, _ = oracle.xmatch(A, B, r * ARCSEC)
        assert len(p) == want
        p2, _, _ = oracle.xmatch(B, A, r * ARCSEC)   # the mirror branch
        assert len(p2) == want
    p, d, _ = oracle.xmatch(A, B, 3 * ARCSEC)
    assert d[0] == pytest.approx(np.radians(0.0006), rel=1e-9)


def test_pole_pairs():
    # two sources 1" from the north pole on opposite meridians are 2" apart
    A = _objs([1], [10.0], [90 - ARCSEC])
    B = _objs([2], [190.0], [90 - ARCSEC])
    p, d, _ = oracle.xmatch(A, B, 2.5 * ARCSEC)
    assert len(p) == 1
    assert d[0] == pytest.approx(np.radians(2 * ARCSEC), rel=1e-6)
    p, _, _ = oracle.xmatch(A, B, 1.9 * ARCSEC)
    assert len(p) == 0


def test_dec_plus_90_kept_and_invalid_dropped():
    A = _objs([1, 2, 3, 4], [0.0, 0.0, 0.0, np.nan], [90.0, 91.0, np.nan, 0.0])
    B = _objs([5], [123.0], [90.0])
    p, _, st = oracle.xmatch(A, B, ARCSEC)
    assert st.nA_kept == 1   # dec = 90 kept; dec 91, NaN dec and NaN ra dropped
    assert [tuple(x) for x in p] == [(1, 5)]


def test_segmentation_invariance(fixtures):
    a, _ = fixtures
    whole, _, _ = oracle.xmatch(a, a, 5 * ARCSEC)
    parts = []
    for s in range(0, len(a), 2020):      # Debug Switches.txt:2: -n2020
        for t in range(0, len(a), 2020):
            p, _, _ = oracle.xmatch(a[s:s + 2020], a[t:t + 2020], 5 * ARCSEC)
            parts.append(p)
    assert np.array_equal(sorted_pairs(whole), sorted_pairs(np.concatenate(parts)))


def test_swap_symmetry(fixtures):
    a, a2 = fixtures
    p, _, _ = oracle.xmatch(a2, a, 5 * ARCSEC)
    q, _, _ = oracle.xmatch(a, a2, 5 * ARCSEC)
    assert np.array_equal(sorted_pairs(p), sorted_pairs(q[:, ::-1].copy()))


def test_empty_inputs():
    E = np.empty(0, OBJ_DTYPE)
    A = _objs([1], [1.0], [1.0])
    for x, y in ((E, E), (E, A), (A, E)):
        p, _, _ = oracle.xmatch(x, y, ARCSEC)
        assert len(p) == 0
