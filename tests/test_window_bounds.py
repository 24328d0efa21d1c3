"""CPU test that the pair kernel's RA windows in quantised-ra units hold every
pair the reference's RA cut admits.

The kernel (xm_match.cu, make_win_q) takes an A object's windows from its own
27-bit quantised ra, raq = floor(RN(ra * S)) >> 5 with S the 2^31/pi scale of
the zone build (xm_math.cuh, raq32), and its zone's alpha: half-width
aq = ceil(RN(alpha * S / 32)) + 3 units, clipped to the turn, plus the two
wrapped windows when the direct one crosses ra = 0 or 2 pi.  The RA cut it
must cover is Worker.cu:89,98,110's: |dra| < alpha in one of the branches
dra = ra_a - ra_b, dra - 2 pi, dra + 2 pi.  Here both sides are restated
with numpy's float64 (round-to-nearest products, as __dmul_rn) and every
sampled pair that passes the cut is checked to lie inside the windows."""
import numpy as np

S = float.fromhex("0x1.45f306dc9c883p+29")   # raq32 scale: 2^31 / pi as the zone build rounds it
TURN = 1 << 27
TWO_PI = 2.0 * np.pi


def raq27(ra):
    x = np.floor(ra * S)
    x = np.where(x > 0.0, x, 0.0)
    x = np.minimum(x, 4294967295.0)
    return x.astype(np.uint64) >> np.uint64(5)


def windows(ra_q, alpha):
    """(lo, hi, lo2, hi2, lo3, hi3) as make_win_q computes them (empty: lo > hi)."""
    aqd = np.ceil(alpha * (S / 32.0)) + 3.0
    aq = np.where(aqd < TURN, aqd, TURN).astype(np.int64)
    q = ra_q.astype(np.int64)
    lo = np.maximum(q - aq, 0)
    hi = np.minimum(q + aq, TURN - 1)
    wrap2 = q + aq >= TURN
    lo2 = np.where(wrap2, 0, 1)
    hi2 = np.where(wrap2, q + aq - TURN, 0)
    wrap3 = q < aq
    lo3 = np.where(wrap3, q + TURN - aq, 1)
    hi3 = np.where(wrap3, TURN - 1, 0)
    return lo, hi, lo2, hi2, lo3, hi3


def ra_cut(ra_a, ra_b, alpha):
    d = ra_a - ra_b
    return (np.abs(d) < alpha) | (np.abs(d - TWO_PI) < alpha) | (np.abs(d + TWO_PI) < alpha)


def check(ra_a, ra_b, alpha):
    keep = ra_cut(ra_a, ra_b, alpha) & (ra_b >= 0.0) & (ra_b < TWO_PI)
    ra_a, ra_b, alpha = ra_a[keep], ra_b[keep], alpha[keep]
    assert len(ra_a) > 0
    qb = raq27(ra_b).astype(np.int64)
    lo, hi, lo2, hi2, lo3, hi3 = windows(raq27(ra_a), alpha)
    inside = ((qb >= lo) & (qb <= hi)) | ((qb >= lo2) & (qb <= hi2)) | ((qb >= lo3) & (qb <= hi3))
    bad = np.flatnonzero(~inside)
    assert len(bad) == 0, (ra_a[bad[:5]], ra_b[bad[:5]], alpha[bad[:5]])
    return len(ra_a)


def test_windows_hold_the_ra_cut():
    rng = np.random.default_rng(2024)
    n = 400_000
    tested = 0
    # radii from 0.01" to 10 deg, and alpha up to just below the full-ring limit of 3 rad
    for alpha_scale in (5e-8, 4.8e-6, 1e-4, 3e-2, 0.17, 1.0, 2.99):
        alpha = alpha_scale * rng.uniform(0.5, 1.0, n)
        ra_a = rng.uniform(0.0, TWO_PI, n)
        # A near the ends of the turn
        ra_a[: n // 8] = rng.uniform(0.0, 2 * alpha[: n // 8])
        ra_a[n // 8: n // 4] = TWO_PI - rng.uniform(1e-300, 2 * alpha[n // 8: n // 4])
        ra_a = np.clip(ra_a, 0.0, np.nextafter(TWO_PI, 0.0))
        # B within alpha, uniform and at the very edge of the cut
        frac = rng.uniform(-1.0, 1.0, n)
        frac[::3] = np.sign(frac[::3]) * (1.0 - rng.uniform(0.0, 1e-12, len(frac[::3])))
        ra_b = ra_a + frac * alpha
        ra_b = np.where(ra_b < 0.0, ra_b + TWO_PI, ra_b)
        ra_b = np.where(ra_b >= TWO_PI, ra_b - TWO_PI, ra_b)
        tested += check(ra_a, ra_b, alpha)
    assert tested > 2_000_000


def test_windows_at_exact_turn_ends():
    # ra = 0 and the largest ra below 2 pi, against B just inside the cut on either side
    alpha = np.full(8, 4.8481368110953598e-06)
    top = np.nextafter(TWO_PI, 0.0)
    ra_a = np.array([0.0, 0.0, top, top, 0.0, top, 1e-12, top - 1e-12])
    d = alpha * (1 - 1e-9)
    ra_b = np.array([d[0], TWO_PI - d[1], top - d[2], d[3] - 1e-300, 0.0, 0.0, TWO_PI - d[6], 1e-13])
    ra_b = np.where(ra_b >= TWO_PI, ra_b - TWO_PI, ra_b)
    check(ra_a, ra_b, alpha)
