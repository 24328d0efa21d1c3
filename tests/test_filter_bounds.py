"""The FP32 chord^2 thresholds of XM_FILTER32 (xm_filter_bounds), checked on
the CPU against pairs sampled around the search radius.

The pair kernel rejects a pair when its FP32 chord^2 exceeds thr_hi and, in a
zone with an RA cut (alpha < 3 rad), accepts it without the FP64 predicate
when the value is below thr_lo.  So, for any FP64 positions:
  c32 > thr_hi  =>  FP64 chord^2 >= T                      (no match lost)
  c32 < thr_lo  =>  FP64 chord^2 < T, |dec_a - dec_b| < r, and the RA cut of
                    Worker.cu:89,98,110 passes with alpha(zone(a))
                                                             (no match invented)
The FP32 value is emulated as the kernel forms it: FP32 differences of the
rounded unit vectors, fmaf(dz, dz, fmaf(dy, dy, dx * dx))."""
import numpy as np
import pytest

import xmatch_b200 as xm

RAD2DEG = 57.295779513082323
TWO_PI = 6.283185307179586
ARCSEC = 1.0 / 3600.0


def _unit(ra, dec):
    cd = np.cos(dec)
    return np.stack([cd * np.cos(ra), cd * np.sin(ra), np.sin(dec)], axis=-1)


def _c32(xa, xb):
    d = xa.astype(np.float32) - xb.astype(np.float32)
    dx, dy, dz = d[:, 0], d[:, 1], d[:, 2]
    t = dx * dx                                                          # FP32 product
    t = (dy.astype(np.longdouble) ** 2 + t.astype(np.longdouble)).astype(np.float32)   # fmaf
    return (dz.astype(np.longdouble) ** 2 + t.astype(np.longdouble)).astype(np.float32)


def _pairs(rng, r_deg, n):
    """A anywhere (a third near the poles), B at r (1 + u) in a random direction."""
    dec_a = np.degrees(np.arcsin(rng.uniform(-1, 1, n)))
    polar = rng.random(n) < 0.3
    dec_a[polar] = np.sign(rng.uniform(-1, 1, polar.sum())) * rng.uniform(min(80.0, 90 - 3 * r_deg), 90 - 2 * r_deg,
                                                                       polar.sum())
    ra_a = rng.uniform(0, 360, n)
    ra_a[: n // 10] = rng.uniform(0, 3 * r_deg, n // 10)            # near ra = 0 / 360
    k = rng.random(n)
    u = np.where(k < 0.3, rng.uniform(-0.5, 0.5, n), np.where(k < 0.7, rng.uniform(-0.03, 0.03, n),
                                                               rng.uniform(-1e-6, 1e-6, n)))
    th = np.radians(r_deg) * (1 + u)
    phi = rng.uniform(0, TWO_PI, n)
    a_dec, a_ra = np.radians(dec_a), np.radians(ra_a)
    sb = np.sin(a_dec) * np.cos(th) + np.cos(a_dec) * np.sin(th) * np.cos(phi)
    b_dec = np.arcsin(np.clip(sb, -1, 1))
    b_ra = a_ra + np.arctan2(np.sin(phi) * np.sin(th) * np.cos(a_dec), np.cos(th) - np.sin(a_dec) * sb)
    ra_b = np.mod(np.degrees(b_ra), 360.0)
    return ra_a, dec_a, ra_b, np.degrees(b_dec)


@pytest.mark.parametrize("r_arcsec, zh_ratio", [(0.1, 1.0), (1.0, 1.0), (1.0, 0.5), (60.0, 1.0), (3600.0, 1.0),
                                                (36000.0, 2.0)])
def test_fp32_thresholds_are_sound(r_arcsec, zh_ratio):
    rng = np.random.default_rng(int(r_arcsec * 10) + int(zh_ratio * 7))
    r_deg = r_arcsec * ARCSEC
    zh = r_deg * zh_ratio
    thr_hi, thr_lo = xm.filter_bounds(r_deg)
    assert 0 <= thr_lo < thr_hi
    sr_rad = r_deg / RAD2DEG
    T = (2.0 * np.sin(sr_rad / 2.0)) ** 2
    alpha = xm.alpha_table(r_deg, zh)

    ra_a, dec_a, ra_b, dec_b = _pairs(rng, r_deg, 400_000)
    ra1, dec1, ra2, dec2 = ra_a / RAD2DEG, dec_a / RAD2DEG, ra_b / RAD2DEG, dec_b / RAD2DEG   # as the build
    xa, xb = _unit(ra1, dec1), _unit(ra2, dec2)
    c64 = np.sum((xa - xb) ** 2, axis=1)
    c32 = _c32(xa, xb)

    hi = c32 > thr_hi
    assert np.all(c64[hi] >= T)

    zone = np.clip(np.floor((dec_a + 90.0) / zh).astype(np.int64), 0, len(alpha) - 1)
    al = alpha[zone]
    lo = (c32 < thr_lo) & (al < 3.0)
    assert np.all(c64[lo] < T)
    assert np.all(np.abs(dec1[lo] - dec2[lo]) < sr_rad)
    d = ra1[lo] - ra2[lo]
    a = al[lo]
    assert np.all((np.abs(d) < a) | (np.abs(d - TWO_PI) < a) | (np.abs(d + TWO_PI) < a))

    # the sample straddles the radius: both sides and the band in between are exercised
    inside = c64 < T
    assert hi.sum() > 1000 and inside.sum() > 1000
    if r_arcsec >= 1.0:
        assert lo.sum() > 1000


def test_small_radius_sends_every_pair_to_fp64():
    thr_hi, thr_lo = xm.filter_bounds(1e-9)   # r eta below the FP64 rounding of the cuts
    assert thr_lo == 0 and thr_hi > 0
