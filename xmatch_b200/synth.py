"""Seeded synthetic catalogs with the shapes of the benchmark configurations.

No survey data is involved: the reference ships only a 10,000-source SDSS
slice (Data/test.idradec), so every workload here is generated from a stated
distribution and seed.
"""
import numpy as np

# .idradec record (Obj.h:21-25), 24 bytes; defined here too so that this file
# also loads on its own (by path), without the package and its library
OBJ_DTYPE = np.dtype([("id", "<i8"), ("ra", "<f8"), ("dec", "<f8")])

ARCSEC = 1.0 / 3600.0


def _unit(ra_deg, dec_deg):
    ra = np.radians(ra_deg)
    de = np.radians(dec_deg)
    cd = np.cos(de)
    return np.stack([cd * np.cos(ra), cd * np.sin(ra), np.sin(de)], axis=-1)


def _radec(v):
    v = v / np.linalg.norm(v, axis=-1, keepdims=True)
    ra = np.degrees(np.arctan2(v[..., 1], v[..., 0])) % 360.0
    ra = np.where(ra >= 360.0, 0.0, ra)
    dec = np.degrees(np.arcsin(np.clip(v[..., 2], -1.0, 1.0)))
    return ra, dec


def perturb(rng, ra_deg, dec_deg, sigma_deg):
    """Isotropic Gaussian offset of sigma (per axis) in the tangent plane."""
    ra = np.radians(ra_deg)
    de = np.radians(dec_deg)
    p = _unit(ra_deg, dec_deg)
    e_ra = np.stack([-np.sin(ra), np.cos(ra), np.zeros_like(ra)], axis=-1)
    e_de = np.stack([-np.sin(de) * np.cos(ra), -np.sin(de) * np.sin(ra), np.cos(de)], axis=-1)
    s = np.radians(sigma_deg)
    dx = rng.normal(0.0, s, len(ra))[:, None]
    dy = rng.normal(0.0, s, len(ra))[:, None]
    return _radec(p + dx * e_ra + dy * e_de)


def uniform_sphere(rng, n, dec_min=-90.0, dec_max=90.0):
    ra = rng.uniform(0.0, 360.0, n)
    s0, s1 = np.sin(np.radians(dec_min)), np.sin(np.radians(dec_max))
    dec = np.degrees(np.arcsin(rng.uniform(s0, s1, n)))
    return ra, dec


def make_objs(ids, ra, dec):
    o = np.empty(len(ids), OBJ_DTYPE)
    o["id"] = ids
    o["ra"] = ra
    o["dec"] = dec
    return o


def config0(n_a=200_000, n_b=200_000, seed=1000, band=10.0, frac_pert=0.6, sigma_arcsec=0.5):
    """Plain zone crossmatch, small: A uniform in dec [-band, band]; B = 60 % of A
    perturbed by sigma plus 40 % uniform in the band.  r = zh = 3 arcsec."""
    rng = np.random.default_rng(seed)
    ra, dec = uniform_sphere(rng, n_a, -band, band)
    A = make_objs(np.arange(n_a, dtype=np.int64), ra, dec)
    npert = int(round(frac_pert * n_b))
    src = rng.choice(n_a, npert, replace=False)
    pra, pdec = perturb(rng, ra[src], dec[src], sigma_arcsec * ARCSEC)
    rra, rdec = uniform_sphere(rng, n_b - npert, -band, band)
    B = make_objs(np.arange(n_b, dtype=np.int64) + 10_000_000_000,
                  np.concatenate([pra, rra]), np.concatenate([pdec, rdec]))
    return A, B


def mixture(rng, n, n_clusters=500, frac_cluster=0.2, sigma_cluster=0.1, centers=None):
    """80 % uniform on the sphere, 20 % in Gaussian clusters of sigma degrees."""
    nc = int(round(frac_cluster * n))
    nu = n - nc
    ra_u, dec_u = uniform_sphere(rng, nu)
    if centers is None:
        centers = uniform_sphere(rng, n_clusters)
    which = rng.integers(0, n_clusters, nc)
    ra_c, dec_c = perturb(rng, centers[0][which], centers[1][which], sigma_cluster)
    return np.concatenate([ra_u, ra_c]), np.concatenate([dec_u, dec_c]), centers


def add_edges(rng, ra, dec, n_wrap=10_000, n_pole=10_000):
    """Overwrite the first sources with ones at ra within 1 arcsec of 0/360 and
    at |dec| > 89 (a tenth of those within 1 arcsec of a pole)."""
    k = 0
    w = rng.uniform(0, ARCSEC, n_wrap)
    ra[k:k + n_wrap] = np.where(rng.random(n_wrap) < 0.5, w, 360.0 - w)
    ra[k:k + n_wrap] = np.where(ra[k:k + n_wrap] >= 360.0, 0.0, ra[k:k + n_wrap])
    k += n_wrap
    pole = rng.uniform(89.0, 90.0, n_pole)
    close = rng.random(n_pole) < 0.1
    pole = np.where(close, 90.0 - rng.uniform(0, ARCSEC, n_pole), pole)
    sign = np.where(rng.random(n_pole) < 0.5, 1.0, -1.0)
    dec[k:k + n_pole] = sign * pole
    ra[k:k + n_pole] = rng.uniform(0, 360.0, n_pole)
    return ra, dec


def config1(n=50_000_000, seed=1001, frac_pert=0.7, sigma_arcsec=0.3, edges=True):
    """Full-scale: A and B of n sources each, 80 % uniform + 20 % in 500 clusters
    (sigma 0.1 deg); B = 70 % perturbed copies of A (sigma 0.3") + 30 % random
    from the same mixture; wrap and polar sources forced in.  r = zh = 1"."""
    rng = np.random.default_rng(seed)
    ra, dec, centers = mixture(rng, n)
    if edges:
        m = min(n // 10, 10_000)
        ra, dec = add_edges(rng, ra, dec, m, m)
    A = make_objs(np.arange(n, dtype=np.int64), ra, dec)
    npert = int(round(frac_pert * n))
    src = rng.choice(n, npert, replace=False) if n < 5_000_000 else rng.integers(0, n, npert)
    pra, pdec = perturb(rng, ra[src], dec[src], sigma_arcsec * ARCSEC)
    rra, rdec, _ = mixture(rng, n - npert, centers=centers)
    B = make_objs(np.arange(n, dtype=np.int64) + 100_000_000_000,
                  np.concatenate([pra, rra]), np.concatenate([pdec, rdec]))
    perm = rng.permutation(n)
    return A, B[perm]


def planted(rng, n_pairs, r_deg, kmax=100, rel=1e-9):
    """Pairs at separation r (1 +- k rel), k uniform in 1..kmax, random position angle.
    Returns (A_ra, A_dec, B_ra, B_dec, sign, k) with sign +1 for r(1 + k rel) (outside).
    The offset k rel r is only meaningful where it is well above the FP64 spacing
    of the stored coordinates (about 1e-15 rad for degrees up to 360)."""
    ra, dec = uniform_sphere(rng, n_pairs)
    k = rng.integers(1, kmax + 1, n_pairs)
    sign = np.where(rng.random(n_pairs) < 0.5, 1.0, -1.0)
    sep = np.radians(r_deg) * (1.0 + sign * k * rel)
    pa = rng.uniform(0, 2 * np.pi, n_pairs)
    p = _unit(ra, dec)
    rar = np.radians(ra)
    der = np.radians(dec)
    e_ra = np.stack([-np.sin(rar), np.cos(rar), np.zeros_like(rar)], axis=-1)
    e_de = np.stack([-np.sin(der) * np.cos(rar), -np.sin(der) * np.sin(rar), np.cos(der)], axis=-1)
    t = np.cos(pa)[:, None] * e_ra + np.sin(pa)[:, None] * e_de
    q = np.cos(sep)[:, None] * p + np.sin(sep)[:, None] * t
    bra, bdec = _radec(q)
    return ra, dec, bra, bdec, sign, k


def config3(n=10_000_000, n_planted=1_000_000, r_arcsec=0.1, seed=1003):
    """Precision stress: n uniform per side plus n_planted pairs at r(1 +- k 1e-9).
    Returns (A, B, sign, k); planted pair i is (A id n + i, B id 1e11 + n + i)."""
    rng = np.random.default_rng(seed)
    ra, dec = uniform_sphere(rng, n)
    pra, pdec, qra, qdec, sign, k = planted(rng, n_planted, r_arcsec * ARCSEC)
    A = make_objs(np.arange(n + n_planted, dtype=np.int64), np.concatenate([ra, pra]),
                  np.concatenate([dec, pdec]))
    rb, db = uniform_sphere(rng, n)
    B = make_objs(np.arange(n + n_planted, dtype=np.int64) + 100_000_000_000,
                  np.concatenate([rb, qra]), np.concatenate([db, qdec]))
    return A, B, sign, k


def config2_jobs(n_jobs=4096, seed=1002, median=20_000, sigma=1.0, lo=1_000, hi=2_000_000, scale=1.0):
    """Uneven batch: per job, side sizes ~ LogNormal(median, sigma) clipped to
    [lo, hi] (scaled by `scale`), a random dec band 0.5-5 deg wide, r ~ U[0.5",
    5"], zh = r, sources generated as config 0 (60 % perturbed / 40 % random)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_jobs):
        na = int(np.clip(median * np.exp(rng.normal(0, sigma)), lo, hi) * scale)
        nb = int(np.clip(median * np.exp(rng.normal(0, sigma)), lo, hi) * scale)
        na, nb = max(na, 1), max(nb, 1)
        width = rng.uniform(0.5, 5.0)
        c = rng.uniform(-85.0, 85.0 - width)
        r = rng.uniform(0.5, 5.0)
        ra, dec = uniform_sphere(rng, na, c, c + width)
        A = make_objs(np.arange(na, dtype=np.int64) + j * 10_000_000, ra, dec)
        npert = int(round(0.6 * nb))
        src = rng.integers(0, na, npert)
        pra, pdec = perturb(rng, ra[src], dec[src], 0.5 * ARCSEC)
        rra, rdec = uniform_sphere(rng, nb - npert, c, c + width)
        B = make_objs(np.arange(nb, dtype=np.int64) + j * 10_000_000 + 5_000_000,
                      np.concatenate([pra, rra]), np.concatenate([pdec, rdec]))
        jobs.append((A, B, r))
    return jobs
