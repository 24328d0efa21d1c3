/*
 * xm_oracle.c -- CPU ORACLE for the zone crossmatch (TEST INFRASTRUCTURE ONLY).
 *
 * This file is the checker, never the product.  Only the test-suite, the
 * smoke check and the CPU-baseline leg of the benchmark load it.  It restates
 * the reference's algorithm (matthiaslee/Xmatch, BoostXmatch) in plain C so
 * that the GPU path can be compared with it pair-for-pair:
 *
 *   zone id           floor((dec+90)/zh)              BoostXmatch/Sorter.cu:20-24
 *   zone count        ceil(180/zh)                    BoostXmatch/Sorter.cu:156
 *   sort              by (zone, ra)                   BoostXmatch/Sorter.cu:27-43,153
 *   zone begin/end    lower/upper bound per zone      BoostXmatch/Sorter.cu:156-165
 *   degrees->radians  division by RAD2DEG             BoostXmatch/Sorter.cu:52-62, Common.h:9
 *   RA half-width     calc_alpha(theta, |dec|)        BoostXmatch/Common.cu:7-15
 *                     calc_alpha(theta, zh, zone)     BoostXmatch/Common.cu:17-23
 *   nz, sr_rad, chord threshold                       BoostXmatch/Worker.cu:310-317
 *   zone-pair loop    zid1, zid2 in zid1 +- nz        BoostXmatch/Worker.cu:330-366
 *   pair predicate    dec cut, 3 RA branches, chord   BoostXmatch/Worker.cu:82-123
 *   unit vector       radec2xyz                       BoostXmatch/Worker.cu:31-40
 *
 * Two reference defects are FIXED here, and the fixed form is the parity
 * contract of the project:
 *   1. Worker.cu:284,289 copy vRadec.size() BYTES instead of 16*size; the
 *      oracle simply uses all objects.
 *   2. Worker.cu:110-121 (branch ra_a ~ 0, ra_b ~ 2pi) subtracts |y2|, which
 *      flips the sign of y_b; the oracle uses the unit vector of the
 *      unshifted (ra, dec) for every branch, i.e. the true chord.
 * One documented divergence: dec = +90 exactly falls in zone n_zones when
 * 180/zh is integral (Sorter.cu:23,156) and the reference then never matches
 * it; here it is clamped into the last zone.  Objects whose zone is still
 * outside [0, n_zones) (|dec| > 90, NaN) are dropped, as in the reference;
 * so are objects with a non-finite ra, which can never pass the RA cut.
 *
 * The unit vectors come from the project's own FP64 sincos (Cody-Waite
 * reduction by pi/2 + truncated Taylor series; constants derived by
 * xmatch_b200/csrc/gen_sincos_consts.py), written out again here from the
 * same specification so that oracle and GPU produce identical bits.  This
 * file must be compiled with -ffp-contract=off.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_RAD2DEG 57.295779513082323                 /* Common.h:9 */
#define OR_M_PI2 6.2831853071795864769252867665590057683943387987502116419498 /* Worker.cu:23 */

/* ------------------------------------------------------------------ */
/* project sincos specification (see the header comment)              */
/* ------------------------------------------------------------------ */
#define OR_PIO2_1 0x1.921fb54442d18p+0
#define OR_PIO2_2 0x1.1a62633145c07p-54
#define OR_PIO2_3 -0x1.f1976b7ed8fbcp-110
#define OR_2_OVER_PI 0x1.45f306dc9c883p-1
static const double OR_S[8] = {
    -0x1.5555555555555p-3, 0x1.1111111111111p-7, -0x1.a01a01a01a01ap-13,
    0x1.71de3a556c734p-19, -0x1.ae64567f544e4p-26, 0x1.6124613a86d09p-33,
    -0x1.ae7f3e733b81fp-41, 0x1.952c77030ad4ap-49};
static const double OR_C[9] = {
    -0x1.0000000000000p-1, 0x1.5555555555555p-5, -0x1.6c16c16c16c17p-10,
    0x1.a01a01a01a01ap-16, -0x1.27e4fb7789f5cp-22, 0x1.1eed8eff8d898p-29,
    -0x1.93974a8c07c9dp-37, 0x1.ae7f3e733b81fp-45, -0x1.6827863b97d97p-53};

void or_sincos(double x, double *s, double *c)
{
    double kd = rint(x * OR_2_OVER_PI);
    double r = fma(-kd, OR_PIO2_1, x);
    r = fma(-kd, OR_PIO2_2, r);
    r = fma(-kd, OR_PIO2_3, r);
    double r2 = r * r;
    /* sin: r + r^3 * P(r^2), Horner from the highest coefficient */
    double ps = OR_S[7];
    for (int i = 6; i >= 0; --i) ps = fma(ps, r2, OR_S[i]);
    double r3 = r2 * r;
    double sn = fma(r3, ps, r);
    /* cos: 1 + r^2 * Q(r^2) */
    double pc = OR_C[8];
    for (int i = 7; i >= 0; --i) pc = fma(pc, r2, OR_C[i]);
    double cs = fma(r2, pc, 1.0);
    long long k = (long long)kd;
    switch ((int)(k & 3)) {
    case 0: *s = sn;  *c = cs;  break;
    case 1: *s = cs;  *c = -sn; break;
    case 2: *s = -sn; *c = -cs; break;
    default: *s = -cs; *c = sn; break;
    }
}

/* Worker.cu:31-40 */
static inline void or_radec2xyz(double ra, double dec, double *x, double *y, double *z)
{
    double sr, cr, sd, cd;
    or_sincos(ra, &sr, &cr);
    or_sincos(dec, &sd, &cd);
    *x = cd * cr;
    *y = cd * sr;
    *z = sd;
}

/* Common.cu:7-15 (parenthesisation kept: atan(sin t) / sqrt(...)) */
double or_calc_alpha(double theta, double abs_dec)
{
    if (abs_dec + theta > 89.99) return 180;
    return fabs(atan(sin(theta / OR_RAD2DEG))
                / sqrt(fabs(cos((abs_dec - theta) / OR_RAD2DEG)
                            * cos((abs_dec + theta) / OR_RAD2DEG))));
}

/* Common.cu:17-23 */
double or_calc_alpha_zone(double theta, double zh_deg, int zone)
{
    double dec = fabs(zone * zh_deg - 90);
    double dec2 = fabs((zone + 1) * zh_deg - 90);
    dec = (dec > dec2 ? dec : dec2);
    return or_calc_alpha(theta, dec + 0.01 * theta);
}

/* Sorter.cu:20-24, plus the +90 clamp; returns -1 for dropped objects */
static inline int64_t or_zone_id(double dec_deg, double zh_deg, int64_t n_zones)
{
    double zd = floor((dec_deg + 90) / zh_deg);
    if (!(zd >= 0.0)) return -1;
    if (zd >= (double)n_zones) {
        if (zd == (double)n_zones && dec_deg <= 90.0) return n_zones - 1;
        return -1;
    }
    return (int64_t)zd;
}

/* ------------------------------------------------------------------ */
/* zone build                                                          */
/* ------------------------------------------------------------------ */
typedef struct {
    int64_t id;
    double ra, dec;
} or_obj; /* Obj.h:21-25, 24 bytes */

typedef struct {
    int64_t n;          /* objects kept */
    int64_t n_zones;
    double zh_deg;
    int64_t *id;
    double *ra_deg;     /* kept for the sort key / windows */
    double *ra, *dec;   /* radians (Sorter.cu:52-62) */
    double *x, *y, *z;
    int64_t *zbeg, *zend;
} or_seg;

typedef struct {
    int64_t zone;
    double ra;
    int64_t idx;
} or_key;

static int or_key_cmp(const void *pa, const void *pb)
{
    const or_key *a = (const or_key *)pa, *b = (const or_key *)pb;
    if (a->zone != b->zone) return a->zone < b->zone ? -1 : 1;
    if (a->ra < b->ra) return -1;
    if (a->ra > b->ra) return 1;
    return a->idx < b->idx ? -1 : (a->idx > b->idx);
}

static void or_seg_free(or_seg *s)
{
    free(s->id); free(s->ra_deg); free(s->ra); free(s->dec);
    free(s->x); free(s->y); free(s->z); free(s->zbeg); free(s->zend);
    memset(s, 0, sizeof(*s));
}

static int or_seg_build(or_seg *s, const or_obj *o, int64_t n, double zh_deg)
{
    memset(s, 0, sizeof(*s));
    s->zh_deg = zh_deg;
    s->n_zones = (int64_t)ceil(180 / zh_deg);
    or_key *k = (or_key *)malloc(sizeof(or_key) * (size_t)(n > 0 ? n : 1));
    if (!k) return -1;
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t z = or_zone_id(o[i].dec, zh_deg, s->n_zones);
        if (z < 0 || !isfinite(o[i].ra)) continue;   /* non-finite ra never passes the RA cut */
        k[m].zone = z; k[m].ra = o[i].ra; k[m].idx = i; ++m;
    }
    qsort(k, (size_t)m, sizeof(or_key), or_key_cmp);
    size_t nb = (size_t)(m > 0 ? m : 1);
    s->n = m;
    s->id = (int64_t *)malloc(8 * nb);
    s->ra_deg = (double *)malloc(8 * nb);
    s->ra = (double *)malloc(8 * nb);
    s->dec = (double *)malloc(8 * nb);
    s->x = (double *)malloc(8 * nb);
    s->y = (double *)malloc(8 * nb);
    s->z = (double *)malloc(8 * nb);
    s->zbeg = (int64_t *)calloc((size_t)s->n_zones, 8);
    s->zend = (int64_t *)calloc((size_t)s->n_zones, 8);
    if (!s->id || !s->ra_deg || !s->ra || !s->dec || !s->x || !s->y || !s->z || !s->zbeg || !s->zend) {
        free(k); or_seg_free(s); return -1;
    }
    for (int64_t j = 0; j < m; ++j) {
        const or_obj *p = &o[k[j].idx];
        s->id[j] = p->id;
        s->ra_deg[j] = p->ra;
        s->ra[j] = p->ra / OR_RAD2DEG;
        s->dec[j] = p->dec / OR_RAD2DEG;
        or_radec2xyz(s->ra[j], s->dec[j], &s->x[j], &s->y[j], &s->z[j]);
    }
    /* zone [begin, end) = lower/upper bound of each zone id */
    int64_t j = 0;
    for (int64_t z = 0; z < s->n_zones; ++z) {
        s->zbeg[z] = j;
        while (j < m && k[j].zone == z) ++j;
        s->zend[z] = j;
    }
    free(k);
    return 0;
}

/* ------------------------------------------------------------------ */
/* match                                                               */
/* ------------------------------------------------------------------ */
enum {
    OR_MODE_ALLPAIRS = 0,        /* reference loop, unit vectors precomputed */
    OR_MODE_ALLPAIRS_SINCOS = 1, /* reference loop and cost: xyz per pair     */
    OR_MODE_WINDOWED = 2         /* same predicate, RA window by bisection    */
};

typedef struct {
    uint64_t n_tested;  /* pairs the loop evaluated                    */
    uint64_t n_cand;    /* pairs passing the dec and RA cuts (C_alg)   */
    uint64_t n_match;   /* pairs passing the full predicate            */
    uint64_t nA_kept, nB_kept;
    int64_t n_zones;
    int32_t nz;
    double sr_rad, sr_dist2;
} or_stats;

typedef struct {
    int64_t *pairs;   /* 2 per match */
    double *dist;
    uint64_t n, cap;
    uint64_t tested, cand;
} or_buf;

static int or_buf_push(or_buf *b, int64_t ia, int64_t ib, double d)
{
    if (b->n == b->cap) {
        uint64_t nc = b->cap ? b->cap * 2 : 256;
        int64_t *np = (int64_t *)realloc(b->pairs, nc * 16);
        if (!np) return -1;
        b->pairs = np;
        double *nd = (double *)realloc(b->dist, nc * 8);
        if (!nd) return -1;
        b->dist = nd;
        b->cap = nc;
    }
    b->pairs[2 * b->n] = ia;
    b->pairs[2 * b->n + 1] = ib;
    b->dist[b->n] = d;
    b->n++;
    return 0;
}

typedef struct {
    const or_seg *A, *B;
    double sr_deg, sr_rad, sr_dist2;
    int nz;
    int mode;
    double *alpha;       /* per zone of A */
    int64_t n_chunks, zones_per_chunk;
    or_buf *bufs;        /* one per chunk, concatenated in order */
    volatile int64_t next;
    int err;
} or_job;

/* Worker.cu:82-123 with the branch-3 sign fix: returns 1 on a match and
 * stores the chord^2; *cand is set when the dec and RA cuts pass. */
static inline int or_test(const or_seg *A, int64_t i1, const or_seg *B, int64_t i2,
                          double sr_rad, double alpha, double sr_dist2, int per_pair_sincos,
                          int *cand, double *c2)
{
    *cand = 0;
    double ra1 = A->ra[i1], de1 = A->dec[i1];
    double ra2 = B->ra[i2], de2 = B->dec[i2];
    if (!(fabs(de1 - de2) < sr_rad)) return 0;
    double d = ra1 - ra2;
    if (!(fabs(d) < alpha || fabs(d - OR_M_PI2) < alpha || fabs(d + OR_M_PI2) < alpha)) return 0;
    *cand = 1;
    double x1, y1, z1, x2, y2, z2;
    if (per_pair_sincos) {
        or_radec2xyz(ra1, de1, &x1, &y1, &z1);
        or_radec2xyz(ra2, de2, &x2, &y2, &z2);
    } else {
        x1 = A->x[i1]; y1 = A->y[i1]; z1 = A->z[i1];
        x2 = B->x[i2]; y2 = B->y[i2]; z2 = B->z[i2];
    }
    double dx = x1 - x2, dy = y1 - y2, dz = z1 - z2;
    double c = dx * dx + dy * dy + dz * dz;
    *c2 = c;
    return c < sr_dist2;
}

/* first index in [lo,hi) with ra[i] >= v */
static int64_t or_lower(const double *ra, int64_t lo, int64_t hi, double v)
{
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (ra[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}
/* first index in [lo,hi) with ra[i] > v */
static int64_t or_upper(const double *ra, int64_t lo, int64_t hi, double v)
{
    while (lo < hi) {
        int64_t mid = lo + (hi - lo) / 2;
        if (ra[mid] <= v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

static int or_run_pair_range(or_job *J, or_buf *b, int64_t i1, int64_t b0, int64_t b1, double alpha)
{
    const or_seg *A = J->A, *B = J->B;
    for (int64_t i2 = b0; i2 < b1; ++i2) {
        int cand;
        double c2 = 0;
        b->tested++;
        int m = or_test(A, i1, B, i2, J->sr_rad, alpha, J->sr_dist2,
                        J->mode == OR_MODE_ALLPAIRS_SINCOS, &cand, &c2);
        b->cand += (uint64_t)cand;
        if (m && or_buf_push(b, A->id[i1], B->id[i2], 2.0 * asin(sqrt(c2) / 2.0))) return -1;
    }
    return 0;
}

static void or_run_chunk(or_job *J, int64_t c)
{
    const or_seg *A = J->A, *B = J->B;
    or_buf *b = &J->bufs[c];
    int64_t z0 = c * J->zones_per_chunk;
    int64_t z1 = z0 + J->zones_per_chunk;
    if (z1 > A->n_zones) z1 = A->n_zones;
    /* Worker.cu:330-366 */
    for (int64_t zid1 = z0; zid1 < z1; ++zid1) {
        int64_t i1s = A->zbeg[zid1], i1e = A->zend[zid1];
        if (i1e - i1s < 1) continue;
        int64_t zs = zid1 - J->nz > 0 ? zid1 - J->nz : 0;
        int64_t ze = zid1 + J->nz < A->n_zones - 1 ? zid1 + J->nz : A->n_zones - 1;
        double alpha = J->alpha[zid1];
        for (int64_t zid2 = zs; zid2 <= ze; ++zid2) {
            int64_t i2s = B->zbeg[zid2], i2e = B->zend[zid2];
            if (i2e - i2s < 1) continue;
            for (int64_t i1 = i1s; i1 < i1e; ++i1) {
                if (J->mode != OR_MODE_WINDOWED || alpha >= 3.0) {
                    if (or_run_pair_range(J, b, i1, i2s, i2e, alpha)) { J->err = 1; return; }
                    continue;
                }
                /* conservative windows on ra (radians); the predicate decides */
                const double eps = 1e-12;
                double ra1 = A->ra[i1];
                double lo = ra1 - alpha - eps, hi = ra1 + alpha + eps;
                int64_t a0 = or_lower(B->ra, i2s, i2e, lo), a1 = or_upper(B->ra, i2s, i2e, hi);
                if (or_run_pair_range(J, b, i1, a0, a1, alpha)) { J->err = 1; return; }
                /* branch 2: ra1 ~ 2pi, ra2 ~ 0 */
                double lo2 = lo - OR_M_PI2 - eps, hi2 = hi - OR_M_PI2 + eps;
                if (hi2 >= B->ra[i2s]) {
                    int64_t w0 = or_lower(B->ra, i2s, i2e, lo2), w1 = or_upper(B->ra, i2s, i2e, hi2);
                    if (w0 < a0) { if (w1 > a0) w1 = a0; if (or_run_pair_range(J, b, i1, w0, w1, alpha)) { J->err = 1; return; } }
                }
                /* branch 3: ra1 ~ 0, ra2 ~ 2pi */
                double lo3 = lo + OR_M_PI2 - eps, hi3 = hi + OR_M_PI2 + eps;
                if (lo3 <= B->ra[i2e - 1]) {
                    int64_t w0 = or_lower(B->ra, i2s, i2e, lo3), w1 = or_upper(B->ra, i2s, i2e, hi3);
                    if (w0 < a1) w0 = a1;
                    if (w0 < w1 && or_run_pair_range(J, b, i1, w0, w1, alpha)) { J->err = 1; return; }
                }
            }
        }
    }
}

static void *or_worker(void *p)
{
    or_job *J = (or_job *)p;
    for (;;) {
        int64_t c = __atomic_fetch_add(&J->next, 1, __ATOMIC_RELAXED);
        if (c >= J->n_chunks || J->err) break;
        or_run_chunk(J, c);
    }
    return NULL;
}

/*
 * Full crossmatch of two catalogs (all objects of each as one segment).
 * Writes up to `cap` matches as (idA, idB) pairs plus the distance in
 * radians (2 asin(chord/2)), and returns the TOTAL number of matches, or a
 * negative value on error.  The output order is deterministic: zone order
 * of A, then zone of B, then A order, then B order.
 */
int64_t or_xmatch(const or_obj *A, int64_t nA, const or_obj *B, int64_t nB,
                  double sr_deg, double zh_deg, int mode, int nthreads,
                  int64_t *pairs_out, double *dist_out, uint64_t cap, or_stats *st)
{
    if (!(zh_deg > 0) || !(sr_deg > 0) || nA < 0 || nB < 0) return -2;
    or_seg sa, sb;
    if (or_seg_build(&sa, A, nA, zh_deg)) return -1;
    if (or_seg_build(&sb, B, nB, zh_deg)) { or_seg_free(&sa); return -1; }
    or_job J;
    memset(&J, 0, sizeof(J));
    J.A = &sa; J.B = &sb; J.mode = mode;
    J.sr_deg = sr_deg;
    J.nz = (int)ceil(sr_deg / zh_deg);                  /* Worker.cu:313 */
    J.sr_rad = sr_deg / OR_RAD2DEG;                     /* Worker.cu:315 */
    J.sr_dist2 = 2.0 * sin(J.sr_rad / 2.0);             /* Worker.cu:316-317 */
    J.sr_dist2 *= J.sr_dist2;
    J.alpha = (double *)malloc(sizeof(double) * (size_t)sa.n_zones);
    for (int64_t z = 0; z < sa.n_zones; ++z) J.alpha[z] = or_calc_alpha_zone(sr_deg, zh_deg, (int)z);
    if (nthreads < 1) nthreads = 1;
    J.zones_per_chunk = 64;
    J.n_chunks = (sa.n_zones + J.zones_per_chunk - 1) / J.zones_per_chunk;
    J.bufs = (or_buf *)calloc((size_t)J.n_chunks, sizeof(or_buf));
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    int started = 0;
    for (int t = 1; t < nthreads; ++t)
        if (pthread_create(&th[t], NULL, or_worker, &J) == 0) started++; else break;
    or_worker(&J);
    for (int t = 1; t <= started; ++t) pthread_join(th[t], NULL);
    free(th);
    int64_t total = 0;
    uint64_t tested = 0, cand = 0;
    for (int64_t c = 0; c < J.n_chunks; ++c) {
        or_buf *b = &J.bufs[c];
        for (uint64_t i = 0; i < b->n; ++i) {
            uint64_t o = (uint64_t)total + i;
            if (o < cap) {
                if (pairs_out) { pairs_out[2 * o] = b->pairs[2 * i]; pairs_out[2 * o + 1] = b->pairs[2 * i + 1]; }
                if (dist_out) dist_out[o] = b->dist[i];
            }
        }
        total += (int64_t)b->n;
        tested += b->tested; cand += b->cand;
        free(b->pairs); free(b->dist);
    }
    if (st) {
        st->n_tested = tested; st->n_cand = cand; st->n_match = (uint64_t)total;
        st->nA_kept = (uint64_t)sa.n; st->nB_kept = (uint64_t)sb.n;
        st->n_zones = sa.n_zones; st->nz = J.nz; st->sr_rad = J.sr_rad; st->sr_dist2 = J.sr_dist2;
    }
    int err = J.err;
    free(J.bufs); free(J.alpha);
    or_seg_free(&sa); or_seg_free(&sb);
    return err ? -1 : total;
}

/* ---- small helpers used by the tests ---- */
void or_sincos_batch(const double *x, int64_t n, double *s, double *c)
{
    for (int64_t i = 0; i < n; ++i) or_sincos(x[i], &s[i], &c[i]);
}

/* unit vectors of (ra, dec) in degrees, as the zone builder computes them */
void or_unit_vectors(const double *ra_deg, const double *dec_deg, int64_t n, double *xyz)
{
    for (int64_t i = 0; i < n; ++i)
        or_radec2xyz(ra_deg[i] / OR_RAD2DEG, dec_deg[i] / OR_RAD2DEG, &xyz[3 * i], &xyz[3 * i + 1], &xyz[3 * i + 2]);
}

void or_alpha_table(double sr_deg, double zh_deg, int64_t n_zones, double *out)
{
    for (int64_t z = 0; z < n_zones; ++z) out[z] = or_calc_alpha_zone(sr_deg, zh_deg, (int)z);
}

/* ------------------------------------------------------------------ */
/* segment order of the GPU zone builder (for export comparisons)      */
/* ------------------------------------------------------------------ */
/* quantised ra: floor(ra_rad * 2^31/pi), clamped to [0, 2^32-1] */
static inline uint32_t or_raq32(double ra_rad)
{
    double x = floor(ra_rad * 0x1.45f306dc9c883p+29);
    if (!(x > 0.0)) return 0u;
    if (x >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

/* raq bits kept in the sort key and in the segment (2^27 steps per turn) */
int or_raq_bits(int64_t n_zones)
{
    (void)n_zones;
    return 27;
}

typedef struct {
    uint64_t key;   /* zone << raq_bits | raq */
    int64_t idx;
} or_qkey;

static int or_qkey_cmp(const void *pa, const void *pb)
{
    const or_qkey *a = (const or_qkey *)pa, *b = (const or_qkey *)pb;
    if (a->key != b->key) return a->key < b->key ? -1 : 1;
    return a->idx < b->idx ? -1 : (a->idx > b->idx);
}

/* Sorted segment as the GPU builder lays it out: ordered by (zone, leading
 * raq bits, input index); id, ra/dec radians, zone begin/end
 * (Segment.h:36-38).  Returns the number of objects kept. */
int64_t or_build_export(const or_obj *o, int64_t n, double zh_deg, int64_t *id, double *radec,
                        int64_t *zbeg, int64_t *zend, int64_t zcap)
{
    int64_t n_zones = (int64_t)ceil(180 / zh_deg);
    int rb = or_raq_bits(n_zones);
    or_qkey *k = (or_qkey *)malloc(sizeof(or_qkey) * (size_t)(n > 0 ? n : 1));
    if (!k) return -1;
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t z = or_zone_id(o[i].dec, zh_deg, n_zones);
        if (z < 0 || !isfinite(o[i].ra)) continue;
        double ra = o[i].ra / OR_RAD2DEG;
        k[m].key = ((uint64_t)z << rb) | (uint64_t)(or_raq32(ra) >> (32 - rb));
        k[m].idx = i;
        ++m;
    }
    qsort(k, (size_t)m, sizeof(or_qkey), or_qkey_cmp);
    for (int64_t j = 0; j < m; ++j) {
        const or_obj *p = &o[k[j].idx];
        if (id) id[j] = p->id;
        if (radec) { radec[2 * j] = p->ra / OR_RAD2DEG; radec[2 * j + 1] = p->dec / OR_RAD2DEG; }
    }
    int64_t j = 0;
    for (int64_t z = 0; z < n_zones && z < zcap; ++z) {
        if (zbeg) zbeg[z] = j;
        while (j < m && (int64_t)(k[j].key >> rb) == z) ++j;
        if (zend) zend[z] = j;
    }
    free(k);
    return m;
}
