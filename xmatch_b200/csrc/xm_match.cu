// xm_match.cu -- zone-pair window search + pair test + compaction, as one
// persistent work-stealing launch.
//
// Replaces the reference's per-zone-pair launches (Worker.cu:330-366) of the
// all-pairs kernel xmatch_kernel (Worker.cu:65-241).
//
// Work decomposition.  A work item is `zc` consecutive zones of one job's A
// segment.  A pre-pass (one thread per item) cuts items into tiles of at
// most TILE objects -- a zone holding more than TILE/2 objects is split into
// near-equal single-zone tiles, consecutive smaller zones are packed into
// one tile -- and writes a staging plan per tile:
//   WHOLE   the B zones within nz of the tile's zones (Worker.cu:338-341) are
//           one contiguous range of the zone-sorted B segment; copied whole;
//   UNION   (a single-zone tile whose band is too large) per B zone only the
//           union of the tile's RA windows, [ra_first - alpha, ra_last +
//           alpha], when no RA-wraparound window can be non-empty;
//   pieces  a band too large for one stage, cut along B into consecutive
//           ranges that are each staged as a WHOLE plan (see tile_pieces);
//   GLOBAL  none of these fits: the windows are bisected in global memory.
//
// Pair kernel.  Warp-specialised and persistent: warp 0 claims tiles from a
// global counter (`chunk` at a time) and streams each tile's A objects and
// staged B ranges into a ring of shared-memory stages with bulk asynchronous
// copies (cp.async.bulk, completion counted on an mbarrier; no multicast);
// warps 1..TILE/32 consume a stage, one A object per thread, and release it
// on an "empty" mbarrier.  Every wait is bounded; a timeout sets an error
// flag that the host reports.
//
// Pair test.  Every thread bisects its own windows (direct, and the two
// wrapped ones for the RA branches of Worker.cu:89,98,110) in the staged
// quantised ra (raq, xyz.w) of its three B zones; the warp then walks the
// flattened list of its lanes' candidates.  The reference predicate
// (Worker.cu:88-97) is: dec cut, RA cut, chord^2 < (2 sin(r/2))^2, all FP64
// with the unit vectors of the unshifted (ra, dec) -- the branch-3 sign error
// of Worker.cu:118 fixed.  XM_FILTER32 evaluates chord^2 in FP32 from the
// FP32 unit vectors first: above thr_hi the pair cannot match; below thr_lo
// (zones with an RA cut) it matches and the cuts provably hold; in between,
// and in full-ring zones, B's ra/dec is read, both FP64 unit vectors are
// computed from the ra/dec of the pair (the builder's sincos, so the same bits
// every time) and the FP64 predicate decides.  The bounds are derived in xm_make_params, so
// the pair set is the FP64 one bit for bit.  XM_PLAIN64 applies the FP64
// predicate with per-pair sincos to every candidate.
//
// Output.  Matches are compacted per warp with __ballot_sync/__popc into the
// warp's buffer in shared memory (idA, and the job and index of the B object),
// which goes to global memory 32 entries at a time: one atomicAdd reserves the
// slots, the idB loads are issued under it, and the 32 records are stored
// coalesced (Worker.cu:128-240 uses two Hillis-Steele scans per block).  A full output
// buffer is detected and reported, never silently truncated (Worker.cu:147-148).
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

#include "xm_internal.h"

#include "xm_async.cuh"
#include "xm_match.cuh"
#include "xm_math.cuh"

namespace xm {

namespace {

constexpr double kWinEps = 1e-12;  // window widening (radians), >> FP64 rounding of ra +- alpha

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- bisection on the quantised ra (xyz.w) ----
__device__ __forceinline__ uint32_t raq_at(const float4 *xyz, uint32_t k) { return __float_as_uint(xyz[k].w); }
__device__ __forceinline__ uint32_t raq_at_g(const float4 *xyz, uint32_t k) { return __float_as_uint(__ldg(&xyz[k].w)); }

// first k in [lo, hi) with raq[k] >= t   (global memory)
__device__ __forceinline__ uint32_t lower_raq_g(const float4 *__restrict__ xyz, uint32_t lo, uint32_t hi, uint32_t t)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (raq_at_g(xyz, mid) < t) lo = mid + 1; else hi = mid;
    }
    return lo;
}
// first k in [lo, hi) with raq[k] > t    (global memory)
__device__ __forceinline__ uint32_t upper_raq_g(const float4 *__restrict__ xyz, uint32_t lo, uint32_t hi, uint32_t t)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (raq_at_g(xyz, mid) <= t) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Window bounds of one A object in quantised-ra space: any B with ra in the
// FP64 window has raq in [t_lo, t_hi] (raq is monotone in ra).
struct Win {
    uint32_t lo, hi;     // direct window
    uint32_t lo2, hi2;   // branch 2 (B near 0)
    uint32_t lo3, hi3;   // branch 3 (B near 2 pi)
};

// The wraparound windows are empty (lo > hi) unless the direct window crosses
// ra = 2 pi (branch 2: B with ra < hi - 2 pi) or ra = 0 (branch 3: B with
// ra > lo + 2 pi); ra of a kept object lies in [0, 2 pi).
__device__ __forceinline__ Win make_win(double ra, double alpha, int shift)
{
    const double lo = ra - alpha - kWinEps, hi = ra + alpha + kWinEps;
    Win w;
    w.lo = xm::raq32(lo) >> shift;
    w.hi = xm::raq32(hi) >> shift;
    w.lo2 = w.lo3 = 0xFFFFFFFFu;
    w.hi2 = w.hi3 = 0u;
    if (hi - XM_TWO_PI + kWinEps > 0.0) {
        w.lo2 = xm::raq32(lo - XM_TWO_PI - kWinEps) >> shift;
        w.hi2 = xm::raq32(hi - XM_TWO_PI + kWinEps) >> shift;
    }
    if (lo - kWinEps < 0.0) {
        w.lo3 = xm::raq32(lo + XM_TWO_PI - kWinEps) >> shift;
        w.hi3 = xm::raq32(hi + XM_TWO_PI + kWinEps) >> shift;
    }
    return w;
}

// The same windows in quantised-ra units from A's own quantised ra (xyz.w) and
// alpha: any B within alpha of A in ra (in one of the three branches) has a
// quantised ra within alpha * 2^26 / pi + 3 of A's -- 1 for the floor of each,
// 1 for the rounding of each product in raq32 -- so these windows hold every
// object of the FP64 ones, and the predicate decides.  Used with alpha < 3
// (pi - 3 apart, the three windows are disjoint); full-ring zones enumerate
// the whole zone instead.
constexpr double kRaqPerRad = XM_RAQ_SCALE / 32.0;   // 2^26 / pi: units of the 27-bit quantised ra per radian

__device__ __forceinline__ Win make_win_q(uint32_t ra_q, double alpha)
{
    constexpr uint32_t kTurn = 1u << 27;
    const double aqd = ceil(__dmul_rn(alpha, kRaqPerRad)) + 3.0;
    // alpha < 0 marks a tile whose zone offsets disagree (already reported as an error)
    const uint32_t aq = !(aqd >= 0.0) ? 0u : aqd < (double)kTurn ? (uint32_t)aqd : kTurn;
    Win w;
    w.lo = ra_q > aq ? ra_q - aq : 0u;
    w.hi = min(ra_q + aq, kTurn - 1u);   // ra_q, aq <= 2^27: no overflow
    w.lo2 = w.lo3 = 0xFFFFFFFFu;
    w.hi2 = w.hi3 = 0u;
    if (ra_q + aq >= kTurn) {            // branch 2: B near 0
        w.lo2 = 0u;
        w.hi2 = ra_q + aq - kTurn;
    }
    if (ra_q < aq) {                     // branch 3: B near 2 pi
        w.lo3 = ra_q + kTurn - aq;
        w.hi3 = kTurn - 1u;
    }
    return w;
}

// FP64 chord^2 of two positions from their unit vectors, computed as the zone
// builder computes them (the same bits).
__device__ __forceinline__ double chord2_radec_inl(double ra1, double dec1, double ra2, double dec2)
{
    double x1, y1, z1, x2, y2, z2;
    radec2xyz(ra1, dec1, x1, y1, z1);
    radec2xyz(ra2, dec2, x2, y2, z2);
    return chord2(x1, y1, z1, x2, y2, z2);
}

// Without distances the chord is needed only for the few pairs inside the FP32
// margin band: out of line, which measured faster than inlined (3.75 against
// 4.05 ms at 50M x 50M).  With distances it runs for every match: inlined
// (4.95 against 6.19 ms).
__device__ __noinline__ double chord2_radec_call(double ra1, double dec1, double ra2, double dec2)
{
    return chord2_radec_inl(ra1, dec1, ra2, dec2);
}

template <bool DIST>
__device__ __forceinline__ double chord2_radec(double ra1, double dec1, double ra2, double dec2)
{
    return DIST ? chord2_radec_inl(ra1, dec1, ra2, dec2) : chord2_radec_call(ra1, dec1, ra2, dec2);
}

// A source (a thread's object).
struct AObj {
    double ra, dec;
    float fx, fy, fz;
    double alpha;
    long long id;
    uint32_t gi;        // index in the A segment
    int zone;
    bool full_ring;     // alpha >= 3: every object of a zone is a candidate
    Win w;              // quantised windows
};

// View of B for window enumeration.
//   WHOLE  (staged, whole): band zone zb -> [zoff[k] - base, zoff[k+1] - base),
//          k = zb - band_lo, global index = base + q;
//   UNION  (staged): band zone k -> [off[k], off[k+1]), global g[k] + (q - off[k]);
//   global: zone zb -> [zoff[zb], zoff[zb+1]) of the segment itself.
struct BView {
    const float4 *xyz;
    bool staged, whole;
    int band_lo;
    uint32_t base, len;     // WHOLE: staged objects are [base, base + len) of the segment
    const uint32_t *off;
    const uint32_t *g;
    const uint32_t *zoff;
    const uint16_t *bins;   // WHOLE: bin index rows of the band's zones (bin_log2 > 0)
    int bin_log2;
};

constexpr int kRaqBitsB = 27;   // quantised-ra bits of the segments (xyz.w)

// Candidate enumeration state: B zones of the band, and in each zone up to
// three ra windows (direct, branch 2 with B near 0, branch 3 with B near 2 pi).
struct Cursor {
    int zb, zb_end;
    int win;                // 0 direct, 1 branch 2, 2 branch 3
    uint32_t j, j_end;      // candidate positions (view indices) of the current window
    uint32_t b0, b1;        // current zone range (view indices)
    uint32_t hi_cur;        // raq upper end of the current window
    uint32_t w1_lo, w1_hi;  // direct window (keeps the wrapped ones disjoint from it)
};

__device__ __forceinline__ uint32_t lower_v(const BView &V, uint32_t lo, uint32_t hi, uint32_t t)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (raq_at(V.xyz, mid) < t) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t upper_v(const BView &V, uint32_t lo, uint32_t hi, uint32_t t)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (raq_at(V.xyz, mid) <= t) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// First k in [lo, end) with raq[k] > t, by galloping from lo: a window holds
// few objects, so the common answers (lo, lo + 1) take one or two loads.
__device__ __forceinline__ uint32_t upper_gallop(const BView &V, uint32_t lo, uint32_t end, uint32_t t)
{
    uint32_t step = 1, b;
    for (;;) {                     // every k in [lo_start, lo) has raq[k] <= t
        b = lo + step - 1;
        if (b >= end) {
            b = end;
            break;
        }
        if (raq_at(V.xyz, b) > t) break;   // answer in [lo, b]
        lo = b + 1;
        step <<= 1;
    }
    return upper_v(V, lo, b, t);
}

// Narrows [lo, hi), the view positions of B zone zb, to the bin of raq t in the
// zone's bin index (when the view carries one): the first object with raq >= t
// lies between the start of t's bin and the start of the next bin.  Staged
// WHOLE views index the band's rows and clip to the staged piece as zone_range
// does; the global view indexes the segment's rows.
__device__ __forceinline__ void bins_narrow(const BView &V, int zb, uint32_t t, uint32_t &lo, uint32_t &hi)
{
    if (!V.bin_log2 || (V.staged && !V.whole)) return;
    const uint32_t kk = V.staged ? (uint32_t)(zb - V.band_lo) : (uint32_t)zb;
    const uint32_t zs = V.zoff[kk], ze = V.zoff[kk + 1];
    if (ze - zs >= 0xFFFFu) return;   // the index saturates: bisect the whole zone
    const uint32_t bin = t >> (kRaqBitsB - V.bin_log2);
    const uint16_t *row = V.bins + ((size_t)kk << V.bin_log2);
    uint32_t s0 = zs + (bin ? (uint32_t)row[bin - 1] : 0u), s1 = zs + (uint32_t)row[bin];
    if (V.staged) {
        s0 = min(max(s0, V.base), V.base + V.len) - V.base;
        s1 = min(max(s1, V.base), V.base + V.len) - V.base;
    }
    lo = s0;
    hi = s1;
}

__device__ __forceinline__ void open_window(const BView &V, const AObj &a, Cursor &c)
{
    c.j = c.j_end = 0;
    if (a.full_ring) {
        if (c.win != 0) return;
        c.j = c.b0;
        c.j_end = c.b1;
        c.hi_cur = 0xFFFFFFFFu;
        return;
    }
    if (c.win == 0) {
        uint32_t lo = c.b0, hi = c.b1;
        bins_narrow(V, c.zb, a.w.lo, lo, hi);
        c.j = lower_v(V, lo, hi, a.w.lo);
        c.j_end = c.b1;
        c.hi_cur = a.w.hi;
        c.w1_lo = c.j;
        c.w1_hi = c.j;
        return;
    }
    if (c.win == 1) {   // branch 2: below the direct window
        if (a.w.hi2 < raq_at(V.xyz, c.b0)) return;
        c.j = lower_v(V, c.b0, c.w1_lo, a.w.lo2);
        c.j_end = c.w1_lo;
        c.hi_cur = a.w.hi2;
        return;
    }
    // branch 3: above the direct window
    if (a.w.lo3 > raq_at(V.xyz, c.b1 - 1)) return;
    c.j = lower_v(V, c.w1_hi, c.b1, a.w.lo3);
    c.j_end = c.b1;
    c.hi_cur = a.w.hi3;
}

__device__ __forceinline__ bool next_candidate(const BView &V, const AObj &a, Cursor &c, uint32_t &out)
{
    for (;;) {
        if (c.j < c.j_end) {
            const uint32_t j = c.j;
            if (raq_at(V.xyz, j) <= c.hi_cur) {
                c.j = j + 1;
                if (c.win == 0) c.w1_hi = c.j;
                out = j;
                return true;
            }
            c.j = c.j_end;
        }
        if (c.win < 2 && !a.full_ring) {
            c.win++;
            open_window(V, a, c);
            continue;
        }
        c.zb++;
        if (c.zb > c.zb_end) return false;
        if (V.whole) {
            const int k = c.zb - V.band_lo;
            c.b0 = min(max(V.zoff[k], V.base), V.base + V.len) - V.base;
            c.b1 = min(max(V.zoff[k + 1], V.base), V.base + V.len) - V.base;
        } else if (V.staged) {
            const int k = c.zb - V.band_lo;
            c.b0 = V.off[k];
            c.b1 = V.off[k + 1];
        } else {
            c.b0 = __ldg(&V.zoff[c.zb]);
            c.b1 = __ldg(&V.zoff[c.zb + 1]);
        }
        c.win = 0;
        if (c.b0 >= c.b1) {
            c.j = c.j_end = 0;
            c.win = 2;
            continue;
        }
        open_window(V, a, c);
    }
}

__device__ __forceinline__ uint32_t global_index(const BView &V, int zb, uint32_t q)
{
    if (V.whole) return V.base + q;
    if (!V.staged) return q;
    const int k = zb - V.band_lo;
    return V.g[k] + (q - V.off[k]);
}

struct Counters {
    unsigned long long tested, cand, border, exact;
};

__device__ __forceinline__ bool cuts_pass(const JobDev &J, const AObj &a, double2 rb)
{
    if (!(fabs(__dsub_rn(a.dec, rb.y)) < J.sr_rad)) return false;
    const double d = __dsub_rn(a.ra, rb.x);
    return fabs(d) < a.alpha || fabs(__dsub_rn(d, XM_TWO_PI)) < a.alpha || fabs(__dadd_rn(d, XM_TWO_PI)) < a.alpha;
}

__device__ __forceinline__ int find_job(const JobDev *__restrict__ jobs, int n_jobs, uint32_t item)
{
    int lo = 0, hi = n_jobs;   // last j with item_begin <= item
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(&jobs[mid].item_begin) <= item) lo = mid; else hi = mid;
    }
    return lo;
}

// Per-warp match buffer: 64 entries, written out 32 at a time.  Each round of
// phase 2 adds at most 32 matches to a buffer holding fewer than 32, so the
// staged path never overflows it.
constexpr int kWarpBuf = 64;

constexpr int kMaxRanges = 9;   // 3 windows x up to 3 zones per lane; beyond that the cursor path

// Per-warp candidate ranges of phase 1: start | length << 16 (staged indices < 2^16).
struct WList {
    uint32_t r[32][kMaxRanges];
    uint32_t mark[32];             // phase 2: 1 + the lane whose candidates start at this position
    double alpha[32];
};

// An entry holds idA and (job << 32 | index of the B object in its segment);
// idB is loaded when the entry is written out, all lanes at once, instead of
// one dependent load per match.  Distances are held only by the DIST kernels.
template <bool DIST>
struct WBufT {
    longlong2 ab[kWarpBuf];     // idA, job << 32 | B index
    double d[DIST ? kWarpBuf : 1];
    uint32_t count;             // entries [0, min(count, kWarpBuf)) are held; the rest went out directly
};

// Where B's ids are: in the consumer's current job, or for entries left from a
// previous tile of a batch, in that job's entry of the job table.
struct IdSrc {
    const JobDev *jobs;
    const JobDev *cur;          // the current job's entry
    int job;                    // its index
    __device__ __forceinline__ long long id_of(unsigned long long e) const
    {
        const int j = (int)(e >> 32);
        const long long *p = (j == job ? cur : jobs + j)->b_id;
        return __ldg(p + (uint32_t)e);
    }
};

__device__ __forceinline__ long long b_entry(uint32_t job, uint32_t gq)
{
    return (long long)(((unsigned long long)job << 32) | gq);
}

// Warp-aggregated append of this iteration's matches to the warp's buffer
// (gq: index of the matched B object in its segment).  Entries beyond the
// buffer, which only the per-lane cursor path can produce, are written out
// directly.
template <bool DIST>
__device__ __forceinline__ void emit_w(WBufT<DIST> &wb, const MatchOut &out, const IdSrc &ids, bool m, long long ida,
                                       uint32_t gq, double dist, uint32_t job)
{
    const unsigned act = __activemask();
    const unsigned bal = __ballot_sync(act, m);
    if (!m) return;
    const int leader = __ffs(bal) - 1;
    const unsigned lane = threadIdx.x & 31;
    const uint32_t n = (uint32_t)__popc(bal);
    const uint32_t rank = (uint32_t)__popc(bal & lanemask_lt());
    uint32_t base = 0;
    if ((int)lane == leader) {
        base = wb.count;
        wb.count = base + n;
    }
    base = __shfl_sync(bal, base, leader);
    const uint32_t slot = base + rank;
    if (slot < (uint32_t)kWarpBuf) {
        wb.ab[slot] = make_longlong2(ida, b_entry(job, gq));
        if (DIST) wb.d[slot] = dist;
    }
    if (base + n <= (uint32_t)kWarpBuf) return;
    const uint32_t keep = base >= (uint32_t)kWarpBuf ? 0u : (uint32_t)kWarpBuf - base;
    unsigned over = bal;
    for (uint32_t q = 0; q < keep; ++q) over &= over - 1;
    if (slot < (uint32_t)kWarpBuf) return;
    const int l2 = __ffs(over) - 1;
    unsigned long long g = 0;
    if ((int)lane == l2) g = atomicAdd(&out.counters[0], (unsigned long long)__popc(over));
    const long long idb = ids.id_of((unsigned long long)b_entry(job, gq));
    g = __shfl_sync(over, g, l2);
    g += (unsigned long long)__popc(over & lanemask_lt());
    if (g < out.cap) {
        reinterpret_cast<longlong2 *>(out.pairs)[g] = make_longlong2(ida, idb);
        if (DIST && out.dist) out.dist[g] = dist;
        if (out.job) out.job[g] = job;
    }
}

// Whole warp (converged): writes out the buffer's first min(count, 32)
// entries -- one atomicAdd reserves their output slots, the idB loads are
// issued under it, then entry k is stored by lane k (coalesced) -- and moves
// the rest to the front.
template <bool DIST>
__device__ __forceinline__ void out_flush(WBufT<DIST> &wb, const MatchOut &out, const IdSrc &ids)
{
    __syncwarp();
    const unsigned lane = threadIdx.x & 31;
    const uint32_t held = min(wb.count, (uint32_t)kWarpBuf);
    const uint32_t n = min(held, 32u);
    unsigned long long g = 0;
    if (lane == 0 && n) g = atomicAdd(&out.counters[0], (unsigned long long)n);
    longlong2 e = make_longlong2(0, 0);
    double d = 0;
    uint32_t jb = 0;
    if (lane < n) {
        e = wb.ab[lane];
        jb = (uint32_t)((unsigned long long)e.y >> 32);
        e.y = ids.id_of((unsigned long long)e.y);
        if (DIST) d = wb.d[lane];
    }
    const uint32_t rest = held - n;
    longlong2 e2 = make_longlong2(0, 0);
    double d2 = 0;
    if (lane < rest) {
        e2 = wb.ab[32 + lane];
        if (DIST) d2 = wb.d[32 + lane];
    }
    __syncwarp();
    if (lane < rest) {
        wb.ab[lane] = e2;
        if (DIST) wb.d[lane] = d2;
    }
    if (lane == 0) wb.count = rest;
    g = __shfl_sync(0xffffffffu, g, 0) + lane;
    if (lane < n && g < out.cap) {
        reinterpret_cast<longlong2 *>(out.pairs)[g] = e;
        if (DIST && out.dist) out.dist[g] = d;
        if (out.job) out.job[g] = jb;
    }
    __syncwarp();
}

// Per-tile job scalars kept in registers.  The FP32-filter kernels read the
// FP64 radius and chord threshold from the job entry for the few pairs that
// need them (inside the margin band, full-ring zones) instead of holding them.
struct JobScalars {
    double sr_rad, sr_dist2;
    float thr_hi, thr_lo;
    int n_zones, nz;
    int raq_shift;
};

__device__ __forceinline__ JobScalars load_scalars(const JobDev &J)
{
    JobScalars k;
    k.sr_rad = J.sr_rad;
    k.sr_dist2 = J.sr_dist2;
    k.thr_hi = J.thr_hi;
    k.thr_lo = J.thr_lo;
    k.n_zones = J.n_zones;
    k.nz = J.nz;
    k.raq_shift = J.raq_shift;
    return k;
}

__device__ __forceinline__ bool cuts_k(double sr_rad, double ra_a, double dec_a, double alpha, double2 rb)
{
    if (!(fabs(__dsub_rn(dec_a, rb.y)) < sr_rad)) return false;
    const double d = __dsub_rn(ra_a, rb.x);
    return fabs(d) < alpha || fabs(__dsub_rn(d, XM_TWO_PI)) < alpha || fabs(__dadd_rn(d, XM_TWO_PI)) < alpha;
}

// Staged index range of band zone zb (clipped to the staged piece for WHOLE).
__device__ __forceinline__ void zone_range(const BView &V, int zb, uint32_t &b0, uint32_t &b1)
{
    const int k = zb - V.band_lo;
    if (V.whole) {
        b0 = min(max(V.zoff[k], V.base), V.base + V.len) - V.base;
        b1 = min(max(V.zoff[k + 1], V.base), V.base + V.len) - V.base;
    } else {
        b0 = V.off[k];
        b1 = V.off[k + 1];
    }
}

// lane_ranges for at most three B zones with an RA cut (nz = 1): the three
// direct-window bisections run interleaved, one step of each per iteration,
// so that their shared-memory loads overlap; the upper ends are galloped.
__device__ __forceinline__ int lane_ranges3(const BView &V, const Win &w, int zlo, int zhi, uint32_t *rr, int &nr)
{
    uint32_t b0[3], b1[3], lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        b0[k] = b1[k] = 0;
        if (zlo + k <= zhi) zone_range(V, zlo + k, b0[k], b1[k]);
        lo[k] = b0[k];
        hi[k] = b1[k];
        if (zlo + k <= zhi) bins_narrow(V, zlo + k, w.lo, lo[k], hi[k]);
    }
    // first k in [b0, b1) with raq >= w.lo, per zone
    while (lo[0] < hi[0] || lo[1] < hi[1] || lo[2] < hi[2]) {
        uint32_t v[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) v[k] = raq_at(V.xyz, lo[k] < hi[k] ? (lo[k] + hi[k]) >> 1 : 0u);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (lo[k] < hi[k]) {
                const uint32_t mid = (lo[k] + hi[k]) >> 1;
                if (v[k] < w.lo) lo[k] = mid + 1; else hi[k] = mid;
            }
        }
    }
    int total = 0;
    nr = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint32_t j0 = lo[k];
        uint32_t j1 = j0;
        if (j0 < b1[k] && raq_at(V.xyz, j0) <= w.hi) j1 = upper_gallop(V, j0 + 1, b1[k], w.hi);
        if (j1 > j0) {
            rr[nr++] = j0 | ((j1 - j0) << 16);
            total += (int)(j1 - j0);
        }
        if (b0[k] >= b1[k]) continue;
        if (w.lo2 <= w.hi2 && w.hi2 >= raq_at(V.xyz, b0[k])) {
            const uint32_t w0 = lower_v(V, b0[k], j0, w.lo2);
            const uint32_t w1 = upper_gallop(V, w0, j0, w.hi2);
            if (w1 > w0) {
                rr[nr++] = w0 | ((w1 - w0) << 16);
                total += (int)(w1 - w0);
            }
        }
        if (w.lo3 <= w.hi3 && w.lo3 <= raq_at(V.xyz, b1[k] - 1)) {
            const uint32_t w0 = lower_v(V, j1, b1[k], w.lo3);
            const uint32_t w1 = upper_gallop(V, w0, b1[k], w.hi3);
            if (w1 > w0) {
                rr[nr++] = w0 | ((w1 - w0) << 16);
                total += (int)(w1 - w0);
            }
        }
    }
    return total;
}

// Phase 1: a lane's candidate ranges in the staged view (same sets as the
// cursor enumeration of next_candidate).  Returns the number of candidates,
// or -1 if the ranges do not fit the per-lane list.
__device__ __forceinline__ int lane_ranges(const BView &V, const JobScalars &K, const Win &w, bool full_ring,
                                           int zone, uint32_t *rr, int &nr)
{
    nr = 0;
    int total = 0;
    const int zlo = max(0, zone - K.nz), zhi = min(K.n_zones - 1, zone + K.nz);
    if (!full_ring && zhi - zlo <= 2) return lane_ranges3(V, w, zlo, zhi, rr, nr);
    for (int zb = zlo; zb <= zhi; ++zb) {
        uint32_t b0, b1;
        const int k = zb - V.band_lo;
        if (V.whole) {
            b0 = min(max(V.zoff[k], V.base), V.base + V.len) - V.base;
            b1 = min(max(V.zoff[k + 1], V.base), V.base + V.len) - V.base;
        } else {
            b0 = V.off[k];
            b1 = V.off[k + 1];
        }
        if (b0 >= b1) continue;
        // append [s, e) to the lane's list
#define XM_PUSH(s_, e_)                                    \
    do {                                                   \
        if ((e_) > (s_)) {                                 \
            if (nr == kMaxRanges) return -1;               \
            rr[nr++] = (s_) | (((e_) - (s_)) << 16);       \
            total += (int)((e_) - (s_));                   \
        }                                                  \
    } while (0)
        if (full_ring) {
            XM_PUSH(b0, b1);
        } else {
            uint32_t s0 = b0, s1 = b1;
            bins_narrow(V, zb, w.lo, s0, s1);
            const uint32_t j0 = lower_v(V, s0, s1, w.lo);
            const uint32_t j1 = upper_gallop(V, j0, b1, w.hi);
            XM_PUSH(j0, j1);
            if (w.lo2 <= w.hi2 && w.hi2 >= raq_at(V.xyz, b0)) {
                const uint32_t w0 = lower_v(V, b0, j0, w.lo2);
                const uint32_t w1 = upper_gallop(V, w0, j0, w.hi2);
                XM_PUSH(w0, w1);
            }
            if (w.lo3 <= w.hi3 && w.lo3 <= raq_at(V.xyz, b1 - 1)) {
                const uint32_t w0 = lower_v(V, j1, b1, w.lo3);
                const uint32_t w1 = upper_gallop(V, w0, b1, w.hi3);
                XM_PUSH(w0, w1);
            }
        }
#undef XM_PUSH
    }
    return total;
}

// Zone of A object i of the staged tile; -1 if the offsets disagree.
template <class Stage>
__device__ __forceinline__ int a_zone_s(const Stage &S, uint32_t i)
{
    if (S.zf == S.zl) return S.zf;
    const uint32_t *zo = S.azo_s + S.azo_skew;   // zo[k] = a_zoff[zf + k]
    int lo = 0, hi = S.zl - S.zf;                // last k with zo[k] <= i
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (zo[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return (zo[lo] <= i && i < zo[lo + 1]) ? S.zf + lo : -1;
}

// Staged B index -> global B index.
__device__ __forceinline__ uint32_t staged_global(const BView &V, int nseg, uint32_t q)
{
    if (V.whole) return V.base + q;
    int k = 0;
    while (k + 1 < nseg && V.off[k + 1] <= q) ++k;
    return V.g[k] + (q - V.off[k]);
}

// All candidates of one A object against the view; emits matches.
template <int VARIANT, bool COUNT_CAND, bool DIST>
__device__ __forceinline__ void test_object(const JobDev &J, AObj &a, const BView &V, WBufT<DIST> &wb,
                                            const MatchOut &out, const IdSrc &ids, uint32_t jx, Counters &cn)
{
    a.w = make_win(a.ra, a.alpha, J.raq_shift);
    Cursor c;
    c.zb = max(0, a.zone - J.nz) - 1;
    c.zb_end = min(J.n_zones - 1, a.zone + J.nz);
    c.win = 2;
    c.j = c.j_end = 0;
    c.b0 = c.b1 = 0;
    c.hi_cur = 0;
    c.w1_lo = c.w1_hi = 0;
    uint32_t q;
    while (next_candidate(V, a, c, q)) {
        cn.tested++;
        bool m = false;
        double c2 = 0;
        const double2 rb = __ldg(&J.b_radec[global_index(V, c.zb, q)]);
        if (VARIANT == 0) {   // FP32 reject above thr_hi, accept below thr_lo, FP64 decision between
            if (COUNT_CAND) cn.cand += cuts_pass(J, a, rb) ? 1ull : 0ull;
            const float4 fb = V.xyz[q];
            const float dx = a.fx - fb.x, dy = a.fy - fb.y, dz = a.fz - fb.z;
            const float c32 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            if (!(c32 > J.thr_hi)) {
                const bool band = c32 >= J.thr_lo;
                cn.border += band ? 1ull : 0ull;
                if (cuts_pass(J, a, rb)) {
                    m = true;
                    if (band || DIST) {
                        c2 = chord2_radec<DIST>(a.ra, a.dec, rb.x, rb.y);
                        if (band) {
                            cn.exact++;
                            m = c2 < J.sr_dist2;
                        }
                    }
                }
            }
        } else {              // plain all-FP64: cuts, then unit vectors by sincos per pair
            if (cuts_pass(J, a, rb)) {
                cn.cand++;
                cn.exact++;
                double x1, y1, z1, x2, y2, z2;
                radec2xyz(a.ra, a.dec, x1, y1, z1);
                radec2xyz(rb.x, rb.y, x2, y2, z2);
                c2 = chord2(x1, y1, z1, x2, y2, z2);
                m = c2 < J.sr_dist2;
            }
        }
        uint32_t gq = 0;
        double dist = 0;
        if (m) {
            gq = global_index(V, c.zb, q);
            if (DIST) dist = 2.0 * asin(sqrt(c2) * 0.5);
        }
        emit_w<DIST>(wb, out, ids, m, a.id, gq, dist, jx);
    }
}

// ---------------------------------------------------------------------------
// Tile plans (pre-pass, one thread per work item)
// ---------------------------------------------------------------------------
constexpr int kMaxBand = 72;       // B zones a staged band may span
constexpr int kMaxPlanSeg = 4;     // per-zone windows of a UNION plan
constexpr uint32_t kHeavyPairs = 16384;   // pairs above which a full-ring tile is split along B
constexpr uint32_t kMaxPieces = 1024;

enum : uint32_t { PLAN_WHOLE = 0, PLAN_UNION = 1, PLAN_GLOBAL = 2 };

struct __align__(16) TilePlan {    // 64 bytes
    uint32_t a_start, a_len;
    uint32_t mode;                 // mode | nseg << 8 | (zl - zf) << 16 (nseg = band zones)
    int32_t zf;                    // first A zone of the tile
    int32_t band_lo;
    uint32_t job;
    uint32_t b_start, b_len;       // WHOLE: the band's contiguous B range; UNION: total staged
    uint32_t seg_g[kMaxPlanSeg];   // UNION: first staged B object of band zone k
    uint32_t seg_len[kMaxPlanSeg];
};
static_assert(sizeof(TilePlan) == 64, "plan layout");

__device__ __forceinline__ void store_plan(TilePlan *dst, const TilePlan &P)
{
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    d[0] = make_uint4(P.a_start, P.a_len, P.mode, (uint32_t)P.zf);
    d[1] = make_uint4((uint32_t)P.band_lo, P.job, P.b_start, P.b_len);
    d[2] = make_uint4(P.seg_g[0], P.seg_g[1], P.seg_g[2], P.seg_g[3]);
    d[3] = make_uint4(P.seg_len[0], P.seg_len[1], P.seg_len[2], P.seg_len[3]);
}

// Cuts work item `item` into tiles (see the file header); calls f(start, len, zf, zl).
// Zone offsets of A and B and RA half-widths of A's zones, read from shared
// memory when a work item's slice is cached there, else from the job's arrays.
struct ZoneView {
    const uint32_t *azo;
    int az0;               // a_zoff[z] = azo[z - az0]
    const uint32_t *bzo;
    int bz0;
    const double *al;
    int al0;
    __device__ __forceinline__ uint32_t a(int z) const { return azo[z - az0]; }
    __device__ __forceinline__ uint32_t b(int z) const { return bzo[z - bz0]; }
    __device__ __forceinline__ double alpha(int z) const { return al[z - al0]; }
};

__device__ __forceinline__ ZoneView global_view(const JobDev &J)
{
    return ZoneView{J.a_zoff, 0, J.b_zoff, 0, J.alpha, J.alpha_z0};
}

template <class F>
__device__ __forceinline__ void for_each_tile(const JobDev &J, const ZoneView &V, uint32_t item, uint32_t zc,
                                              uint32_t tile, F f)
{
    const int z0 = J.z_lo + (int)((item - J.item_begin) * zc);
    const int z1 = min(z0 + (int)zc, J.z_hi + 1);
    int z = z0;
    uint32_t pos = V.a(z0);
    while (true) {
        while (z < z1 && pos >= V.a(z + 1)) {
            ++z;
            pos = max(pos, V.a(z));
        }
        if (z >= z1) return;
        const uint32_t zb0 = V.a(z), zb1 = V.a(z + 1);
        const uint32_t cnt = zb1 - zb0;
        if (cnt > tile / 2) {            // large zone: near-equal single-zone tiles
            const uint32_t k = (cnt + tile - 1) / tile;
            const uint32_t size = (cnt + k - 1) / k;
            const uint32_t len = min(size, zb1 - pos);
            f(pos, len, z, z);
            pos += len;
        } else {                         // consecutive small zones packed together
            const uint32_t start = pos;
            uint32_t end = zb1;
            int zl = z, zn = z + 1;
            while (zn < z1) {
                const uint32_t e1 = V.a(zn + 1);
                const uint32_t c1 = e1 - V.a(zn);
                if (c1 > tile / 2 || e1 - start > tile) break;
                if (c1 > 0) {
                    zl = zn;
                    end = e1;
                }
                ++zn;
            }
            f(start, end - start, z, zl);
            pos = end;
            z = zn;
        }
    }
}

// Tiles whose B band does not fit one stage are split along B into pieces,
// each staged and tested as its own WHOLE plan over a consecutive B range
// (the pair kernel clips every zone's window to the piece):
//  - a tile whose zones have no RA cut (alpha >= 3, near the poles) tests its
//    whole band; when that is many pairs it is cut into pieces of at most
//    cap_b objects that go to the "heavy" queue the pair kernel hands out
//    first, one at a time;
//  - a tile whose objects cover the whole RA ring (several packed zones, or
//    one whole small zone) has no narrower union of windows to stage; when
//    its band holds more than cap_b objects it is cut into at most
//    kMaxSplit near-equal normal pieces (beyond that, the global cursor).
// Returns the number of pieces (1 = not split), the piece size and the queue.
constexpr uint32_t kMaxSplit = 8;

__device__ __forceinline__ uint32_t tile_pieces(const JobDev &J, const ZoneView &V, uint32_t len, int zf, int zl,
                                                uint32_t tile, uint32_t cap_b, uint32_t *piece, bool *heavy)
{
    const int band_lo = max(0, zf - J.nz), band_hi = min(J.n_zones - 1, zl + J.nz);
    const uint32_t nseg = (uint32_t)(band_hi - band_lo + 1);
    const uint32_t b_len = V.b(band_hi + 1) - V.b(band_lo);
    *piece = b_len;
    *heavy = false;
    if ((int)nseg > kMaxBand) return 1;
    const bool full_ring = V.alpha(zf) >= 3.0 || V.alpha(zl) >= 3.0;
    if (full_ring && (uint64_t)len * b_len > kHeavyPairs) {
        uint32_t pc = max(32u, kHeavyPairs / max(len, 1u));
        pc = min(pc, cap_b);
        uint32_t n = (b_len + pc - 1) / pc;
        if (n > kMaxPieces) {
            pc = (b_len + kMaxPieces - 1) / kMaxPieces;
            if (pc > cap_b) return 1;
            n = (b_len + pc - 1) / pc;   // every piece starts inside the band
        }
        if (n <= 1) return 1;
        *piece = pc;
        *heavy = true;
        return n;
    }
    if (b_len > cap_b && (zf != zl || 2 * len <= tile)) {
        const uint32_t n = (b_len + cap_b - 1) / cap_b;
        if (n > kMaxSplit) return 1;
        *piece = (b_len + n - 1) / n;
        return n;
    }
    return 1;
}

// Tiles per work item: cnt[item] normal plans, cnt[n_items + item] heavy pieces.
__global__ void tiles_count(const JobDev *__restrict__ jobs, int n_jobs, uint32_t n_items, uint32_t zc,
                            uint32_t tile, uint32_t cap_b, uint32_t *__restrict__ cnt)
{
    const uint32_t item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= n_items) return;
    const JobDev &J = jobs[n_jobs > 1 ? find_job(jobs, n_jobs, item) : 0];
    uint32_t c = 0, h = 0;
    const ZoneView V = global_view(J);
    for_each_tile(J, V, item, zc, tile, [&](uint32_t, uint32_t len, int zf, int zl) {
        uint32_t piece;
        bool heavy;
        const uint32_t n = tile_pieces(J, V, len, zf, zl, tile, cap_b, &piece, &heavy);
        if (heavy) h += n; else c += n;
    });
    cnt[item] = c;
    cnt[n_items + item] = h;
}

// Plans: heavy pieces first (off[n_items + item] within [0, n_heavy)), then the
// normal ones (n_heavy + off[item]).  One warp per work item: the item's zone
// offsets and RA half-widths are first loaded into shared memory by all lanes
// at once, then every lane walks the tiles in step (uniform control flow, the
// same values); lane 0 writes the normal plans, all lanes the heavy pieces.
constexpr int kMakeWarps = 4;
constexpr int kZcMax = 64;           // zones per work item at most (xm_run_jobs checks)
constexpr int kBandCache = 224;      // B zone offsets cached per item

__global__ void __launch_bounds__(32 * kMakeWarps)
tiles_make(const JobDev *__restrict__ jobs, int n_jobs, uint32_t n_items, uint32_t zc, uint32_t tile, uint32_t cap_b,
           const uint32_t *__restrict__ off_n, const uint32_t *__restrict__ off_h, TilePlan *__restrict__ plans,
           uint32_t max_tiles, unsigned long long *err)
{
    __shared__ uint32_t s_azo[kMakeWarps][kZcMax + 1];
    __shared__ uint32_t s_bzo[kMakeWarps][kBandCache];
    __shared__ double s_al[kMakeWarps][kZcMax];
    const int w = threadIdx.x >> 5;
    const unsigned lane = threadIdx.x & 31;
    const uint32_t item = blockIdx.x * kMakeWarps + w;
    if (item >= n_items) return;   // whole warp
    const int jx = n_jobs > 1 ? find_job(jobs, n_jobs, item) : 0;
    const JobDev &J = jobs[jx];
    const int z0 = J.z_lo + (int)((item - J.item_begin) * zc);
    const int z1 = min(z0 + (int)zc, J.z_hi + 1);
    const int nza = z1 - z0;
    const int blo = max(0, z0 - J.nz), bhi = min(J.n_zones - 1, z1 - 1 + J.nz);
    const int nbo = bhi + 2 - blo;   // B offsets [blo, bhi + 1]
    ZoneView V = global_view(J);
    if (nza <= kZcMax && nbo <= kBandCache) {
        for (int k = lane; k <= nza; k += 32) s_azo[w][k] = __ldg(&J.a_zoff[z0 + k]);
        for (int k = lane; k < nbo; k += 32) s_bzo[w][k] = __ldg(&J.b_zoff[blo + k]);
        for (int k = lane; k < nza; k += 32) s_al[w][k] = __ldg(&J.alpha[z0 + k - J.alpha_z0]);
        __syncwarp();
        V = ZoneView{s_azo[w], z0, s_bzo[w], blo, s_al[w], z0};
    }
    const uint32_t n_heavy = off_h[n_items];
    uint32_t o = n_heavy + off_n[item];
    uint32_t oh = off_h[item];
    for_each_tile(J, V, item, zc, tile, [&](uint32_t start, uint32_t len, int zf, int zl) {
        TilePlan P;
        P.a_start = start;
        P.a_len = len;
        P.job = (uint32_t)jx;
        const int band_lo = max(0, zf - J.nz), band_hi = min(J.n_zones - 1, zl + J.nz);
        P.band_lo = band_lo;
        P.zf = zf;
        const uint32_t nseg = (uint32_t)(band_hi - band_lo + 1);
        const uint32_t B0 = V.b(band_lo), B1 = V.b(band_hi + 1);
        P.b_start = B0;
        P.b_len = B1 - B0;
        for (int k = 0; k < kMaxPlanSeg; ++k) P.seg_g[k] = P.seg_len[k] = 0;
        const uint32_t zword = (min(nseg, 255u) << 8) | ((uint32_t)(zl - zf) << 16);
        uint32_t piece;
        bool heavy;
        const uint32_t npc = tile_pieces(J, V, len, zf, zl, tile, cap_b, &piece, &heavy);
        if (npc > 1) {
            // WHOLE plans over consecutive B pieces of the band, one per lane
            P.mode = PLAN_WHOLE | zword;
            uint32_t &dst = heavy ? oh : o;
            for (uint32_t q = lane; q < npc; q += 32) {
                TilePlan Q = P;
                Q.b_start = B0 + q * piece;
                Q.b_len = min(piece, B1 - Q.b_start);
                if (dst + q < max_tiles) store_plan(plans + dst + q, Q);
                else atomicExch(err, 1ull);
            }
            dst += npc;
            return;
        }
        uint32_t mode = PLAN_GLOBAL;
        if ((int)nseg <= kMaxBand && P.b_len <= cap_b) {
            mode = PLAN_WHOLE;
        } else if (zf == zl && (int)nseg <= kMaxPlanSeg && V.alpha(zf) < 3.0) {
            const double alpha = V.alpha(zf);
            // A is ordered by raq: every tile object's ra is within one raq step q of
            // [ra_first, ra_last]; widen by 2q
            const double q2 = 2.0 * ldexp(XM_TWO_PI, J.raq_shift - 32);
            const double ra_f = J.a_radec[start].x - q2, ra_l = J.a_radec[start + len - 1].x + q2;
            const int sh = J.raq_shift;
            const uint32_t t_lo = xm::raq32(ra_f - alpha - kWinEps) >> sh;
            const uint32_t t_hi = xm::raq32(ra_l + alpha + kWinEps) >> sh;
            const uint32_t t_hi2 = xm::raq32(ra_l + alpha + 2 * kWinEps - XM_TWO_PI) >> sh;
            const uint32_t t_lo3 = xm::raq32(ra_f - alpha - 2 * kWinEps + XM_TWO_PI) >> sh;
            uint32_t total = 0;
#pragma unroll
            for (int k = 0; k < kMaxPlanSeg; ++k) {
                if (k >= (int)nseg) break;
                const uint32_t b0 = V.b(band_lo + k), b1 = V.b(band_lo + k + 1);
                uint32_t sb = b0, ln = b1 - b0;
                if (ln > 0) {
                    const bool wrap = !(t_hi2 < raq_at_g(J.b_xyz, b0) && t_lo3 > raq_at_g(J.b_xyz, b1 - 1));
                    if (!wrap) {
                        sb = lower_raq_g(J.b_xyz, b0, b1, t_lo);
                        ln = upper_raq_g(J.b_xyz, sb, b1, t_hi) - sb;
                    }
                }
                P.seg_g[k] = sb;
                P.seg_len[k] = ln;
                total += ln;
            }
            if (total <= cap_b) {
                mode = PLAN_UNION;
                P.b_len = total;
            }
        }
        // nseg is only read for WHOLE (<= kMaxBand) and UNION (<= kMaxPlanSeg) plans
        P.mode = mode | zword;
        if (lane == 0) {
            if (o < max_tiles) store_plan(plans + o, P);
            else atomicExch(err, 1ull);
        }
        ++o;
    });
}

// ---------------------------------------------------------------------------
// Warp-specialised pair kernel: warp 0 produces (bulk copies into a ring of
// stages), warps 1..C consume (one A object per thread).
// ---------------------------------------------------------------------------
// B's ra/dec are staged only for the all-FP64 variant (RADEC), which cuts every
// candidate; the FP32 filter reads them from global memory for the few pairs
// inside its margin band.  Without them a stage is small enough for three.
constexpr int kBinZones = 8;   // band zones whose bin index rows a stage carries

template <int TILE, bool RADEC>
struct StageT {
    static constexpr int kCapB = 4 * TILE;
    static constexpr int kStages = RADEC ? 2 : 3;
    double2 b_radec[RADEC ? kCapB : 1];
    float4 b_xyz[kCapB];
    double2 a_radec[TILE];
    float4 a_xyz[TILE];
    long long a_id[TILE + 2];
    uint32_t zoff[kMaxBand + 8];   // B zone offsets of the band (WHOLE), 16-byte aligned copy
    // descriptor (written by the producer before the full-barrier arrive)
    uint32_t a_start, a_len, mode, nseg;
    int32_t band_lo, zf, zl;
    uint32_t job, b_start, b_len, id_skew, zoff_skew, done;
    uint32_t seg_off[kMaxPlanSeg + 1];
    uint32_t seg_g[kMaxPlanSeg];
    // A's zones of the tile: RA half-widths of [zf, zl] from alpha_s[alpha_skew], zone
    // offsets of [zf, zl + 1] from azo_s[azo_skew] (copied with the tile)
    uint32_t alpha_skew, azo_skew;
    alignas(16) double alpha_s[kZcMax + 2];     // bulk-copy destinations: 16-byte aligned
    alignas(16) uint32_t azo_s[kZcMax + 8];
    // B's bin index rows of the band (WHOLE plans of at most kBinZones zones)
    alignas(16) uint16_t bins[kBinZones << 5];
    uint32_t bin_log2;
};

template <int TILE, bool RADEC>
constexpr bool stage_aligned()
{
    using S = StageT<TILE, RADEC>;
    return offsetof(S, zoff) % 16 == 0 && offsetof(S, a_id) % 16 == 0 && offsetof(S, a_radec) % 16 == 0 &&
           offsetof(S, a_xyz) % 16 == 0 && offsetof(S, b_xyz) % 16 == 0 && offsetof(S, bins) % 16 == 0;
}
static_assert(stage_aligned<64, false>() && stage_aligned<128, false>() && stage_aligned<256, false>() &&
                  stage_aligned<64, true>() && stage_aligned<128, true>() && stage_aligned<256, true>(),
              "bulk-copy destinations in a stage are 16-byte aligned");

// Register caps: blocks of 256 objects two per SM -- registers are allocated
// per scheduler partition, and 5 of a pair of blocks' 18 warps share one, so 96
// a thread (5 x 96 x 32 <= 16K) -- and of 128 four.
template <int TILE, int VARIANT, bool COUNT_CAND, bool DIST>
__global__ void __launch_bounds__(TILE + 32, TILE <= 128 ? 4 : 2)
pair_kernel(const JobDev *__restrict__ jobs, const TilePlan *__restrict__ plans, uint32_t n_heavy,
            uint32_t n_normal, uint32_t chunk, MatchOut out)
{
    constexpr bool RADEC = VARIANT == 1;
    // A's FP64 ra/dec staged only for the kernels that read them for every
    // candidate (plain FP64, candidate counting, distances)
    constexpr bool A_RADEC = RADEC || COUNT_CAND || DIST;
    using Stage = StageT<TILE, RADEC>;
    constexpr int kStages = Stage::kStages;
    constexpr int C = TILE / 32;   // consumer warps
    extern __shared__ __align__(128) unsigned char smem_raw[];
    Stage *stages = reinterpret_cast<Stage *>(smem_raw);
    using WBuf = WBufT<DIST>;
    WBuf *wbufs = reinterpret_cast<WBuf *>(stages + kStages);
    WList *wl = reinterpret_cast<WList *>(wbufs + C);
    uint64_t *full = reinterpret_cast<uint64_t *>(wl + C);
    uint64_t *empty = full + kStages;

    const int warp = threadIdx.x >> 5;
    const unsigned lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], C);
        }
        fence_mbar_init();
    }
    if (warp >= 1 && lane == 0) wbufs[warp - 1].count = 0;
    __syncthreads();

    if (warp == 0) {
        // ================= producer =================
        // Heavy pieces first, one per claim; then normal tiles, `chunk` (<= 32)
        // per claim, lane k prefetching plan k of the claim; lane 0 issues the
        // copies.  The next claim is requested before the current one is issued.
        int s = 0;
        uint32_t phase = 0;
        bool ok = true;
        // stages whose latest copy may still be landing (bit per stage), and the
        // fill parity each was issued with: a stage's bit is cleared once its
        // consumers have released it, which they do only after its copy landed
        uint32_t pend = 0, pend_par = 0;
        int cached_job = -1;
        const double2 *a_radec = nullptr, *b_radec = nullptr;
        const float4 *a_xyz = nullptr, *b_xyz = nullptr;
        const long long *a_id = nullptr, *b_id = nullptr;
        const uint32_t *b_zoff = nullptr, *a_zoff = nullptr;
        const double *alpha = nullptr;
        const uint16_t *b_bins = nullptr;
        int alpha_z0 = 0, b_bin_log2 = 0;
        // issue plan words w[16] into the next stage
        auto issue = [&](const uint32_t (&w)[16]) -> bool {
            if (!mbar_wait(&empty[s], phase ^ 1u)) return false;
            pend &= ~(1u << s);
            if (lane == 0) {
                const uint32_t a_start = w[0], a_len = w[1], mode = w[2] & 255u, nseg = (w[2] >> 8) & 255u;
                const int zf = (int)w[3];
                const int zl = zf + (int)(w[2] >> 16);
                const int band_lo = (int)w[4];
                const uint32_t job = w[5], b_start = w[6], b_len = w[7];
                if ((int)job != cached_job) {
                    const JobDev &J = jobs[job];
                    a_radec = J.a_radec; a_xyz = J.a_xyz; a_id = J.a_id;
                    b_radec = J.b_radec; b_xyz = J.b_xyz; b_zoff = J.b_zoff; b_id = J.b_id;
                    a_zoff = J.a_zoff; alpha = J.alpha; alpha_z0 = J.alpha_z0;
                    b_bins = J.b_bins; b_bin_log2 = J.b_bin_log2;
                    cached_job = (int)job;
                }
                Stage &S = stages[s];
                S.a_start = a_start;
                S.a_len = a_len;
                S.mode = mode;
                S.nseg = nseg;
                S.band_lo = band_lo;
                S.zf = zf;
                S.zl = zl;
                S.job = job;
                S.b_start = b_start;
                S.b_len = b_len;
                S.done = 0;
                const uint32_t a_even = a_start & ~1u;
                S.id_skew = a_start - a_even;
                const uint32_t id_cnt = (a_start + a_len - a_even + 1) & ~1u;
                uint32_t bytes = a_len * (A_RADEC ? 32u : 16u) + id_cnt * 8u;
                // alpha of [zf, zl] and A offsets of [zf, zl + 1], rounded out to 16-byte copies
                // (alpha tables carry 2 spare entries, zone offsets 8)
                const uint32_t ae = (uint32_t)(zf - alpha_z0), ae_al = ae & ~1u;
                S.alpha_skew = ae - ae_al;
                const uint32_t acnt = (S.alpha_skew + (uint32_t)(zl - zf + 1) + 1u) & ~1u;
                const uint32_t az_al = (uint32_t)zf & ~3u;
                S.azo_skew = (uint32_t)zf - az_al;
                const uint32_t azcnt = (S.azo_skew + (uint32_t)(zl - zf + 2) + 3u) & ~3u;
                bytes += acnt * 8u + azcnt * 4u;
                uint32_t zcopy = 0, z_al = 0;
                constexpr uint32_t kBBytes = RADEC ? 32u : 16u;   // staged bytes per B object
                const bool bins = mode == PLAN_WHOLE && nseg <= (uint32_t)kBinZones && b_bin_log2 > 0;
                S.bin_log2 = bins ? (uint32_t)b_bin_log2 : 0u;
                if (bins) bytes += nseg << (b_bin_log2 + 1);
                if (mode == PLAN_WHOLE) {
                    bytes += b_len * kBBytes;
                    z_al = (uint32_t)band_lo & ~3u;
                    S.zoff_skew = (uint32_t)band_lo - z_al;
                    zcopy = (S.zoff_skew + nseg + 1 + 3) & ~3u;
                    bytes += zcopy * 4u;
                } else if (mode == PLAN_UNION) {
                    bytes += b_len * kBBytes;
                    uint32_t o = 0;
#pragma unroll
                    for (uint32_t q = 0; q < (uint32_t)kMaxPlanSeg; ++q) {
                        if (q < nseg) {
                            S.seg_off[q] = o;
                            S.seg_g[q] = w[8 + q];
                            o += w[12 + q];
                        }
                    }
                    S.seg_off[nseg] = o;
                }
                fence_proxy_async();
                mbar_expect_tx(&full[s], bytes);
                if (A_RADEC) bulk_g2s(S.a_radec, a_radec + a_start, a_len * 16u, &full[s]);
                bulk_g2s(S.a_xyz, a_xyz + a_start, a_len * 16u, &full[s]);
                bulk_g2s(S.a_id, a_id + a_even, id_cnt * 8u, &full[s]);
                bulk_g2s(S.alpha_s, alpha + ae_al, acnt * 8u, &full[s]);
                bulk_g2s(S.azo_s, a_zoff + az_al, azcnt * 4u, &full[s]);
                if (mode == PLAN_WHOLE) {
                    if (b_len) {
                        // the band's B ids into L2: matches read them when a warp's buffer is
                        // flushed (16-byte aligned, whole 16-byte units; ids carry 2 spare entries)
                        const uint32_t i0 = b_start & ~1u, i1 = (b_start + b_len + 1) & ~1u;
                        bulk_prefetch_l2(b_id + i0, (i1 - i0) * 8u);
                        if (RADEC) bulk_g2s(S.b_radec, b_radec + b_start, b_len * 16u, &full[s]);
                        bulk_g2s(S.b_xyz, b_xyz + b_start, b_len * 16u, &full[s]);
                    }
                    bulk_g2s(S.zoff, b_zoff + z_al, zcopy * 4u, &full[s]);
                    if (bins)   // rows of 2^bin_log2 16-bit entries: 16-byte multiples
                        bulk_g2s(S.bins, b_bins + ((size_t)band_lo << b_bin_log2), nseg << (b_bin_log2 + 1),
                                 &full[s]);
                } else if (mode == PLAN_UNION) {
#pragma unroll
                    for (uint32_t q = 0; q < (uint32_t)kMaxPlanSeg; ++q) {
                        const uint32_t ln = w[12 + q];
                        if (q >= nseg || !ln) continue;
                        if (RADEC) bulk_g2s(S.b_radec + S.seg_off[q], b_radec + w[8 + q], ln * 16u, &full[s]);
                        bulk_g2s(S.b_xyz + S.seg_off[q], b_xyz + w[8 + q], ln * 16u, &full[s]);
                    }
                }
            }
            __syncwarp();
            pend |= 1u << s;
            pend_par = (pend_par & ~(1u << s)) | (phase << s);
            if (++s == kStages) {
                s = 0;
                phase ^= 1u;
            }
            return true;
        };
        // ---- heavy queue ----
        while (ok) {
            uint32_t h = 0;
            if (lane == 0) h = (uint32_t)atomicAdd(&out.counters[6], 1ull);
            h = __shfl_sync(0xffffffffu, h, 0);
            if (h >= n_heavy) break;
            uint4 pw[4];
            const uint4 *src = reinterpret_cast<const uint4 *>(plans + h);
            pw[0] = src[0]; pw[1] = src[1]; pw[2] = src[2]; pw[3] = src[3];
            uint32_t w[16] = {pw[0].x, pw[0].y, pw[0].z, pw[0].w, pw[1].x, pw[1].y, pw[1].z, pw[1].w,
                              pw[2].x, pw[2].y, pw[2].z, pw[2].w, pw[3].x, pw[3].y, pw[3].z, pw[3].w};
            ok = issue(w);
        }
        // ---- normal queue ----
        const TilePlan *nplans = plans + n_heavy;
        const uint32_t ch = min(chunk, 32u);
        uint32_t t0 = 0;
        if (lane == 0) t0 = (uint32_t)atomicAdd(&out.counters[1], (unsigned long long)ch);
        t0 = __shfl_sync(0xffffffffu, t0, 0);
        while (ok && t0 < n_normal) {
            const uint32_t nt = min(ch, n_normal - t0);
            uint4 pw[4];
            if (lane < nt) {
                const uint4 *src = reinterpret_cast<const uint4 *>(nplans + t0 + lane);
                pw[0] = src[0]; pw[1] = src[1]; pw[2] = src[2]; pw[3] = src[3];
            }
            uint32_t t_next = 0;
            if (lane == 0) t_next = (uint32_t)atomicAdd(&out.counters[1], (unsigned long long)ch);
            for (uint32_t k = 0; k < nt && ok; ++k) {
                uint32_t w[16];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    w[4 * q + 0] = __shfl_sync(0xffffffffu, pw[q].x, k);
                    w[4 * q + 1] = __shfl_sync(0xffffffffu, pw[q].y, k);
                    w[4 * q + 2] = __shfl_sync(0xffffffffu, pw[q].z, k);
                    w[4 * q + 3] = __shfl_sync(0xffffffffu, pw[q].w, k);
                }
                ok = issue(w);
            }
            t0 = __shfl_sync(0xffffffffu, t_next, 0);
        }
        // end of work: a "done" stage for the consumers
        if (ok && mbar_wait(&empty[s], phase ^ 1u)) {
            if (lane == 0) {
                stages[s].done = 1;
                mbar_expect_tx(&full[s], 0);
            }
            __syncwarp();
        } else {
            if (lane == 0) atomicExch(&out.counters[7], 1ull);
            // wait (bounded) for the copies that may still be landing in the
            // stages, each on the parity it was issued with, before leaving
            for (int q = 0; q < kStages; ++q)
                if (pend & (1u << q)) mbar_wait(&full[q], (pend_par >> q) & 1u);
        }
        return;
    }

    // ================= consumers =================
    WBuf &wb = wbufs[warp - 1];
    Counters cn = {0ull, 0ull, 0ull, 0ull};
    int cur_job = -1;
    const JobDev *Jp = jobs;
    JobScalars K = {};
    int s = 0;
    uint32_t phase = 0;
    for (;;) {
        if (!mbar_wait(&full[s], phase)) {
            if (lane == 0) atomicExch(&out.counters[7], 1ull);
            break;
        }
        Stage &S = stages[s];
        if (S.done) break;
        const uint32_t t = (uint32_t)(warp - 1) * 32u + lane;
        if ((int)S.job != cur_job) {   // job scalars stay in registers while the job does not change
            cur_job = (int)S.job;
            Jp = &jobs[cur_job];
            K = load_scalars(*Jp);
        }
        const IdSrc ids = {jobs, Jp, cur_job};
        const JobDev &J = *Jp;
        if (S.mode == PLAN_GLOBAL) {
            // band too large to stage: per-lane cursor over global memory
            if (t < S.a_len) {
                AObj a;
                const float4 fa = S.a_xyz[t];
                const double2 ra = A_RADEC ? S.a_radec[t] : __ldg(&J.a_radec[S.a_start + t]);
                a.ra = ra.x;
                a.dec = ra.y;
                a.fx = fa.x; a.fy = fa.y; a.fz = fa.z;
                a.zone = a_zone_s(S, S.a_start + t);
                if (a.zone < 0) {   // offsets disagree: never for a consistent segment
                    atomicExch(&out.counters[7], 1ull);
                    a.zone = 0;
                    a.alpha = -1.0;   // empty windows, no candidates
                } else {
                    a.alpha = S.alpha_s[S.alpha_skew + (a.zone - S.zf)];
                }
                a.full_ring = a.alpha >= 3.0;
                a.id = S.a_id[S.id_skew + t];
                a.gi = S.a_start + t;
                BView V;
                V.staged = false;
                V.whole = false;
                V.xyz = J.b_xyz;
                V.zoff = J.b_zoff;
                V.band_lo = 0;
                V.bins = J.b_bins;
                V.bin_log2 = J.b_bin_log2;
                test_object<VARIANT, COUNT_CAND, DIST>(J, a, V, wb, out, ids, S.job, cn);
            }
        } else {
            BView V;
            V.staged = true;
            V.whole = S.mode == PLAN_WHOLE;
            V.band_lo = S.band_lo;
            V.xyz = S.b_xyz;
            V.zoff = S.zoff + S.zoff_skew;
            V.base = S.b_start;
            V.len = S.b_len;
            V.off = S.seg_off;
            V.g = S.seg_g;
            V.bins = S.bins;
            V.bin_log2 = (int)S.bin_log2;
            // ---- phase 1: each lane's candidate ranges ----
            WList &L = wl[warp - 1];
            int n = 0, nr = 0, za = 0;
            double alpha = 0;
            if (t < S.a_len) {
                za = a_zone_s(S, S.a_start + t);
                if (za < 0) {
                    atomicExch(&out.counters[7], 1ull);
                    za = 0;
                    alpha = -1.0;
                } else {
                    alpha = S.alpha_s[S.alpha_skew + (za - S.zf)];
                }
                const Win wn = make_win_q(__float_as_uint(S.a_xyz[t].w), alpha);
                n = lane_ranges(V, K, wn, alpha >= 3.0, za, L.r[lane], nr);
            }
            L.alpha[lane] = alpha;
            const bool overflow = __any_sync(0xffffffffu, n < 0);
            if (overflow) {
                // a lane has more windows than the list holds (nz > 1): cursor path for this warp
                if (t < S.a_len) {
                    AObj a;
                    const float4 fa = S.a_xyz[t];
                    const double2 rd = A_RADEC ? S.a_radec[t] : __ldg(&J.a_radec[S.a_start + t]);
                    a.ra = rd.x;
                    a.dec = rd.y;
                    a.fx = fa.x; a.fy = fa.y; a.fz = fa.z;
                    a.zone = za;
                    a.alpha = alpha;
                    a.full_ring = alpha >= 3.0;
                    a.id = S.a_id[S.id_skew + t];
                    a.gi = S.a_start + t;
                        test_object<VARIANT, COUNT_CAND, DIST>(J, a, V, wb, out, ids, S.job, cn);
                }
            } else {
                // inclusive scan of candidate counts across the warp
                uint32_t incl = (uint32_t)n;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= (unsigned)o) incl += y;
                }
                const uint32_t start = incl - (uint32_t)n;
                const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
                // ---- phase 2: the warp walks the flattened candidate list ----
                for (uint32_t c0 = 0; c0 < total; c0 += 32) {
                    const uint32_t c = c0 + lane;
                    // owner of candidate c: the last lane with candidates that start at or
                    // before c -- the lane covering c0 (ballot), or a later lane whose start
                    // mark lies in (c0, c], found by a max-scan over the marks
                    const unsigned before = __ballot_sync(0xffffffffu, n > 0 && start <= c0);
                    L.mark[lane] = 0;
                    __syncwarp();
                    if (n > 0 && start > c0 && start < c0 + 32) L.mark[start - c0] = lane + 1;
                    __syncwarp();
                    int own = (int)L.mark[lane] - 1;
                    if (own < 0) own = before ? 31 - __clz(before) : 0;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, own, o);
                        if (lane >= (unsigned)o) own = max(own, y);
                    }
                    const uint32_t own_start = __shfl_sync(0xffffffffu, start, own);
                    bool m = false;
                    long long ida = 0;
                    uint32_t gq = 0xFFFFFFFFu;   // global index of the candidate, once needed
                    double dist = 0;
                    if (c < total) {
                        const int owner = own;
                        uint32_t k = c - own_start;
                        int r = 0;
                        uint32_t rr = L.r[owner][0];
                        while (k >= (rr >> 16)) {
                            k -= rr >> 16;
                            rr = L.r[owner][++r];
                        }
                        const uint32_t q = (rr & 0xFFFFu) + k;
                        const uint32_t ta = (warp - 1) * 32u + (uint32_t)owner;
                        cn.tested++;
                        // A's FP64 ra/dec: staged for the kernels that cut or measure every
                        // pair, else read for the few pairs that need them
                        double2 ra = make_double2(0.0, 0.0);
                        if (A_RADEC) ra = S.a_radec[ta];
                        const double al = L.alpha[owner];
                        double c2 = 0;
                        if (VARIANT == 0) {
                            const float4 fa = S.a_xyz[ta];
                            const float4 fb = S.b_xyz[q];
                            const float dx = fa.x - fb.x, dy = fa.y - fb.y, dz = fa.z - fb.z;
                            const float c32 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                            if (COUNT_CAND) {
                                gq = staged_global(V, (int)S.nseg, q);
                                cn.cand += cuts_k(J.sr_rad, ra.x, ra.y, al, __ldg(&J.b_radec[gq])) ? 1ull : 0ull;
                            }
                            if (!(c32 > K.thr_hi)) {
                                // below thr_lo the FP64 chord is under the threshold and, in a zone
                                // with an RA cut (alpha < 3), the dec and RA cuts hold (bounds in
                                // xm_make_params): B's ra/dec is read and the FP64 vectors are
                                // computed only inside the band, or for the distance
                                const bool band = c32 >= K.thr_lo;
                                cn.border += band ? 1ull : 0ull;
                                bool pass = true;
                                const bool cut = band || al >= 3.0;
                                double2 rb = make_double2(0.0, 0.0);
                                if (cut || DIST) {
                                    if (gq == 0xFFFFFFFFu) gq = staged_global(V, (int)S.nseg, q);
                                    rb = __ldg(&J.b_radec[gq]);
                                }
                                if (cut) {
                                    if (!A_RADEC) ra = __ldg(&J.a_radec[S.a_start + ta]);
                                    pass = cuts_k(J.sr_rad, ra.x, ra.y, al, rb);
                                }
                                if (pass) {
                                    m = true;
                                    if (band || DIST) {
                                        // FP64 unit vectors of both ends, as the zone builder
                                        // computes them (the same bits), then the chord
                                        c2 = chord2_radec<DIST>(ra.x, ra.y, rb.x, rb.y);
                                        if (band) {
                                            cn.exact++;
                                            m = c2 < J.sr_dist2;
                                        }
                                    }
                                }
                            }
                        } else {
                            const double2 rb = S.b_radec[q];
                            if (cuts_k(K.sr_rad, ra.x, ra.y, al, rb)) {
                                cn.cand++;
                                cn.exact++;
                                double x1, y1, z1, x2, y2, z2;
                                radec2xyz(ra.x, ra.y, x1, y1, z1);
                                radec2xyz(rb.x, rb.y, x2, y2, z2);
                                c2 = chord2(x1, y1, z1, x2, y2, z2);
                                m = c2 < K.sr_dist2;
                            }
                        }
                        if (m) {
                            if (gq == 0xFFFFFFFFu) gq = staged_global(V, (int)S.nseg, q);
                            ida = S.a_id[S.id_skew + ta];
                            if (DIST) dist = 2.0 * asin(sqrt(c2) * 0.5);
                        }
                    }
                    emit_w<DIST>(wb, out, ids, m, ida, gq, dist, S.job);
                    __syncwarp();
                    if (wb.count >= 32u) out_flush<DIST>(wb, out, ids);
                }
            }
        }
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&empty[s])) : "memory");
        if (wb.count >= 32u) out_flush<DIST>(wb, out, ids);
        if (++s == kStages) {
            s = 0;
            phase ^= 1u;
        }
    }
    const IdSrc ids = {jobs, Jp, cur_job};
    while (min(wb.count, (uint32_t)kWarpBuf) > 0) out_flush<DIST>(wb, out, ids);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cn.tested += __shfl_down_sync(0xffffffffu, cn.tested, o);
        cn.cand += __shfl_down_sync(0xffffffffu, cn.cand, o);
        cn.border += __shfl_down_sync(0xffffffffu, cn.border, o);
        cn.exact += __shfl_down_sync(0xffffffffu, cn.exact, o);
    }
    if (lane == 0) {
        atomicAdd(&out.counters[2], cn.tested);
        atomicAdd(&out.counters[3], cn.cand);
        atomicAdd(&out.counters[4], cn.border);
        atomicAdd(&out.counters[5], cn.exact);
    }
}

template <int TILE, bool RADEC, bool DIST>
constexpr size_t smem_bytes()
{
    using Stage = StageT<TILE, RADEC>;
    return Stage::kStages * sizeof(Stage) + (TILE / 32) * (sizeof(WBufT<DIST>) + sizeof(WList)) +
           2 * Stage::kStages * sizeof(uint64_t);
}

// Blocks of 256 objects run two per SM, blocks of 128 of the kernels without
// distances four (228 KB of shared memory per SM, 1 KB of it reserved per block).
static_assert(2 * (smem_bytes<256, true, true>() + 1024) <= 228 * 1024 &&
                  2 * (smem_bytes<256, false, true>() + 1024) <= 228 * 1024 &&
                  4 * (smem_bytes<128, false, false>() + 1024) <= 228 * 1024,
              "pair-kernel blocks per SM");

template <int TILE, int VARIANT, bool CC, bool DIST>
cudaError_t launch_t(const LaunchCfg &L, const JobDev *jobs, const TilePlan *plans, uint32_t n_heavy,
                     uint32_t n_normal, const MatchOut &out, cudaStream_t st)
{
    auto k = pair_kernel<TILE, VARIANT, CC, DIST>;
    const size_t smem = smem_bytes<TILE, VARIANT == 1, DIST>();
    static bool attr = false;   // per instantiation
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    int per_sm = L.blocks_per_sm;
    if (per_sm <= 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TILE + 32, smem);
        if (per_sm < 1) per_sm = 1;
    }
    const uint64_t want = (uint64_t)n_heavy + ((uint64_t)n_normal + L.chunk - 1) / L.chunk;
    unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)L.sm_count * per_sm, std::max<uint64_t>(want, 1));
    k<<<grid, TILE + 32, smem, st>>>(jobs, plans, n_heavy, n_normal, L.chunk, out);
    return cudaGetLastError();
}

template <int TILE>
cudaError_t launch_tile(const LaunchCfg &L, const JobDev *jobs, const TilePlan *plans, uint32_t n_heavy,
                        uint32_t n_normal, const MatchOut &out, cudaStream_t st)
{
    if (L.variant == 1)
        return L.dist ? launch_t<TILE, 1, true, true>(L, jobs, plans, n_heavy, n_normal, out, st)
                      : launch_t<TILE, 1, true, false>(L, jobs, plans, n_heavy, n_normal, out, st);
    if (L.count_cand)
        return L.dist ? launch_t<TILE, 0, true, true>(L, jobs, plans, n_heavy, n_normal, out, st)
                      : launch_t<TILE, 0, true, false>(L, jobs, plans, n_heavy, n_normal, out, st);
    return L.dist ? launch_t<TILE, 0, false, true>(L, jobs, plans, n_heavy, n_normal, out, st)
                  : launch_t<TILE, 0, false, false>(L, jobs, plans, n_heavy, n_normal, out, st);
}

}  // namespace

size_t plan_bytes(uint64_t n_plans) { return (size_t)n_plans * sizeof(TilePlan); }

cudaError_t plan_count(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_items, uint32_t *cnt,
                       uint32_t *off, void *scan_tmp, cudaStream_t st)
{
    const unsigned g = (n_items + 127) / 128;
    tiles_count<<<g, 128, 0, st>>>(jobs, n_jobs, n_items, L.zc, (uint32_t)L.tile, 4u * (uint32_t)L.tile, cnt);
    cudaError_t e = xm_scan_exclusive_u32(cnt, off, n_items, scan_tmp, st);
    if (e != cudaSuccess) return e;
    return xm_scan_exclusive_u32(cnt + n_items, off + n_items + 1, n_items, scan_tmp, st);
}

cudaError_t plan_make(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_items, const uint32_t *off,
                      uint32_t n_normal, uint32_t n_heavy, void *plans, unsigned long long *err, cudaStream_t st)
{
    const unsigned g = (n_items + kMakeWarps - 1) / kMakeWarps;
    tiles_make<<<g, 32 * kMakeWarps, 0, st>>>(jobs, n_jobs, n_items, L.zc, (uint32_t)L.tile, 4u * (uint32_t)L.tile, off,
                                  off + n_items + 1, (TilePlan *)plans, n_normal + n_heavy, err);
    return cudaGetLastError();
}

cudaError_t run_pairs(const LaunchCfg &L, const JobDev *jobs, const void *plans, uint32_t n_normal, uint32_t n_heavy,
                      const MatchOut &out, cudaStream_t st)
{
    const TilePlan *p = (const TilePlan *)plans;
    switch (L.tile) {
    case 64: return launch_tile<64>(L, jobs, p, n_heavy, n_normal, out, st);
    case 256: return launch_tile<256>(L, jobs, p, n_heavy, n_normal, out, st);
    default: return launch_tile<128>(L, jobs, p, n_heavy, n_normal, out, st);
    }
}

}  // namespace xm
