// xm_match.cu -- zone-pair window search + pair test + compaction, as one
// persistent work-stealing launch.
//
// Replaces the reference's per-zone-pair launches (Worker.cu:330-366) of the
// all-pairs kernel xmatch_kernel (Worker.cu:65-241).
//
// Work decomposition.  A work item is `zc` consecutive zones of one job's A
// segment; blocks claim `chunk` items at a time from a global counter.  A
// block cuts its zones into tiles of at most TILE objects (one per thread):
// a zone holding more than TILE/2 objects is split into near-equal
// single-zone tiles, consecutive smaller zones are packed into one tile.
//
// Staging.  For a tile, the B zones within nz of its zones (Worker.cu:
// 338-341) are copied into shared memory with bulk asynchronous copies
// (cp.async.bulk, completion on an mbarrier):
//   * single-zone tile: per B zone only the union of the tile's RA windows,
//     i.e. objects with ra in [ra_first - alpha, ra_last + alpha] (A is
//     ra-sorted), unless an RA-wraparound window could be non-empty or alpha
//     is the "no cut" sentinel, in which case the whole zone;
//   * packed tile: the whole B zones.
// Tiles whose staged set exceeds the buffer fall back to bisecting B in
// global memory.
//
// Pair test.  Every thread bisects its own windows (direct, and the two
// wrapped ones for the RA branches of Worker.cu:89,98,110) in the staged ra
// values and tests each candidate with the reference predicate (Worker.cu:
// 88-97): dec cut, RA cut, chord^2 < (2 sin(r/2))^2, all FP64 with the unit
// vectors of the unshifted (ra, dec) -- the branch-3 sign error of
// Worker.cu:118 fixed.  XM_FILTER32 first evaluates chord^2 in FP32 from the
// stored FP32 unit vectors and discards a pair only when that value exceeds a
// bound proven to imply chord^2_FP64 >= threshold; every other pair is
// decided by the FP64 predicate, so the pair set is the FP64 one bit for bit.
//
// Output.  Matches are compacted per warp with __ballot_sync/__popc into a
// block buffer in shared memory that is appended to global memory with one
// atomicAdd per flush (Worker.cu:128-240 uses two Hillis-Steele scans per
// block).  A full output buffer is detected and reported, never silently
// truncated (Worker.cu:147-148).
#include <algorithm>
#include <cmath>
#include <vector>

#include "xm_internal.h"
#include "xm_match.cuh"
#include "xm_math.cuh"

namespace xm {

namespace {

constexpr int kSbuf = 256;         // block output staging records
constexpr int kStageCap = 1024;    // B objects staged per tile
constexpr int kMaxSeg = 96;        // B zones per tile band
constexpr double kWinEps = 1e-12;  // window widening (radians), >> FP64 rounding of ra +- alpha
constexpr unsigned kWaitLimit = 1u << 26;   // bounded mbarrier wait (iterations)

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// ---- mbarrier + bulk copy (TMA, no multicast) ----
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return done != 0;
}

// Bounded wait for the phase; false if it did not complete within the limit.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t phase)
{
    for (unsigned it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// ---- ra bisection ----
// first k in [lo, hi) with ra[k] >= v   (global memory)
__device__ __forceinline__ uint32_t lower_ra_g(const double2 *__restrict__ radec, uint32_t lo, uint32_t hi, double v)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&radec[mid].x) < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}
// first k in [lo, hi) with ra[k] > v    (global memory)
__device__ __forceinline__ uint32_t upper_ra_g(const double2 *__restrict__ radec, uint32_t lo, uint32_t hi, double v)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&radec[mid].x) <= v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// A source (a thread's object).
struct AObj {
    double ra, dec;
    double x, y, z;     // FP64 unit vector (computed on first use)
    float fx, fy, fz;
    double alpha;
    long long id;
    int zone;
    bool full_ring;     // alpha >= 3: every object of a zone is a candidate
    bool have_xyz;
};

// View of B for window enumeration: either the staged copy in shared
// memory (segments per band zone) or the segment in global memory.
struct BView {
    const double2 *radec;   // staged or global
    const float4 *xyz;
    bool staged;
    // staged: band zone k -> [off[k], off[k+1]) in shared memory, global index g[k] + (q - off[k])
    const uint32_t *off;
    const uint32_t *g;
    int band_lo;
    // global
    const uint32_t *zoff;
};

// Candidate enumeration state: B zones of the band, and in each zone up to
// three ra windows (direct, branch 2 with B near 0, branch 3 with B near 2 pi).
struct Cursor {
    int zb, zb_end;
    int win;                // 0 direct, 1 branch 2, 2 branch 3
    uint32_t j, j_end;      // candidate positions (view indices) of the current window
    uint32_t b0, b1;        // current zone range (view indices)
    double hi_cur;
    uint32_t w1_lo, w1_hi;  // direct window (keeps the wrapped ones disjoint from it)
};

__device__ __forceinline__ uint32_t lower_v(const BView &V, uint32_t lo, uint32_t hi, double v)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (V.radec[mid].x < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void open_window(const BView &V, const AObj &a, Cursor &c)
{
    c.j = c.j_end = 0;
    if (a.full_ring) {
        if (c.win != 0) return;
        c.j = c.b0;
        c.j_end = c.b1;
        c.hi_cur = INFINITY;
        return;
    }
    const double lo = a.ra - a.alpha - kWinEps, hi = a.ra + a.alpha + kWinEps;
    if (c.win == 0) {
        c.j = lower_v(V, c.b0, c.b1, lo);
        c.j_end = c.b1;
        c.hi_cur = hi;
        c.w1_lo = c.j;
        c.w1_hi = c.j;
        return;
    }
    if (c.win == 1) {   // branch 2: ra_b in (ra_a - 2pi - alpha, ra_a - 2pi + alpha)
        const double hi2 = hi - XM_TWO_PI + kWinEps;
        if (hi2 < V.radec[c.b0].x) return;
        c.j = lower_v(V, c.b0, c.b1, lo - XM_TWO_PI - kWinEps);
        c.j_end = c.w1_lo;
        c.hi_cur = hi2;
        return;
    }
    // branch 3: ra_b in (ra_a + 2pi - alpha, ra_a + 2pi + alpha)
    const double lo3 = lo + XM_TWO_PI - kWinEps;
    if (lo3 > V.radec[c.b1 - 1].x) return;
    const uint32_t s = lower_v(V, c.b0, c.b1, lo3);
    c.j = s > c.w1_hi ? s : c.w1_hi;
    c.j_end = c.b1;
    c.hi_cur = hi + XM_TWO_PI + kWinEps;
}

__device__ __forceinline__ bool next_candidate(const BView &V, const AObj &a, Cursor &c, uint32_t &out)
{
    for (;;) {
        if (c.j < c.j_end) {
            const uint32_t j = c.j;
            if (V.radec[j].x <= c.hi_cur) {
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
        if (V.staged) {
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

struct SBuf {
    longlong2 ab[kSbuf];
    double d[kSbuf];
    uint32_t job[kSbuf];
    uint32_t count;
    unsigned long long gbase;
};

// Warp-aggregated append of this iteration's matches to the block buffer.
__device__ __forceinline__ void emit(SBuf &sb, const MatchOut &out, bool m, long long ida, long long idb,
                                     double dist, uint32_t job)
{
    const unsigned act = __activemask();
    const unsigned bal = __ballot_sync(act, m);
    if (!m) return;
    const int leader = __ffs(bal) - 1;
    const unsigned lane = threadIdx.x & 31;
    const uint32_t n = (uint32_t)__popc(bal);
    const uint32_t rank = (uint32_t)__popc(bal & lanemask_lt());
    uint32_t base = 0;
    if ((int)lane == leader) base = atomicAdd(&sb.count, n);
    base = __shfl_sync(bal, base, leader);
    const uint32_t slot = base + rank;
    if (slot < (uint32_t)kSbuf) {
        sb.ab[slot] = make_longlong2(ida, idb);
        sb.d[slot] = dist;
        sb.job[slot] = job;
    }
    if (base + n <= (uint32_t)kSbuf) return;
    // block buffer full: the lanes past its end append straight to global memory
    const uint32_t keep = base >= (uint32_t)kSbuf ? 0u : (uint32_t)kSbuf - base;
    unsigned over = bal;
    for (uint32_t q = 0; q < keep; ++q) over &= over - 1;
    if (slot < (uint32_t)kSbuf) return;
    const int l2 = __ffs(over) - 1;
    unsigned long long g = 0;
    if ((int)lane == l2) g = atomicAdd(&out.counters[0], (unsigned long long)__popc(over));
    g = __shfl_sync(over, g, l2);
    g += (unsigned long long)__popc(over & lanemask_lt());
    if (g < out.cap) {
        reinterpret_cast<longlong2 *>(out.pairs)[g] = make_longlong2(ida, idb);
        if (out.dist) out.dist[g] = dist;
        if (out.job) out.job[g] = job;
    }
}

__device__ __forceinline__ void flush(SBuf &sb, const MatchOut &out)
{
    __syncthreads();
    const uint32_t n = sb.count < (uint32_t)kSbuf ? sb.count : (uint32_t)kSbuf;
    if (threadIdx.x == 0) sb.gbase = n ? atomicAdd(&out.counters[0], (unsigned long long)n) : 0ull;
    __syncthreads();
    const unsigned long long g = sb.gbase;
    for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) {
        if (g + k < out.cap) {
            reinterpret_cast<longlong2 *>(out.pairs)[g + k] = sb.ab[k];
            if (out.dist) out.dist[g + k] = sb.d[k];
            if (out.job) out.job[g + k] = sb.job[k];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) sb.count = 0;
    __syncthreads();
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

// All candidates of one A object against the view; emits matches.
template <int VARIANT, bool COUNT_CAND, bool DIST>
__device__ __forceinline__ void test_object(const JobDev &J, AObj &a, const BView &V, SBuf &sb, const MatchOut &out,
                                            uint32_t jx, Counters &cn)
{
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
        const double2 rb = V.radec[q];
        if (VARIANT == 0) {   // FP32 reject, FP64 decision
            if (COUNT_CAND) cn.cand += cuts_pass(J, a, rb) ? 1ull : 0ull;
            const float4 fb = V.xyz[q];
            const float dx = a.fx - fb.x, dy = a.fy - fb.y, dz = a.fz - fb.z;
            const float c32 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
            if (!(c32 > J.thr_hi)) {
                cn.border += (c32 >= J.thr_lo) ? 1ull : 0ull;
                cn.exact++;
                if (cuts_pass(J, a, rb)) {
                    if (!a.have_xyz) {
                        radec2xyz(a.ra, a.dec, a.x, a.y, a.z);
                        a.have_xyz = true;
                    }
                    double x2, y2, z2;
                    radec2xyz(rb.x, rb.y, x2, y2, z2);
                    c2 = chord2(a.x, a.y, a.z, x2, y2, z2);
                    m = c2 < J.sr_dist2;
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
        long long idb = 0;
        double dist = 0;
        if (m) {
            idb = __ldg(&J.b_id[global_index(V, c.zb, q)]);
            if (DIST) dist = 2.0 * asin(sqrt(c2) * 0.5);
        }
        emit(sb, out, m, a.id, idb, dist, jx);
    }
}

struct Stage {
    double2 radec[kStageCap];
    float4 xyz[kStageCap];
    uint32_t off[kMaxSeg + 1];
    uint32_t g[kMaxSeg];
    uint32_t src[kMaxSeg];
    uint64_t bar;
    // tile descriptor (written by thread 0)
    uint32_t t_start, t_len;
    int t_zf, t_zl;
    int mode;               // 0 staged, 1 global fallback
    int band_lo, nseg;
    uint32_t total;
    double ra_first, ra_last;
    // tile formation state
    int z;                  // current zone
    uint32_t pos;           // current A index
    uint32_t item, item_end;
    int z1;                 // end zone of the item
    int jx;
    int error;
};

template <int TILE, int VARIANT, bool COUNT_CAND, bool DIST>
__global__ void __launch_bounds__(TILE)
pair_kernel(const JobDev *__restrict__ jobs, int n_jobs, uint32_t n_items, uint32_t zc, uint32_t chunk, MatchOut out)
{
    __shared__ SBuf sb;
    __shared__ __align__(128) Stage st;
    const int tid = threadIdx.x;
    const unsigned lane = tid & 31;
    if (tid == 0) {
        sb.count = 0;
        st.error = 0;
        mbar_init(&st.bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    Counters cn = {0ull, 0ull, 0ull, 0ull};
    bool failed = false;

    for (;;) {
        // ---- claim `chunk` work items ----
        if (tid == 0) {
            const uint32_t i0 = (uint32_t)atomicAdd(&out.counters[1], (unsigned long long)chunk);
            st.item = i0;
            st.item_end = min(i0 + chunk, n_items);
            st.jx = -1;
        }
        __syncthreads();
        if (st.item >= n_items) break;
        // ---- tiles of the claimed items ----
        for (;;) {
            if (tid == 0) {
                // next tile: advance (item, zone, pos)
                st.t_len = 0;
                while (st.item < st.item_end) {
                    if (st.jx < 0) {
                        const int jx = n_jobs > 1 ? find_job(jobs, n_jobs, st.item) : 0;
                        const JobDev &Jt = jobs[jx];
                        st.jx = jx;
                        st.z = Jt.z_lo + (int)((st.item - Jt.item_begin) * zc);
                        st.z1 = min(st.z + (int)zc, Jt.z_hi + 1);
                        st.pos = __ldg(&Jt.a_zoff[st.z]);
                    }
                    const JobDev &Jt = jobs[st.jx];
                    const uint32_t *zo = Jt.a_zoff;
                    int z = st.z;
                    uint32_t pos = st.pos;
                    while (z < st.z1 && pos >= __ldg(&zo[z + 1])) {
                        ++z;
                        pos = max(pos, __ldg(&zo[z]));
                    }
                    if (z >= st.z1) {   // item done
                        st.item++;
                        st.jx = -1;
                        continue;
                    }
                    const uint32_t zb0 = __ldg(&zo[z]), zb1 = __ldg(&zo[z + 1]);
                    const uint32_t cnt = zb1 - zb0;
                    if (cnt > (uint32_t)(TILE / 2)) {   // large zone: near-equal single-zone tiles
                        const uint32_t k = (cnt + TILE - 1) / TILE;
                        const uint32_t size = (cnt + k - 1) / k;
                        const uint32_t len = min(size, zb1 - pos);
                        st.t_start = pos;
                        st.t_len = len;
                        st.t_zf = st.t_zl = z;
                        st.pos = pos + len;
                        st.z = z;
                    } else {                          // pack small zones
                        const uint32_t start = pos;
                        uint32_t end = zb1;
                        int zl = z, zn = z + 1;
                        while (zn < st.z1) {
                            const uint32_t e1 = __ldg(&zo[zn + 1]);
                            const uint32_t c1 = e1 - __ldg(&zo[zn]);
                            if (c1 > (uint32_t)(TILE / 2) || e1 - start > (uint32_t)TILE) break;
                            if (c1 > 0) {
                                zl = zn;
                                end = e1;
                            }
                            ++zn;
                        }
                        st.t_start = start;
                        st.t_len = end - start;
                        st.t_zf = z;
                        st.t_zl = zl;
                        st.pos = end;
                        st.z = zn;
                    }
                    break;
                }
            }
            __syncthreads();
            if (st.t_len == 0) break;   // claimed items exhausted
            const JobDev &J = jobs[st.jx];
            const uint32_t t_start = st.t_start, t_len = st.t_len;
            const int zf = st.t_zf, zl = st.t_zl;
            // ---- this thread's A object ----
            AObj a;
            const bool active = (uint32_t)tid < t_len;
            if (active) {
                const uint32_t i = t_start + tid;
                const float4 fa = __ldg(&J.a_xyz[i]);
                const double2 ra = __ldg(&J.a_radec[i]);
                a.ra = ra.x;
                a.dec = ra.y;
                a.fx = fa.x; a.fy = fa.y; a.fz = fa.z;
                a.zone = (int)__float_as_uint(fa.w);
                a.alpha = __ldg(&J.alpha[a.zone]);
                a.full_ring = a.alpha >= 3.0;
                a.id = __ldg(&J.a_id[i]);
                a.have_xyz = false;
                if (tid == 0) st.ra_first = a.ra;
                if ((uint32_t)tid == t_len - 1) st.ra_last = a.ra;
            }
            __syncthreads();
            // ---- staging plan: warp 0 ----
            if (tid < 32) {
                const int band_lo = max(0, zf - J.nz), band_hi = min(J.n_zones - 1, zl + J.nz);
                const int nseg = band_hi - band_lo + 1;
                int mode = nseg > kMaxSeg ? 1 : 0;
                if (mode == 0) {
                    const bool single = zf == zl;
                    const double alpha = __ldg(&J.alpha[zf]);
                    const double ra_f = st.ra_first, ra_l = st.ra_last;
                    uint32_t carry = 0;
                    for (int k0 = 0; k0 < nseg; k0 += 32) {
                        const int k = k0 + (int)lane;
                        uint32_t s = 0, len = 0;
                        if (k < nseg) {
                            const int zb = band_lo + k;
                            const uint32_t b0 = __ldg(&J.b_zoff[zb]), b1 = __ldg(&J.b_zoff[zb + 1]);
                            s = b0;
                            len = b1 - b0;
                            if (len > 0 && single && alpha < 3.0) {
                                const double bmin = __ldg(&J.b_radec[b0].x), bmax = __ldg(&J.b_radec[b1 - 1].x);
                                const bool wrap = !((ra_l + alpha + 2 * kWinEps - XM_TWO_PI < bmin) &&
                                                    (ra_f - alpha - 2 * kWinEps + XM_TWO_PI > bmax));
                                if (!wrap) {
                                    s = lower_ra_g(J.b_radec, b0, b1, ra_f - alpha - kWinEps);
                                    const uint32_t e = upper_ra_g(J.b_radec, s, b1, ra_l + alpha + kWinEps);
                                    len = e - s;
                                }
                            }
                        }
                        // exclusive scan of len across the warp
                        uint32_t x = len;
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) {
                            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                            if (lane >= (unsigned)o) x += y;
                        }
                        if (k < nseg) {
                            st.off[k] = carry + x - len;
                            st.g[k] = s;
                        }
                        carry += __shfl_sync(0xffffffffu, x, 31);
                    }
                    if (lane == 0) {
                        st.off[nseg] = carry;
                        st.total = carry;
                        if (carry > (uint32_t)kStageCap) mode = 1;
                    }
                }
                if (lane == 0) {
                    st.mode = mode;
                    st.band_lo = band_lo;
                    st.nseg = nseg;
                }
            }
            __syncthreads();
            const int mode = st.mode;
            if (mode == 0 && st.total > 0) {
                // ---- bulk copies of the staged windows ----
                if (tid == 0) {
                    fence_proxy_async();
                    mbar_expect_tx(&st.bar, st.total * (uint32_t)(sizeof(double2) + sizeof(float4)));
                    for (int k = 0; k < st.nseg; ++k) {
                        const uint32_t o = st.off[k], len = st.off[k + 1] - o;
                        if (len == 0) continue;
                        bulk_g2s(&st.radec[o], J.b_radec + st.g[k], len * (uint32_t)sizeof(double2), &st.bar);
                        bulk_g2s(&st.xyz[o], J.b_xyz + st.g[k], len * (uint32_t)sizeof(float4), &st.bar);
                    }
                }
                const bool ok = mbar_wait(&st.bar, phase);
                phase ^= 1u;
                if (__syncthreads_or(!ok)) {
                    // copies did not land in time: report, wait once more for them, stop
                    if (tid == 0) {
                        atomicExch((unsigned long long *)&out.counters[7], 1ull);
                        mbar_wait(&st.bar, phase ^ 1u);
                    }
                    __syncthreads();
                    failed = true;
                    break;
                }
            }
            if (active) {
                BView V;
                V.staged = mode == 0;
                if (V.staged) {
                    V.radec = st.radec;
                    V.xyz = st.xyz;
                    V.off = st.off;
                    V.g = st.g;
                    V.band_lo = st.band_lo;
                } else {
                    V.radec = J.b_radec;
                    V.xyz = J.b_xyz;
                    V.zoff = J.b_zoff;
                }
                test_object<VARIANT, COUNT_CAND, DIST>(J, a, V, sb, out, (uint32_t)st.jx, cn);
            }
            __syncthreads();
            if (sb.count >= (uint32_t)(kSbuf / 2)) flush(sb, out);
        }
        if (failed) break;
        flush(sb, out);
    }
    // statistics: one atomic per warp
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

template <int TILE, int VARIANT, bool CC, bool DIST>
cudaError_t launch_t(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_items, const MatchOut &out,
                     cudaStream_t st)
{
    auto k = pair_kernel<TILE, VARIANT, CC, DIST>;
    int per_sm = L.blocks_per_sm;
    if (per_sm <= 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TILE, 0);
        if (per_sm < 1) per_sm = 1;
    }
    const uint64_t want = ((uint64_t)n_items + L.chunk - 1) / L.chunk;
    unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)L.sm_count * per_sm, std::max<uint64_t>(want, 1));
    k<<<grid, TILE, 0, st>>>(jobs, n_jobs, n_items, L.zc, L.chunk, out);
    return cudaGetLastError();
}

template <int TILE>
cudaError_t launch_tile(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_items, const MatchOut &out,
                        cudaStream_t st)
{
    if (L.variant == 1)
        return L.dist ? launch_t<TILE, 1, true, true>(L, jobs, n_jobs, n_items, out, st)
                      : launch_t<TILE, 1, true, false>(L, jobs, n_jobs, n_items, out, st);
    if (L.count_cand)
        return L.dist ? launch_t<TILE, 0, true, true>(L, jobs, n_jobs, n_items, out, st)
                      : launch_t<TILE, 0, true, false>(L, jobs, n_jobs, n_items, out, st);
    return L.dist ? launch_t<TILE, 0, false, true>(L, jobs, n_jobs, n_items, out, st)
                  : launch_t<TILE, 0, false, false>(L, jobs, n_jobs, n_items, out, st);
}

}  // namespace

cudaError_t launch_pairs(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_items, const MatchOut &out,
                         cudaStream_t st)
{
    switch (L.tile) {
    case 64: return launch_tile<64>(L, jobs, n_jobs, n_items, out, st);
    case 256: return launch_tile<256>(L, jobs, n_jobs, n_items, out, st);
    default: return launch_tile<128>(L, jobs, n_jobs, n_items, out, st);
    }
}

}  // namespace xm
