// xm_match.cu -- zone-pair window search + pair test + compaction, as one
// persistent work-stealing launch over tiles of A objects.
//
// Replaces the reference's per-zone-pair launches (Worker.cu:330-366) of the
// all-pairs kernel xmatch_kernel (Worker.cu:65-241):
//   * a tile is `TILE` consecutive objects of A in (zone, ra) order, one per
//     thread; blocks claim `chunk` tiles at a time from a global counter, so
//     uneven zones and uneven jobs balance themselves;
//   * for every B zone within nz of its own zone (Worker.cu:338-341) a thread
//     bisects the ra-sorted zone for the window (ra - alpha, ra + alpha) and
//     the two wrapped windows (+-2 pi) of the RA branches of
//     Worker.cu:89,98,110, instead of testing the whole zone;
//   * the pair test is the reference predicate (Worker.cu:88-97): dec cut,
//     RA cut, chord^2 < (2 sin(r/2))^2, all FP64 with the unit vectors of the
//     unshifted (ra, dec) (the branch-3 sign error of Worker.cu:118 fixed).
//     XM_FILTER32 first evaluates chord^2 in FP32 from the stored FP32 unit
//     vectors and discards a pair only when that value exceeds a bound proven
//     to imply chord^2_FP64 >= threshold; every other pair is decided by the
//     FP64 predicate, so the pair set is the FP64 one bit for bit.
//   * matches are compacted per warp with __ballot_sync/__popc into a block
//     buffer in shared memory, which is appended to the global output with a
//     single atomicAdd per flush (Worker.cu:128-240 uses two Hillis-Steele
//     scans per block instead); a full output buffer is detected, never
//     silently truncated (Worker.cu:147-148).
#include <algorithm>
#include <cmath>
#include <vector>

#include "xm_internal.h"
#include "xm_match.cuh"
#include "xm_math.cuh"

namespace xm {

namespace {

constexpr int kSbuf = 1024;       // block output staging records
constexpr double kWinEps = 1e-12; // window widening (radians), >> FP64 rounding of ra +- alpha

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// first k in [lo, hi) with ra[k] >= v
__device__ __forceinline__ uint32_t lower_ra(const double2 *__restrict__ radec, uint32_t lo, uint32_t hi, double v)
{
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&radec[mid].x) < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Candidate enumeration state of one A object: the B zones in its band and,
// in each zone, up to three ra windows (direct, and the two wrapped ones).
struct Cursor {
    int zb, zb_end;     // current B zone, last B zone
    int win;            // 0 direct, 1 branch 2 (B near 0), 2 branch 3 (B near 2 pi), 3 done
    uint32_t j, j_end;  // candidate index range inside the current window
    uint32_t b0, b1;    // current zone range
    double hi_cur;      // window upper end (ra); j advances while ra[j] <= hi_cur
    uint32_t w1_lo, w1_hi;  // direct window range (to keep the wrapped ones disjoint)
};

struct AObj {
    double ra, dec;
    double x, y, z;     // FP64 unit vector
    float fx, fy, fz;
    double alpha;
    long long id;
    bool full_ring;     // alpha >= 3: every object of the zone is a candidate
};

// Open window `win` of the current zone; returns false if it is empty.
__device__ __forceinline__ bool open_window(const JobDev &J, const AObj &a, Cursor &c)
{
    const double2 *__restrict__ br = J.b_radec;
    c.j = c.j_end = 0;
    if (a.full_ring) {
        if (c.win != 0) return false;
        c.j = c.b0;
        c.j_end = c.b1;
        c.hi_cur = INFINITY;
        return c.j < c.j_end;
    }
    const double lo = a.ra - a.alpha - kWinEps, hi = a.ra + a.alpha + kWinEps;
    if (c.win == 0) {
        c.j = lower_ra(br, c.b0, c.b1, lo);
        c.j_end = c.b1;
        c.hi_cur = hi;
        c.w1_lo = c.j;
        c.w1_hi = c.j;   // advanced while the window is consumed
        return c.j < c.j_end;
    }
    if (c.win == 1) {   // branch 2: ra_b in (ra_a - 2pi - alpha, ra_a - 2pi + alpha)
        const double hi2 = hi - XM_TWO_PI + kWinEps;
        if (hi2 < __ldg(&br[c.b0].x)) return false;
        const double lo2 = lo - XM_TWO_PI - kWinEps;
        c.j = lower_ra(br, c.b0, c.b1, lo2);
        c.j_end = c.w1_lo;  // below the direct window
        c.hi_cur = hi2;
        return c.j < c.j_end;
    }
    // branch 3: ra_b in (ra_a + 2pi - alpha, ra_a + 2pi + alpha)
    const double lo3 = lo + XM_TWO_PI - kWinEps;
    if (lo3 > __ldg(&br[c.b1 - 1].x)) return false;
    const double hi3 = hi + XM_TWO_PI + kWinEps;
    const uint32_t s = lower_ra(br, c.b0, c.b1, lo3);
    c.j = s > c.w1_hi ? s : c.w1_hi;   // above the direct window
    c.j_end = c.b1;
    c.hi_cur = hi3;
    return c.j < c.j_end;
}

// Advance to the next candidate index; false when the zone band is exhausted.
// Windows of one zone are visited in the order direct, branch 2, branch 3;
// the direct one is consumed first, so w1_hi is its true end when branch 3
// is opened.
__device__ __forceinline__ bool next_candidate(const JobDev &J, const AObj &a, Cursor &c, uint32_t &out)
{
    for (;;) {
        if (c.j < c.j_end) {
            const uint32_t j = c.j;
            if (__ldg(&J.b_radec[j].x) <= c.hi_cur) {
                c.j = j + 1;
                if (c.win == 0) c.w1_hi = c.j;
                out = j;
                return true;
            }
            c.j = c.j_end;   // past the window's upper end
        }
        if (c.win < 2 && !a.full_ring) {
            c.win++;
            open_window(J, a, c);
            continue;
        }
        c.zb++;
        if (c.zb > c.zb_end) return false;
        c.b0 = __ldg(&J.b_zoff[c.zb]);
        c.b1 = __ldg(&J.b_zoff[c.zb + 1]);
        c.win = 0;
        if (c.b0 >= c.b1) {
            c.j = c.j_end = 0;
            c.win = 2;       // empty zone: skip its windows
            if (!a.full_ring) continue;
            continue;
        }
        open_window(J, a, c);
    }
}

struct Counters {
    unsigned long long tested, cand, border, exact;
};

// FP64 predicate of Worker.cu:88-97 on one pair (unit vector of B by sincos).
__device__ __forceinline__ bool exact_test(const JobDev &J, const AObj &a, double2 rb, double &c2)
{
    if (!(fabs(__dsub_rn(a.dec, rb.y)) < J.sr_rad)) return false;
    double d = __dsub_rn(a.ra, rb.x);
    if (!(fabs(d) < a.alpha || fabs(__dsub_rn(d, XM_TWO_PI)) < a.alpha || fabs(__dadd_rn(d, XM_TWO_PI)) < a.alpha))
        return false;
    double x2, y2, z2;
    radec2xyz(rb.x, rb.y, x2, y2, z2);
    c2 = chord2(a.x, a.y, a.z, x2, y2, z2);
    return c2 < J.sr_dist2;
}

__device__ __forceinline__ bool cuts_pass(const JobDev &J, const AObj &a, double2 rb)
{
    if (!(fabs(__dsub_rn(a.dec, rb.y)) < J.sr_rad)) return false;
    double d = __dsub_rn(a.ra, rb.x);
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

__device__ __forceinline__ int find_job(const JobDev *__restrict__ jobs, int n_jobs, uint32_t t)
{
    int lo = 0, hi = n_jobs;   // last j with tile_begin <= t
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(&jobs[mid].tile_begin) <= t) lo = mid; else hi = mid;
    }
    return lo;
}

template <int TILE, int VARIANT, bool COUNT_CAND, bool DIST>
__global__ void __launch_bounds__(TILE)
pair_kernel(const JobDev *__restrict__ jobs, int n_jobs, uint32_t n_tiles, uint32_t chunk, MatchOut out)
{
    __shared__ SBuf sb;
    __shared__ uint32_t s_t0;
    if (threadIdx.x == 0) sb.count = 0;
    Counters cn = {0ull, 0ull, 0ull, 0ull};
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_t0 = (uint32_t)atomicAdd(&out.counters[1], (unsigned long long)chunk);
        __syncthreads();
        const uint32_t t0 = s_t0;
        if (t0 >= n_tiles) break;
        const uint32_t t1 = min(t0 + chunk, n_tiles);
        for (uint32_t t = t0; t < t1; ++t) {
            const int jx = n_jobs > 1 ? find_job(jobs, n_jobs, t) : 0;
            const JobDev J = jobs[jx];
            const uint32_t i = (t - J.tile_begin) * TILE + threadIdx.x;
            if (i < J.nA) {
                AObj a;
                const float4 fa = __ldg(&J.a_xyz[i]);
                const double2 ra = __ldg(&J.a_radec[i]);
                a.ra = ra.x;
                a.dec = ra.y;
                a.fx = fa.x; a.fy = fa.y; a.fz = fa.z;
                const int za = (int)__float_as_uint(fa.w);
                a.alpha = __ldg(&J.alpha[za]);
                a.full_ring = a.alpha >= 3.0;
                a.id = __ldg(&J.a_id[i]);
                radec2xyz(a.ra, a.dec, a.x, a.y, a.z);
                Cursor c;
                c.zb = max(0, za - J.nz) - 1;
                c.zb_end = min(J.n_zones - 1, za + J.nz);
                c.win = 2;
                c.j = c.j_end = 0;
                c.b0 = c.b1 = 0;
                c.hi_cur = 0;
                c.w1_lo = c.w1_hi = 0;
                uint32_t k;
                while (next_candidate(J, a, c, k)) {
                    cn.tested++;
                    bool m = false;
                    double c2 = 0;
                    if (VARIANT == 0) {   // FP32 reject, FP64 decision
                        if (COUNT_CAND) cn.cand += cuts_pass(J, a, __ldg(&J.b_radec[k])) ? 1ull : 0ull;
                        const float4 fb = __ldg(&J.b_xyz[k]);
                        const float dx = a.fx - fb.x, dy = a.fy - fb.y, dz = a.fz - fb.z;
                        const float c32 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
                        if (!(c32 > J.thr_hi)) {
                            cn.border += (c32 >= J.thr_lo) ? 1ull : 0ull;
                            cn.exact++;
                            m = exact_test(J, a, __ldg(&J.b_radec[k]), c2);
                        }
                    } else {              // plain all-FP64
                        const double2 rb = __ldg(&J.b_radec[k]);
                        if (cuts_pass(J, a, rb)) {
                            cn.cand++;
                            cn.exact++;
                            double x2, y2, z2;
                            radec2xyz(rb.x, rb.y, x2, y2, z2);
                            c2 = chord2(a.x, a.y, a.z, x2, y2, z2);
                            m = c2 < J.sr_dist2;
                        }
                    }
                    long long idb = 0;
                    double dist = 0;
                    if (m) {
                        idb = __ldg(&J.b_id[k]);
                        if (DIST) dist = 2.0 * asin(sqrt(c2) * 0.5);
                    }
                    emit(sb, out, m, a.id, idb, dist, (uint32_t)jx);
                }
            }
            __syncthreads();
            if (sb.count >= (uint32_t)(kSbuf / 2)) flush(sb, out);
        }
        flush(sb, out);
    }
    // statistics: one atomic per warp
    const unsigned lane = threadIdx.x & 31;
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
cudaError_t launch_t(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_tiles, const MatchOut &out,
                     cudaStream_t st)
{
    auto k = pair_kernel<TILE, VARIANT, CC, DIST>;
    int per_sm = L.blocks_per_sm;
    if (per_sm <= 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, TILE, 0);
        if (per_sm < 1) per_sm = 1;
    }
    unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)L.sm_count * per_sm, std::max<uint32_t>(n_tiles, 1));
    k<<<grid, TILE, 0, st>>>(jobs, n_jobs, n_tiles, L.chunk, out);
    return cudaGetLastError();
}

template <int TILE>
cudaError_t launch_tile(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_tiles,
                        const MatchOut &out, cudaStream_t st)
{
    const bool plain = L.variant == 1;
    if (plain) {
        return L.dist ? launch_t<TILE, 1, true, true>(L, jobs, n_jobs, n_tiles, out, st)
                      : launch_t<TILE, 1, true, false>(L, jobs, n_jobs, n_tiles, out, st);
    }
    if (L.count_cand)
        return L.dist ? launch_t<TILE, 0, true, true>(L, jobs, n_jobs, n_tiles, out, st)
                      : launch_t<TILE, 0, true, false>(L, jobs, n_jobs, n_tiles, out, st);
    return L.dist ? launch_t<TILE, 0, false, true>(L, jobs, n_jobs, n_tiles, out, st)
                  : launch_t<TILE, 0, false, false>(L, jobs, n_jobs, n_tiles, out, st);
}

}  // namespace

cudaError_t launch_pairs(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_tiles,
                         const MatchOut &out, cudaStream_t st)
{
    switch (L.tile) {
    case 64: return launch_tile<64>(L, jobs, n_jobs, n_tiles, out, st);
    case 256: return launch_tile<256>(L, jobs, n_jobs, n_tiles, out, st);
    default: return launch_tile<128>(L, jobs, n_jobs, n_tiles, out, st);
    }
}

}  // namespace xm
