// xm_build.cu -- device zone builder (replaces Sorter::Sort, Sorter.cu:141-185).
//
// Input: n records {int64 id, f64 ra_deg, f64 dec_deg} in device memory.
// Records with a zone outside [0, n_zones) or a non-finite ra are dropped
// (a non-finite ra can never pass the RA cut of Worker.cu:89-110); dec = +90
// on the upper edge is kept in the last zone.
//
// Output (per segment), ordered by (zone, raq, input index):
//   zone_off[n_zones + 1]  first object of each zone (zone_off[z+1] = end),
//                          the zone begin/end of Sorter.cu:156-165
//   id[n]                  int64
//   radec[n]               double2 radians, deg / RAD2DEG (Sorter.cu:52-62)
//   xyz[n]                 float4: FP32 unit vector (the project sincos,
//                          Worker.cu:31-40, rounded to FP32), w = raq bits
// zone = floor((dec + 90) / zh) (Sorter.cu:20-24); raq = the leading 27
// bits of floor(ra_rad * 2^31 / pi), a monotone quantisation of ra (its
// step is 2 pi / 2^27, 4.7e-8 rad), so within a zone
// the objects are sorted by ra up to that step and window searches on raq
// give supersets of the RA windows.  (The reference sorts by (zone, ra) with
// a comparison sort, Sorter.cu:27-43,153; the pair set does not depend on
// the order inside a zone.)
//
// Passes:
//   1. zb_keys     key = zone << raq_bits | raq, value = input index; digit
//                  histograms of every radix pass; populated zone range
//   2. LSD radix sort of (key, value), 8-bit digits, one pass per non-constant
//      digit: rs_upsweep (per-tile digit counts) + exclusive scan +
//      rs_downsweep (stable in-tile ranking by warp match_any, coalesced
//      scatter through shared memory)
//   3. zb_gather   SoA in sorted order, unit vectors by the project sincos
//   4. zb_bounds   zone offsets from the sorted keys
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "xm_async.cuh"
#include "xm_internal.h"
#include "xm_math.cuh"

namespace {

constexpr int kTileItems = 8;                 // keys per thread per radix tile
constexpr int kRsThreads = 512;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kTile = kRsThreads * kTileItems;   // 4096 keys
constexpr int kMaxPasses = 8;
constexpr int kRaqBits = 27;                  // raq bits kept; the 5 above carry the zone in a bucket

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

struct KeyParams {
    double zh_deg;
    int n_zones;
    int raq_shift;     // 32 - raq_bits
    int raq_bits;
    int passes;
};

__global__ void zb_keys(const xm_obj *__restrict__ objs, unsigned long long n, KeyParams kp,
                        unsigned long long *__restrict__ keys, uint32_t *__restrict__ vals,
                        uint32_t *__restrict__ hist, uint32_t *__restrict__ misc)
{
    __shared__ uint32_t h[kMaxPasses][256];
    __shared__ unsigned s_lo, s_hi, s_bad;
    for (int i = threadIdx.x; i < kMaxPasses * 256; i += blockDim.x) (&h[0][0])[i] = 0;
    if (threadIdx.x == 0) {
        s_lo = 0xFFFFFFFFu;
        s_hi = 0u;
        s_bad = 0u;
    }
    __syncthreads();
    unsigned zlo = 0xFFFFFFFFu, zhi = 0u, bad = 0u;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned long long warp0 = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull;
    for (unsigned long long wb = warp0; wb < n; wb += stride) {
        const unsigned long long i = wb + (threadIdx.x & 31);
        unsigned long long key = ~0ull;
        if (i < n) {
            const xm_obj o = objs[i];
            const int z = isfinite(o.ra_deg) ? xm::zone_of(o.dec_deg, kp.zh_deg, kp.n_zones) : -1;
            if (z < 0) {
                key = (unsigned long long)kp.n_zones << kp.raq_bits;   // after every valid zone
                ++bad;
            } else {
                const double ra = __ddiv_rn(o.ra_deg, XM_RAD2DEG);
                key = ((unsigned long long)z << kp.raq_bits) | (xm::raq32(ra) >> kp.raq_shift);
                zlo = min(zlo, (unsigned)z);
                zhi = max(zhi, (unsigned)z);
            }
            keys[i] = key;
            vals[i] = (uint32_t)i;
        }
        // warp-aggregated histogram updates
        for (int p = 0; p < kp.passes; ++p) {
            const int d = i < n ? (int)((key >> (8 * p)) & 255u) : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if (d >= 0 && (threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1))
                atomicAdd(&h[p][d], (uint32_t)__popc(peers));
        }
    }
    zlo = __reduce_min_sync(0xffffffffu, zlo);
    zhi = __reduce_max_sync(0xffffffffu, zhi);
    bad = __reduce_add_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&s_lo, zlo);
        atomicMax(&s_hi, zhi);
        atomicAdd(&s_bad, bad);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kp.passes * 256; i += blockDim.x) {
        const uint32_t v = (&h[0][0])[i];
        if (v) atomicAdd(&hist[i], v);
    }
    if (threadIdx.x == 0) {
        if (s_lo != 0xFFFFFFFFu) atomicMin(&misc[0], s_lo);
        atomicMax(&misc[1], s_hi);
        if (s_bad) atomicAdd(&misc[2], s_bad);
    }
}

// Per-tile digit counts, digit-major: cnt[d * n_tiles + tile].
__global__ void __launch_bounds__(kRsThreads)
rs_upsweep(const unsigned long long *__restrict__ keys, unsigned long long n, int shift, uint32_t n_tiles,
           uint32_t *__restrict__ cnt)
{
    __shared__ uint32_t h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const unsigned long long base = (unsigned long long)blockIdx.x * kTile;
#pragma unroll
    for (int k = 0; k < kTileItems; ++k) {
        const unsigned long long pos = base + (unsigned long long)k * kRsThreads + threadIdx.x;
        int d = -1;
        if (pos < n) d = (int)((keys[pos] >> shift) & 255u);
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (d >= 0 && (threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += blockDim.x) cnt[(size_t)d * n_tiles + blockIdx.x] = h[d];
}

// Stable scatter of one tile: items of warp w are w*256 + k*32 + lane
// (k = 0..7), processed in k order, so lower ranks go to earlier items.
__global__ void __launch_bounds__(kRsThreads)
rs_downsweep(const unsigned long long *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
             unsigned long long n, int shift, uint32_t n_tiles, const uint32_t *__restrict__ off,
             unsigned long long *__restrict__ keys_out, uint32_t *__restrict__ vals_out)
{
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned long long *skeys = (unsigned long long *)smem;           // [kTile]
    uint32_t *svals = (uint32_t *)(skeys + kTile);                     // [kTile]
    uint32_t *wcnt = svals + kTile;                                    // [kRsWarps][256]
    uint32_t *dbase = wcnt + kRsWarps * 256;                           // [256] tile-local digit start
    uint32_t *gbase = dbase + 256;                                     // [256] global start
    const int warp = threadIdx.x >> 5;
    const unsigned lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kRsWarps * 256; i += blockDim.x) wcnt[i] = 0;
    __syncthreads();
    const unsigned long long base = (unsigned long long)blockIdx.x * kTile;
    unsigned long long key[kTileItems];
    uint32_t val[kTileItems], rank[kTileItems];
    int dig[kTileItems];
#pragma unroll
    for (int k = 0; k < kTileItems; ++k) {
        const unsigned long long pos = base + (unsigned long long)warp * 256 + k * 32 + lane;
        int d = -1;
        key[k] = 0;
        val[k] = 0;
        if (pos < n) {
            key[k] = keys_in[pos];
            val[k] = vals_in[pos];
            d = (int)((key[k] >> shift) & 255u);
        }
        dig[k] = d;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        uint32_t c = 0;
        if (d >= 0 && (int)lane == leader) {
            c = wcnt[warp * 256 + d];
            wcnt[warp * 256 + d] = c + (uint32_t)__popc(peers);
        }
        c = __shfl_sync(0xffffffffu, c, leader);
        rank[k] = c + (uint32_t)__popc(peers & lanemask_lt());
    }
    __syncthreads();
    // warp prefixes per digit and the tile's digit totals
    if (threadIdx.x < 256) {
        const int d = threadIdx.x;
        uint32_t run = 0;
        for (int w = 0; w < kRsWarps; ++w) {
            const uint32_t t = wcnt[w * 256 + d];
            wcnt[w * 256 + d] = run;
            run += t;
        }
        dbase[d] = run;   // total, turned into an exclusive prefix below
        gbase[d] = off[(size_t)d * n_tiles + blockIdx.x];
    }
    __syncthreads();
    if (threadIdx.x < 32) {   // exclusive scan of the 256 totals by one warp
        uint32_t v[8], s = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            v[q] = dbase[lane * 8 + q];
            s += v[q];
        }
        uint32_t x = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (unsigned)o) x += y;
        }
        uint32_t run = x - s;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            dbase[lane * 8 + q] = run;
            run += v[q];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kTileItems; ++k) {
        const int d = dig[k];
        if (d >= 0) {
            const uint32_t p = dbase[d] + wcnt[warp * 256 + d] + rank[k];
            skeys[p] = key[k];
            svals[p] = val[k];
        }
    }
    __syncthreads();
    const unsigned long long rem = n - base;
    const uint32_t m = rem < (unsigned long long)kTile ? (uint32_t)rem : (uint32_t)kTile;
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
        const unsigned long long kk = skeys[i];
        const int d = (int)((kk >> shift) & 255u);
        const uint32_t g = gbase[d] + (i - dbase[d]);
        keys_out[g] = kk;
        vals_out[g] = svals[i];
    }
}

__global__ void zb_gather(const unsigned long long *__restrict__ keys, const uint32_t *__restrict__ vals,
                          const xm_obj *__restrict__ objs, unsigned long long n_kept, unsigned long long raq_mask,
                          long long *__restrict__ id, double2 *__restrict__ radec, float4 *__restrict__ xyz)
{
    for (unsigned long long j = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; j < n_kept;
         j += (unsigned long long)gridDim.x * blockDim.x) {
        const xm_obj o = objs[vals[j]];
        const double ra = __ddiv_rn(o.ra_deg, XM_RAD2DEG);
        const double dec = __ddiv_rn(o.dec_deg, XM_RAD2DEG);
        double x, y, z;
        xm::radec2xyz(ra, dec, x, y, z);
        id[j] = o.id;
        radec[j] = make_double2(ra, dec);
        xyz[j] = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z),
                             __uint_as_float((uint32_t)(keys[j] & raq_mask)));
    }
}

// zone_off[z] = first sorted position whose zone is >= z, for z in [0, n_zones]:
// the first object of every populated zone marks its zone, then empty zones
// take the position found by bisecting the sorted keys.
__global__ void zb_bounds_mark(const unsigned long long *__restrict__ keys, unsigned long long n, int raq_bits,
                               int n_zones, uint32_t *__restrict__ zone_off)
{
    for (unsigned long long j = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; j < n;
         j += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long z = keys[j] >> raq_bits;
        if (z < (unsigned long long)n_zones && (j == 0 || (keys[j - 1] >> raq_bits) != z)) zone_off[z] = (uint32_t)j;
    }
}

__global__ void zb_bounds_fill(const unsigned long long *__restrict__ keys, unsigned long long n, int raq_bits,
                               int n_zones, uint32_t *__restrict__ zone_off)
{
    for (unsigned long long z = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; z <= (unsigned long long)n_zones;
         z += (unsigned long long)gridDim.x * blockDim.x) {
        if (z < (unsigned long long)n_zones && zone_off[z] != 0xFFFFFFFFu) continue;
        const unsigned long long t = z << raq_bits;
        unsigned long long lo = 0, hi = n;   // first key >= t
        while (lo < hi) {
            const unsigned long long mid = (lo + hi) >> 1;
            if (keys[mid] < t) lo = mid + 1; else hi = mid;
        }
        zone_off[z] = (uint32_t)lo;
    }
}

// ---------------------------------------------------------------------------
// Zone-bucket build.
//   zc_count     objects per bucket of 2^bucket_shift consecutive zones (a
//                shared-memory histogram per block), the populated zone range
//                and the dropped count; reads ra and dec only
//   scan         bucket offsets (the buckets' atomic cursors)
//   zc_scatter   records streamed through shared memory (bulk async copies),
//                each kept record into its bucket as a 32-byte ZRec through
//                the bucket cursors (few enough buckets that their write
//                fronts stay in L2)
//   zs_bucket    one block per bucket: zone counts and offsets, the bucket's
//                (raq, input index) keys into zone order in shared memory,
//                each zone of at most kWarpZone objects ranked by one warp and
//                written out as the segment's SoA
//   zs_block     zones of kWarpZone+1 .. kBlockZone objects: bitonic sort of a
//                block
// Zones above kBlockZone objects send the segment to the radix-sort build.
// ---------------------------------------------------------------------------
constexpr int kWarpZone = 256;
constexpr int kBlockZone = 8192;
constexpr int kZsThreads = 512;
constexpr int kBucketMaxShift = 5;   // at most 32 zones per bucket
constexpr int kBucketThreads = 256;

struct ZRec {          // 32 bytes, one per kept object
    double ra, dec;    // radians
    long long id;
    uint32_t raq;      // zone within its bucket << kRaqBits | leading kRaqBits of raq32(ra)
    uint32_t idx;      // input index
};
constexpr uint32_t kRaqMask = (1u << kRaqBits) - 1u;

// A ZRec moves in one 256-bit global access (sm_100's widest): one store
// transaction per scattered record instead of two, which measured 1.73 against
// 2.49 ms for the scatter of 50M records when half of each record was written.
__device__ __forceinline__ void st_rec(ZRec *q, double ra, double dec, unsigned long long id, uint32_t key,
                                       uint32_t idx)
{
    const unsigned long long w3 = ((unsigned long long)idx << 32) | key;
    asm volatile("st.global.v4.b64 [%0], {%1, %2, %3, %4};" ::"l"(q), "l"(__double_as_longlong(ra)),
                 "l"(__double_as_longlong(dec)), "l"(id), "l"(w3)
                 : "memory");
}

// ---- record tiles streamed through shared memory (scatter pass) ----
// A block walks its tiles of kTileRecs records through two shared-memory
// buffers.  A full tile of a 16-byte aligned input is one bulk asynchronous
// copy (cp.async.bulk, completion counted on the buffer's mbarrier), issued
// while the previous tile is processed; a partial last tile, or a tile of an
// input that is only 8-byte aligned, is copied by the block's threads.
constexpr int kStageThreads = 256;
constexpr int kPerThread = 8;                              // records per thread per tile
constexpr int kTileRecs = kStageThreads * kPerThread;      // 2048 records, 48 KB
constexpr uint32_t kTileBytes = kTileRecs * 24u;

struct TileRing {
    unsigned long long w[2][kTileRecs * 3];   // raw records: id, ra bits, dec bits
    uint64_t bar[2];
};

__device__ __forceinline__ double rec_ra(const unsigned long long *w, uint32_t i)
{
    return __longlong_as_double((long long)w[3 * i + 1]);
}
__device__ __forceinline__ double rec_dec(const unsigned long long *w, uint32_t i)
{
    return __longlong_as_double((long long)w[3 * i + 2]);
}

// Zone of a record; -1 if it is dropped (zone outside the sphere, non-finite ra).
__device__ __forceinline__ int rec_zone(double ra_deg, double dec_deg, const KeyParams &kp)
{
    return isfinite(ra_deg) ? xm::zone_of(dec_deg, kp.zh_deg, kp.n_zones) : -1;
}

// Calls f(first record, count, records in shared memory) for every tile of the
// block (tiles blockIdx.x, blockIdx.x + gridDim.x, ...).  Returns false (the
// same on every thread) if a bounded wait for a bulk copy ran out; the copies
// still in flight have then been waited for (bounded) before returning.
template <class F>
__device__ bool for_each_tile(const xm_obj *__restrict__ objs, unsigned long long n, bool bulk_ok, TileRing &R,
                              F f)
{
    const unsigned long long n_tiles = (n + kTileRecs - 1) / kTileRecs;
    const unsigned long long step = gridDim.x;
    auto bulk = [&](unsigned long long t) { return bulk_ok && (t + 1) * kTileRecs <= n; };
    if (threadIdx.x == 0) {
        xm::mbar_init(&R.bar[0], 1);
        xm::mbar_init(&R.bar[1], 1);
        xm::fence_mbar_init();
    }
    __syncthreads();
    uint32_t par = 0;        // bit b: parity of buffer b's next phase
    uint32_t pend = 0;       // bit b: a bulk copy into buffer b is in flight
    auto issue = [&](unsigned long long t, int b) {   // thread 0
        xm::fence_proxy_async();
        xm::mbar_expect_tx(&R.bar[b], kTileBytes);
        xm::bulk_g2s(R.w[b], objs + t * kTileRecs, kTileBytes, &R.bar[b]);
    };
    unsigned long long t = blockIdx.x;
    if (t < n_tiles && bulk(t)) {
        if (threadIdx.x == 0) issue(t, 0);
        pend |= 1u;
    }
    bool ok = true;
    for (int b = 0; t < n_tiles; t += step, b ^= 1) {
        const unsigned long long tn = t + step;
        if (tn < n_tiles && bulk(tn)) {   // the other buffer was released by the last __syncthreads
            if (threadIdx.x == 0) issue(tn, b ^ 1);
            pend |= 2u >> b;
        }
        const uint32_t cnt = (uint32_t)min((unsigned long long)kTileRecs, n - t * kTileRecs);
        if (bulk(t)) {
            const bool got = xm::mbar_wait(&R.bar[b], (par >> b) & 1u);
            par ^= 1u << b;
            pend &= ~(1u << b);
            if (!__syncthreads_and(got)) {
                ok = false;
                pend |= 1u << b;
                par ^= 1u << b;
                break;
            }
        } else {
            const unsigned long long *src = reinterpret_cast<const unsigned long long *>(objs + t * kTileRecs);
            for (uint32_t i = threadIdx.x; i < 3 * cnt; i += blockDim.x) R.w[b][i] = __ldg(src + i);
            __syncthreads();
        }
        f(t * kTileRecs, cnt, R.w[b]);
        __syncthreads();
    }
    if (!ok) {   // drain: wait (bounded) for the copies still in flight
        for (int b = 0; b < 2; ++b)
            if (pend & (1u << b)) xm::mbar_wait(&R.bar[b], (par >> b) & 1u);
        __syncthreads();
    }
    return ok;
}

// Lanes whose value equals the previous lane's form runs (consecutive equal
// zones, as in dec-ordered input); the run's first lane acts for the run.
struct Run {
    unsigned head;     // first lane of the calling lane's run
    unsigned len;      // run length (valid on the head lane)
    bool is_head;
};

__device__ __forceinline__ Run warp_run(int v, unsigned lane)
{
    const int prev = __shfl_up_sync(0xffffffffu, v, 1);
    const bool h = lane == 0 || prev != v;
    const unsigned heads = __ballot_sync(0xffffffffu, h);
    const unsigned le = (2u << lane) - 1u;   // lanes <= lane (all lanes for lane 31)
    Run r;
    r.head = 31u - __clz(heads & le);
    const unsigned after = heads & ~le;
    r.len = (after ? (unsigned)(__ffs(after) - 1) : 32u) - lane;
    r.is_head = h;
    return r;
}

// Pass 1: objects per bucket of 2^shift zones (a shared-memory histogram when
// the buckets fit, else run-aggregated global atomics), the populated zone
// range (misc[0], misc[1]) and the dropped count (misc[2]).  Only ra and dec
// of each record are read.
constexpr int kCountU = 8;                // records per lane per iteration
constexpr int kHistMax = 24 * 1024;       // buckets of a shared-memory histogram (96 KB)

template <bool SMEM>
__global__ void __launch_bounds__(256)
zc_count(const xm_obj *__restrict__ objs, unsigned long long n, KeyParams kp, int shift, int n_buckets,
         uint32_t *__restrict__ bcnt, uint32_t *__restrict__ misc)
{
    extern __shared__ uint32_t s_hist[];   // [n_buckets] when SMEM
    __shared__ unsigned s_lo, s_hi, s_bad;
    if (SMEM)
        for (int i = threadIdx.x; i < n_buckets; i += blockDim.x) s_hist[i] = 0;
    if (threadIdx.x == 0) {
        s_lo = 0xFFFFFFFFu;
        s_hi = 0u;
        s_bad = 0u;
    }
    __syncthreads();
    const unsigned lane = threadIdx.x & 31;
    unsigned zlo = 0xFFFFFFFFu, zhi = 0u, bad = 0u;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x * kCountU;
    const unsigned long long warp0 =
        (((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull) * kCountU;
    for (unsigned long long wb = warp0; wb < n; wb += stride) {
        double ra[kCountU], dec[kCountU];
#pragma unroll
        for (int u = 0; u < kCountU; ++u) {
            const unsigned long long i = wb + 32u * u + lane;
            ra[u] = 0.0;
            dec[u] = 0.0;
            if (i < n) {
                ra[u] = __ldg(&objs[i].ra_deg);
                dec[u] = __ldg(&objs[i].dec_deg);
            }
        }
#pragma unroll
        for (int u = 0; u < kCountU; ++u) {
            const unsigned long long i = wb + 32u * u + lane;
            int bk = -2;
            if (i < n) {
                const int z = rec_zone(ra[u], dec[u], kp);
                if (z < 0) {
                    ++bad;
                    bk = -1;
                } else {
                    zlo = min(zlo, (unsigned)z);
                    zhi = max(zhi, (unsigned)z);
                    bk = z >> shift;
                }
            }
            if (SMEM) {
                if (bk >= 0) atomicAdd(&s_hist[bk], 1u);
            } else {
                const Run r = warp_run(bk, lane);
                if (r.is_head && bk >= 0) atomicAdd(&bcnt[bk], r.len);
            }
        }
    }
    zlo = __reduce_min_sync(0xffffffffu, zlo);
    zhi = __reduce_max_sync(0xffffffffu, zhi);
    bad = __reduce_add_sync(0xffffffffu, bad);
    if (lane == 0) {
        atomicMin(&s_lo, zlo);
        atomicMax(&s_hi, zhi);
        atomicAdd(&s_bad, bad);
    }
    __syncthreads();
    if (SMEM)
        for (int i = threadIdx.x; i < n_buckets; i += blockDim.x) {
            const uint32_t v = s_hist[i];
            if (v) atomicAdd(&bcnt[i], v);
        }
    if (threadIdx.x == 0) {
        if (s_lo != 0xFFFFFFFFu) atomicMin(&misc[0], s_lo);
        atomicMax(&misc[1], s_hi);
        if (s_bad) atomicAdd(&misc[2], s_bad);
    }
}

// Pass 2: every kept record into its bucket (unordered inside it) as a 32-byte
// ZRec; bcur holds the buckets' start offsets and ends as their end offsets.
// Records stream through shared memory (for_each_tile); each thread first
// claims the slots of its 8 records (8 independent atomics in flight, one per
// run of equal buckets in a warp), then writes them.
__global__ void __launch_bounds__(kStageThreads, 2)
zc_scatter(const xm_obj *__restrict__ objs, unsigned long long n, KeyParams kp, int shift, bool bulk_ok,
           uint32_t *__restrict__ bcur, ZRec *__restrict__ recs, uint32_t *__restrict__ misc)
{
    extern __shared__ __align__(128) unsigned char scat_smem[];
    TileRing &R = *reinterpret_cast<TileRing *>(scat_smem);
    const unsigned lane = threadIdx.x & 31;
    const uint32_t zmask = (1u << shift) - 1u;
    const bool ok = for_each_tile(objs, n, bulk_ok, R, [&](unsigned long long first, uint32_t cnt,
                                                            const unsigned long long *w) {
        uint32_t base[kPerThread];
        unsigned head[kPerThread];
        int zl[kPerThread];   // zone within the bucket, -1 = no record
#pragma unroll
        for (int u = 0; u < kPerThread; ++u) {
            const uint32_t i = threadIdx.x + (uint32_t)u * kStageThreads;
            int bk = -2;
            zl[u] = -1;
            if (i < cnt) {
                const int z = rec_zone(rec_ra(w, i), rec_dec(w, i), kp);
                bk = z < 0 ? -1 : (z >> shift);
                if (z >= 0) zl[u] = (int)((uint32_t)z & zmask);
            }
            const Run r = warp_run(bk, lane);
            head[u] = r.head;
            base[u] = 0;
            if (r.is_head && bk >= 0) base[u] = atomicAdd(&bcur[bk], r.len);
        }
#pragma unroll
        for (int u = 0; u < kPerThread; ++u) {
            const uint32_t b0 = __shfl_sync(0xffffffffu, base[u], head[u]);
            if (zl[u] >= 0) {
                const uint32_t i = threadIdx.x + (uint32_t)u * kStageThreads;
                const double ra = __ddiv_rn(rec_ra(w, i), XM_RAD2DEG);
                const double dec = __ddiv_rn(rec_dec(w, i), XM_RAD2DEG);
                st_rec(recs + b0 + (lane - head[u]), ra, dec, w[3 * i],
                       (uint32_t)zl[u] << kRaqBits | xm::raq32(ra) >> (32 - kRaqBits), (uint32_t)(first + i));
            }
        }
    });
    if (!ok && threadIdx.x == 0) atomicOr(&misc[5], 2u);
}

struct ZOut {
    long long *id;
    double2 *radec;
    float4 *xyz;
    uint16_t *zbin;    // per-zone bin index, or null
    int bin_log2;
};

// Per-zone bin index of a segment (xm_segment::zbin).  With K = 2^bin_log2
// bins of the quantised-ra turn, entry j of zone z's row is the number of the
// zone's objects whose raq is below (j + 1) << (kRaqBits - bin_log2), i.e.
// the start of bin j + 1 relative to the zone's first object (saturated at
// 0xFFFF).  The pair kernel's window search starts inside the bin of the
// window's lower end instead of bisecting the whole zone.  One warp per zone:
// a shared-memory histogram of the zone's bins, then its inclusive scan.
template <class R>
__device__ __forceinline__ void zone_bins_warp(uint32_t mz, R raq_of, uint32_t *hist, uint16_t *row, int bin_log2,
                                               unsigned lane)
{
    hist[lane] = 0;
    __syncwarp();
    for (uint32_t q = lane; q < mz; q += 32) atomicAdd(&hist[raq_of(q) >> (kRaqBits - bin_log2)], 1u);
    __syncwarp();
    uint32_t incl = hist[lane];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= (unsigned)d) incl += y;
    }
    if ((int)lane < (1 << bin_log2)) row[lane] = (uint16_t)min(incl, 0xFFFFu);
    __syncwarp();
}

// The index of a sorted segment from its quantised ra (xyz.w), one warp per
// zone (the radix-sort build).
__global__ void zb_bins(const float4 *__restrict__ xyz, const uint32_t *__restrict__ zone_off, int n_zones,
                        int bin_log2, uint16_t *__restrict__ zbin)
{
    __shared__ uint32_t hist[8][32];
    const unsigned lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    for (int z = blockIdx.x * 8 + w; z < n_zones; z += gridDim.x * 8) {
        const uint32_t b = zone_off[z], m = zone_off[z + 1] - b;
        zone_bins_warp(m, [&](uint32_t q) { return __float_as_uint(xyz[b + q].w) & kRaqMask; }, hist[w],
                       zbin + ((size_t)z << bin_log2), bin_log2, lane);
    }
}

// A record of a buffer the running kernel does not write: one 256-bit load
// through the read-only path.
__device__ __forceinline__ ZRec zs_load_ro(const ZRec *p)
{
    unsigned long long a, b, c, d;
    asm("ld.global.nc.v4.b64 {%0, %1, %2, %3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(p));
    ZRec r;
    r.ra = __longlong_as_double((long long)a);
    r.dec = __longlong_as_double((long long)b);
    r.id = (long long)c;
    r.raq = (uint32_t)d;
    r.idx = (uint32_t)(d >> 32);
    return r;
}

// A record the running kernel's block wrote (before a barrier): coherent loads.
__device__ __forceinline__ ZRec zs_load(const ZRec *p)
{
    const double2 a = reinterpret_cast<const double2 *>(p)[0];
    const uint4 b = reinterpret_cast<const uint4 *>(p)[1];
    ZRec r;
    r.ra = a.x;
    r.dec = a.y;
    r.id = (long long)(((unsigned long long)b.y << 32) | b.x);
    r.raq = b.z;
    r.idx = b.w;
    return r;
}

__device__ __forceinline__ void zs_emit(const ZRec &r, unsigned long long j, const ZOut &o)
{
    double x, y, z;
    xm::radec2xyz(r.ra, r.dec, x, y, z);
    o.id[j] = r.id;
    o.radec[j] = make_double2(r.ra, r.dec);
    o.xyz[j] = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z),
                           __uint_as_float(r.raq & kRaqMask));
}

// Sort key of a record inside its zone: (raq, input index).
__device__ __forceinline__ unsigned long long zrec_key(const ZRec *p)
{
    const uint4 t = reinterpret_cast<const uint4 *>(p)[1];
    return ((unsigned long long)(t.z & kRaqMask) << 32) | t.w;
}

// Per-warp scratch of the in-zone sort.
// In-zone ranking groups the keys by the top kSortGroupBits of raq (128 sub-ranges
// of the turn: about one key per group in a zone of 100 objects) and ranks each
// inside its group; 32 groups measured 0.76 ms of the bucket sort's 2.18 at 50M.
constexpr int kSortGroupBits = 7;
constexpr int kSortGroups = 1 << kSortGroupBits;

struct WarpSort {
    unsigned long long key[kWarpZone];   // keys grouped by raq sub-range
    uint16_t at[kWarpZone];              // zone entry at each rank
    uint32_t cnt[kSortGroups], base[kSortGroups];
    uint32_t hist[32];                   // bin index histogram
};

// Ranks the m <= kWarpZone keys key_of(0..m) of one zone by value (distinct:
// the input index is part of the key): W.at[rank] = entry.  Keys are grouped
// by the top kSortGroupBits raq bits (kSortGroups sub-ranges of the turn), then
// ranked inside their group.
template <int E, class K>
__device__ __forceinline__ void zs_rank_zone(uint32_t m, K key_of, WarpSort &W, unsigned lane)
{
#pragma unroll
    for (int g = 0; g < kSortGroups / 32; ++g) W.cnt[lane + 32 * g] = 0;
    __syncwarp();
    unsigned long long key[E];
    uint32_t sub[E], slot[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint32_t k = lane + 32u * e;
        key[e] = ~0ull;
        sub[e] = 0;
        slot[e] = 0;
        if (k < m) {
            key[e] = key_of(k);
            sub[e] = (uint32_t)(key[e] >> (32 + kRaqBits - kSortGroupBits));
            slot[e] = atomicAdd(&W.cnt[sub[e]], 1u);
        }
    }
    __syncwarp();
    // exclusive scan of the group counts, kSortGroups / 32 consecutive groups per lane
    constexpr int G = kSortGroups / 32;
    uint32_t c[G], t = 0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        c[g] = W.cnt[G * lane + g];
        t += c[g];
    }
    uint32_t incl = t;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= (unsigned)d) incl += y;
    }
    uint32_t run = incl - t;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        W.base[G * lane + g] = run;
        run += c[g];
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint32_t k = lane + 32u * e;
        if (k < m) W.key[W.base[sub[e]] + slot[e]] = key[e];
    }
    __syncwarp();
    // rank = entries of the group with a smaller key, an equal key counting by its
    // slot (keys are distinct here -- the input index is part of them -- but the
    // ranks stay a permutation whatever the keys)
    uint32_t rank[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint32_t k = lane + 32u * e;
        rank[e] = 0;
        if (k < m) {
            const uint32_t b0 = W.base[sub[e]], b1 = b0 + W.cnt[sub[e]], me = b0 + slot[e];
            uint32_t r = b0;
            for (uint32_t q = b0; q < b1; ++q) {
                const unsigned long long kq = W.key[q];
                r += (kq < key[e] || (kq == key[e] && q < me)) ? 1u : 0u;
            }
            rank[e] = r;
        }
    }
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) {
        const uint32_t k = lane + 32u * e;
        if (k < m) W.at[rank[e]] = (uint16_t)k;
    }
    __syncwarp();
}

template <class K>
__device__ __forceinline__ void zs_rank(uint32_t m, K key_of, WarpSort &W, unsigned lane)
{
    if (m <= 32) zs_rank_zone<1>(m, key_of, W, lane);
    else if (m <= 64) zs_rank_zone<2>(m, key_of, W, lane);
    else if (m <= 128) zs_rank_zone<4>(m, key_of, W, lane);
    else zs_rank_zone<8>(m, key_of, W, lane);
}

// Pass 3, one block per bucket (buckets blockIdx.x, + gridDim.x, ...).
// A bucket of at most kBucketCap records is ordered in shared memory by one
// counting sort over (zone, raq sub-range) bins -- kSubBits leading raq bits,
// 128 sub-ranges of the turn per zone, 4096 bins per bucket of 32 zones:
//  1. the bucket's keys (ZRec::raq: zone in bucket, raq) read once,
//     kKeyBatch loads in flight per thread, into shared memory by bucket
//     position; each key's slot inside its bin from the bin count's atomic
//     (few keys per bin, so few collide);
//  2. the exclusive scan of the bin counts by the block: bin bases, which give
//     the zone offsets (zone_off) and the zones' bin index rows directly;
//  3. the bucket positions into bin order (base + slot; shared memory only);
//  4. each key ranked inside its bin by raq, then by input index (read from
//     the records when two raq are equal; about one key per bin in a zone of
//     100 objects): rank = the key's place in the bucket's order;
//  5. the whole block writes the bucket's SoA in that order, gathering each
//     record from the bucket a second time (from L2).
// Zones of more than kWarpZone objects are copied to recs_z in bin order and
// listed for zs_block.  A bucket of more than kBucketCap records orders its
// records through recs_z in global memory, one warp per zone (zs_rank).
constexpr int kBucketCap = 6144;
constexpr uint16_t kNoRecord = 0xFFFF;   // a position of a zone sorted by zs_block
constexpr int kBucketWarps = kBucketThreads / 32;
constexpr int kKeyBatch = 8;             // key loads in flight per thread (step 1)
constexpr int kEmitBatch = 2;            // record loads in flight per thread (step 5)
constexpr int kSubBits = 7;
constexpr int kBinShift = kRaqBits - kSubBits;   // ZRec::raq >> kBinShift = zone in bucket << kSubBits | sub-range
constexpr int kSortBins = 1 << (kBucketMaxShift + kSubBits);
constexpr int kBinsPerThread = kSortBins / kBucketThreads;
static_assert(kBinsPerThread == 16 && (kSortBins >> kBucketMaxShift) == kBucketThreads / 2,
              "a zone's bins are owned by 8 threads of 16 bins each");
// Bin counts and bases are 16-bit (a bucket holds at most kBucketCap records),
// two bins to a word; bin b is in half b & 1 of word b / 2 + b / 16: the 8
// words of a thread's 16 bins start 9 words apart, so the 32 lanes of a warp
// touch 32 different banks.
constexpr int kBinWords = kSortBins / 2 + kSortBins / 16;   // bins 0 .. kSortBins - 1
__device__ __forceinline__ uint32_t bin_word(uint32_t b) { return (b >> 1) + (b >> 4); }
__device__ __forceinline__ uint32_t bin_get(const uint32_t *w, uint32_t b)
{
    return (w[bin_word(b)] >> ((b & 1u) << 4)) & 0xFFFFu;
}
static_assert(kBucketCap < 0x10000, "16-bit bin counts and bases");

// 66 KB (two blocks per SM; three, with the 80 registers a thread that allows, measured
// slower: 1.75 against 1.55 ms at 50M).
struct BucketSmem {
    union {
        struct {
            uint32_t key[kBucketCap];   // ZRec::raq (zone in bucket, raq) at each bucket position
            uint16_t pos[kBucketCap];   // bucket position at each bin-order slot
            uint16_t out[kBucketCap];   // slot inside its bin at each position, then position at each rank
        } s;
        WarpSort ws[kBucketWarps];      // buckets above kBucketCap
    } u;
    uint32_t cnt[kBinWords];            // bin counts (bin_get)
    uint32_t base[kBinWords + 1];       // bin bases (bin_get); bin kSortBins = records placed
    uint32_t zcnt[1 << kBucketMaxShift];
    uint32_t zbeg[(1 << kBucketMaxShift) + 1];
    uint32_t zcur[1 << kBucketMaxShift];
    uint32_t wsum[kBucketWarps];
};

// Zone offsets of the bucket and the list of its zones for zs_block, from
// S.zbeg (warp 0).
__device__ __forceinline__ void zs_zone_offsets(const BucketSmem &S, int bk, int n_buckets, int z0, int nzb,
                                                uint32_t r0, uint32_t r1, uint32_t *zone_off, int n_zones,
                                                uint32_t *big, uint32_t *misc)
{
    const unsigned lane = threadIdx.x;
    const uint32_t c = (int)lane < nzb ? S.zbeg[lane + 1] - S.zbeg[lane] : 0u;
    if ((int)lane < nzb) {
        zone_off[z0 + lane] = r0 + S.zbeg[lane];
        if (c > (uint32_t)kWarpZone) {
            big[atomicAdd(&misc[3], 1u)] = (uint32_t)(z0 + lane);
            atomicMax(&misc[4], c);
        }
    }
    if (bk == n_buckets - 1 && lane == 0) {
        zone_off[n_zones] = r1;
        zone_off[n_zones + 1] = misc[2];
    }
}

// A bucket of m <= kBucketCap records (steps 1-5 above).
__device__ __forceinline__ void zs_bucket_smem(BucketSmem &S, const ZRec *__restrict__ rb, ZRec *__restrict__ rz,
                                               uint32_t m, int bk, int n_buckets, int z0, int nzb, uint32_t r0,
                                               uint32_t r1, uint32_t *zone_off, int n_zones, const ZOut &o,
                                               uint32_t *big, uint32_t *misc)
{
    const unsigned t = threadIdx.x, lane = t & 31;
    const int warp = t >> 5;
    uint32_t *key = S.u.s.key;
    uint16_t *pos = S.u.s.pos, *out = S.u.s.out;
    for (int w = t; w < kBinWords; w += kBucketThreads) S.cnt[w] = 0;
    __syncthreads();
    for (uint32_t i0 = t; i0 < m; i0 += kKeyBatch * kBucketThreads) {   // 1. keys and slots
        uint32_t v[kKeyBatch];
#pragma unroll
        for (int u = 0; u < kKeyBatch; ++u) {
            const uint32_t i = i0 + u * kBucketThreads;
            if (i < m) v[u] = __ldg(&rb[i].raq);
        }
#pragma unroll
        for (int u = 0; u < kKeyBatch; ++u) {
            const uint32_t i = i0 + u * kBucketThreads;
            if (i >= m) break;
            key[i] = v[u];
            if ((v[u] >> kRaqBits) < (uint32_t)nzb) {
                const uint32_t b = v[u] >> kBinShift, sh = (b & 1u) << 4;
                out[i] = (uint16_t)(atomicAdd(&S.cnt[bin_word(b)], 1u << sh) >> sh);
            } else {
                out[i] = kNoRecord;
                atomicOr(&misc[5], 1u);   // cannot happen: written by zc_scatter for this bucket
            }
        }
    }
    __syncthreads();
    {   // 2. exclusive scan; thread t owns bins [kBinsPerThread t, kBinsPerThread (t + 1)),
        //    words [9 t, 9 t + 8) of S.cnt and S.base
        constexpr int W = kBinsPerThread / 2;
        uint32_t c[W], tot = 0;
#pragma unroll
        for (int j = 0; j < W; ++j) {
            c[j] = S.cnt[(W + 1) * t + j];
            tot += (c[j] & 0xFFFFu) + (c[j] >> 16);
        }
        uint32_t incl = tot;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (unsigned)d) incl += y;
        }
        if (lane == 31) S.wsum[warp] = incl;
        __syncthreads();
        uint32_t run = incl - tot;
        for (int w = 0; w < warp; ++w) run += S.wsum[w];
        if ((t & 7) == 0) S.zbeg[t >> 3] = run;   // zone t / 8 begins at bin kBinsPerThread t
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const uint32_t lo = run, hi = run + (c[j] & 0xFFFFu);
            S.base[(W + 1) * t + j] = lo | (hi << 16);
            run = hi + (c[j] >> 16);
        }
        if (t == kBucketThreads - 1) {
            S.base[bin_word(kSortBins)] = run;
            S.zbeg[1 << kBucketMaxShift] = run;
        }
    }
    __syncthreads();
    if (t < 32) zs_zone_offsets(S, bk, n_buckets, z0, nzb, r0, r1, zone_off, n_zones, big, misc);
    if (o.zbin) {   // row j of zone zl: start of bin j + 1 inside the zone
        const int L = o.bin_log2;
        for (int e = t; e < (nzb << L); e += kBucketThreads) {
            const int zl = e >> L, j = e & ((1 << L) - 1);
            const uint32_t v = bin_get(S.base, (zl << kSubBits) + ((j + 1) << (kSubBits - L))) -
                               bin_get(S.base, zl << kSubBits);
            o.zbin[((size_t)(z0 + zl) << L) + j] = (uint16_t)v;
        }
    }
    for (uint32_t i = t; i < m; i += kBucketThreads) {   // 3. positions into bin order
        const uint16_t sl = out[i];
        if (sl != kNoRecord) pos[bin_get(S.base, key[i] >> kBinShift) + sl] = (uint16_t)i;
    }
    __syncthreads();
    const uint32_t mc = bin_get(S.base, kSortBins);   // records placed (= m)
    for (uint32_t q = t; q < mc; q += kBucketThreads) {   // 4. ranks inside the bins
        const uint16_t i = pos[q];
        const uint32_t k = key[i];
        const uint32_t b = k >> kBinShift, zl = b >> kSubBits;
        if (S.zbeg[zl + 1] - S.zbeg[zl] > (uint32_t)kWarpZone) {   // zs_block sorts it from recs_z
            const ZRec r = zs_load_ro(rb + i);
            st_rec(rz + q, r.ra, r.dec, (unsigned long long)r.id, r.raq, r.idx);
            out[q] = kNoRecord;
            continue;
        }
        // order inside the bin: raq, then the input index (read from the records, for
        // the rare equal raq), then the slot -- the ranks stay a permutation whatever
        // the keys
        const uint32_t b0 = bin_get(S.base, b), b1 = bin_get(S.base, b + 1);
        uint32_t rank = b0;
        for (uint32_t p = b0; p < b1; ++p) {
            const uint16_t ip = pos[p];
            const uint32_t kp = key[ip];
            bool before = kp < k;
            if (kp == k && p != q) {
                const uint32_t xp = __ldg(&rb[ip].idx), xq = __ldg(&rb[i].idx);
                before = xp < xq || (xp == xq && p < q);
            }
            rank += before ? 1u : 0u;
        }
        out[rank] = i;
    }
    __syncthreads();
    // 5. the bucket's SoA in order, kEmitBatch records per thread in flight: every
    // lane busy whatever the zone sizes, writes contiguous across zones
    for (uint32_t j0 = t; j0 < mc; j0 += kEmitBatch * kBucketThreads) {
        ZRec x[kEmitBatch];
        uint16_t q[kEmitBatch];
#pragma unroll
        for (int u = 0; u < kEmitBatch; ++u) {
            const uint32_t j = j0 + u * kBucketThreads;
            q[u] = j < mc ? out[j] : kNoRecord;
            if (q[u] != kNoRecord) x[u] = zs_load_ro(rb + q[u]);
        }
#pragma unroll
        for (int u = 0; u < kEmitBatch; ++u)
            if (q[u] != kNoRecord) zs_emit(x[u], (unsigned long long)r0 + j0 + u * kBucketThreads, o);
    }
    __syncthreads();
}

// A bucket of more than kBucketCap records: zone order through recs_z, then
// one warp per zone of at most kWarpZone objects ranks and emits it.
__device__ __forceinline__ void zs_bucket_global(BucketSmem &S, const ZRec *__restrict__ rb, ZRec *__restrict__ rz,
                                                 uint32_t m, int bk, int n_buckets, int z0, int nzb, uint32_t r0,
                                                 uint32_t r1, uint32_t *zone_off, int n_zones, const ZOut &o,
                                                 uint32_t *big, uint32_t *misc)
{
    const unsigned t = threadIdx.x, lane = t & 31;
    const int warp = t >> 5;
    WarpSort &W = S.u.ws[warp];
    if (t < 32) S.zcnt[t] = 0;
    __syncthreads();
    for (uint32_t i = t; i < m; i += kBucketThreads) {   // zone counts
        const uint32_t zl = reinterpret_cast<const uint4 *>(rb + i)[1].z >> kRaqBits;
        if (zl < (uint32_t)nzb) atomicAdd(&S.zcnt[zl], 1u);
        else atomicOr(&misc[5], 1u);   // cannot happen: written by zc_scatter for this bucket
    }
    __syncthreads();
    if (t < 32) {   // exclusive scan of the (at most 32) zone counts
        const uint32_t c = (int)t < nzb ? S.zcnt[t] : 0u;
        uint32_t incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (unsigned)d) incl += y;
        }
        S.zbeg[t] = incl - c;
        S.zcur[t] = incl - c;
        if (t == 31) S.zbeg[32] = incl;
        __syncwarp();
        zs_zone_offsets(S, bk, n_buckets, z0, nzb, r0, r1, zone_off, n_zones, big, misc);
    }
    __syncthreads();
    for (uint32_t i = t; i < m; i += kBucketThreads) {   // records in zone order
        const ZRec *p = rb + i;
        const uint4 v = reinterpret_cast<const uint4 *>(p)[1];
        const uint32_t zl = v.z >> kRaqBits;
        if (zl >= (uint32_t)nzb) continue;
        const uint32_t q = atomicAdd(&S.zcur[zl], 1u);
        reinterpret_cast<double2 *>(rz + q)[0] = reinterpret_cast<const double2 *>(p)[0];
        reinterpret_cast<uint4 *>(rz + q)[1] = v;
    }
    __syncthreads();
    for (int k = warp; k < nzb; k += kBucketWarps) {
        const uint32_t zb = S.zbeg[k], mz = S.zbeg[k + 1] - zb;
        const ZRec *zr = rz + zb;
        if (o.zbin)   // the zone's bin index (the order inside the zone does not matter)
            zone_bins_warp(mz, [&](uint32_t q) { return (uint32_t)(zrec_key(zr + q) >> 32); }, W.hist,
                           o.zbin + ((size_t)(z0 + k) << o.bin_log2), o.bin_log2, lane);
        if (mz == 0 || mz > (uint32_t)kWarpZone) continue;   // zs_block sorts a large zone from recs_z
        zs_rank(mz, [&](uint32_t q) { return zrec_key(zr + q); }, W, lane);
        for (uint32_t p = lane; p < mz; p += 32)
            zs_emit(zs_load(zr + W.at[p]), (unsigned long long)r0 + zb + p, o);
        __syncwarp();
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kBucketThreads, 2)
zs_bucket(const ZRec *__restrict__ recs_b, ZRec *__restrict__ recs_z, const uint32_t *__restrict__ bend,
          uint32_t *__restrict__ zone_off, int n_zones, int shift, int n_buckets, ZOut o,
          uint32_t *__restrict__ big, uint32_t *__restrict__ misc)
{
    extern __shared__ __align__(16) unsigned char bk_smem[];
    BucketSmem &S = *reinterpret_cast<BucketSmem *>(bk_smem);
    for (int bk = blockIdx.x; bk < n_buckets; bk += gridDim.x) {
        const int z0 = bk << shift;
        const int nzb = min(1 << shift, n_zones - z0);
        const uint32_t r0 = bk ? bend[bk - 1] : 0u, r1 = bend[bk];
        const uint32_t m = r1 - r0;
        if (m <= (uint32_t)kBucketCap)
            zs_bucket_smem(S, recs_b + r0, recs_z + r0, m, bk, n_buckets, z0, nzb, r0, r1, zone_off, n_zones, o,
                           big, misc);
        else
            zs_bucket_global(S, recs_b + r0, recs_z + r0, m, bk, n_buckets, z0, nzb, r0, r1, zone_off, n_zones, o,
                             big, misc);
    }
}

// Zones of kWarpZone+1 .. kBlockZone objects: one block each, bitonic sort of
// (raq, idx) keys padded to a power of two, then records emitted in order.
__global__ void __launch_bounds__(kZsThreads)
zs_block(const ZRec *__restrict__ recs, const uint32_t *__restrict__ zone_off, const uint32_t *__restrict__ big,
         const uint32_t *__restrict__ misc, ZOut o)
{
    extern __shared__ __align__(16) unsigned char zs_smem[];
    unsigned long long *sk = (unsigned long long *)zs_smem;        // [kBlockZone]
    uint16_t *sp = (uint16_t *)(sk + kBlockZone);                   // [kBlockZone]
    const uint32_t n_big = misc[3];
    for (uint32_t q = blockIdx.x; q < n_big; q += gridDim.x) {
        const uint32_t z = big[q];
        const uint32_t b = zone_off[z];
        const uint32_t m = zone_off[z + 1] - b;
        if (m > (uint32_t)kBlockZone) continue;   // left to the radix-sort build
        uint32_t P = 1;
        while (P < m) P <<= 1;
        for (uint32_t k = threadIdx.x; k < P; k += blockDim.x) {
            unsigned long long key = ~0ull;
            if (k < m) {
                const uint4 t = reinterpret_cast<const uint4 *>(recs + b + k)[1];
                key = ((unsigned long long)(t.z & kRaqMask) << 32) | t.w;
            }
            sk[k] = key;
            sp[k] = (uint16_t)k;
        }
        for (uint32_t size = 2; size <= P; size <<= 1) {
            for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
                __syncthreads();
                for (uint32_t t = threadIdx.x; t < P / 2; t += blockDim.x) {
                    const uint32_t i = 2 * t - (t & (stride - 1));
                    const uint32_t j = i + stride;
                    const bool up = (i & size) == 0;
                    const unsigned long long ki = sk[i], kj = sk[j];
                    if ((ki > kj) == up) {
                        sk[i] = kj;
                        sk[j] = ki;
                        const uint16_t pi = sp[i];
                        sp[i] = sp[j];
                        sp[j] = pi;
                    }
                }
            }
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < m; k += blockDim.x)
            zs_emit(zs_load_ro(recs + b + sp[k]), (unsigned long long)b + k, o);
        __syncthreads();
    }
}

int grid_for(unsigned long long n, int threads, int sm_count, int per_sm = 8)
{
    unsigned long long blocks = (n + threads - 1) / threads;
    unsigned long long cap = (unsigned long long)sm_count * per_sm;
    if (blocks > cap) blocks = cap;
    return (int)std::max<unsigned long long>(blocks, 1);
}

int bit_width(uint64_t v)
{
    int b = 0;
    while (v) {
        ++b;
        v >>= 1;
    }
    return b;
}

}  // namespace

// Bits of the quantised ra kept in the segment (xyz.w) and in the sort key:
// kRaqBits (2^27 steps per turn, 4.7e-8 rad); radix passes over zone and raq.
void xm_raq_layout(int32_t n_zones, int *raq_bits, int *passes)
{
    const int zb = bit_width((uint64_t)n_zones);   // zone values 0..n_zones (n_zones = dropped)
    *passes = (zb + kRaqBits + 7) / 8;
    *raq_bits = kRaqBits;
}

static xm_status ensure(xm_ctx *ctx, void **p, size_t *have, size_t need)
{
    if (*have >= need && *p) return XM_OK;
    if (*p) xm_dev_free(ctx, *p);
    *p = nullptr;
    *have = 0;
    XM_TRY(xm_dev_alloc(ctx, p, need));
    *have = need;
    return XM_OK;
}

static xm_status build_lsd(xm_segment *seg, const xm_obj *objs, uint64_t n, xm_stats *stats)
{
    xm_ctx *ctx = seg->ctx;
    cudaStream_t st = ctx->stream;
    if (n >= 0xFFFFFFF0ull) {
        ctx->last_error = "segment larger than 2^32-16 records";
        return XM_ERR_INVALID;
    }
    const int nz = seg->n_zones;
    int raq_bits, passes;
    xm_raq_layout(nz, &raq_bits, &passes);
    if (passes > kMaxPasses) {
        ctx->last_error = "too many zones for the sort key";
        return XM_ERR_INVALID;
    }
    seg->raq_bits = raq_bits;
    uint32_t launches = 0;
    XM_TRY(xm_seg_storage(seg, n));
    const uint64_t nn = std::max<uint64_t>(n, 1);
    const uint32_t n_tiles = (uint32_t)((nn + kTile - 1) / kTile);
    // scratch: keys x2, vals x2, tile counts and offsets, scan scratch, histograms
    const size_t kb = ((nn * 8 + 255) & ~(size_t)255), vb = ((nn * 4 + 255) & ~(size_t)255);
    const size_t cb = (((size_t)n_tiles * 256 * 4 + 4 + 255) & ~(size_t)255);
    const size_t sb = ((xm_scan_tmp_bytes((size_t)n_tiles * 256) + 255) & ~(size_t)255);
    const size_t hb = kMaxPasses * 256 * 4 + 64;
    XM_TRY(ensure(ctx, &ctx->build_tmp, &ctx->build_tmp_bytes, 2 * kb + 2 * vb + 2 * cb + sb + hb));
    char *w = (char *)ctx->build_tmp;
    unsigned long long *k0 = (unsigned long long *)w; w += kb;
    unsigned long long *k1 = (unsigned long long *)w; w += kb;
    uint32_t *v0 = (uint32_t *)w; w += vb;
    uint32_t *v1 = (uint32_t *)w; w += vb;
    uint32_t *tcnt = (uint32_t *)w; w += cb;
    uint32_t *toff = (uint32_t *)w; w += cb;
    void *scan_tmp = w; w += sb;
    uint32_t *hist = (uint32_t *)w;               // [passes][256]
    uint32_t *misc = hist + kMaxPasses * 256;     // z_lo, z_hi, dropped

    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[0], st));
    XM_CUDA(ctx, cudaMemsetAsync(hist, 0, hb, st));
    XM_CUDA(ctx, cudaMemsetAsync(misc, 0xFF, 4, st));
    KeyParams kp{seg->zh_deg, nz, 32 - raq_bits, raq_bits, passes};
    if (n > 0) {
        zb_keys<<<grid_for(n, 256, ctx->sm_count, 4), 256, 0, st>>>(objs, n, kp, k0, v0, hist, misc);
        launches++;
    }
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[8], st));
    std::vector<uint32_t> h((size_t)kMaxPasses * 256 + 16, 0);
    XM_CUDA(ctx, cudaMemcpyAsync(h.data(), hist, hb, cudaMemcpyDeviceToHost, st));
    XM_CUDA(ctx, cudaStreamSynchronize(st));
    const uint32_t *hm = h.data() + kMaxPasses * 256;
    const uint64_t dropped = n ? hm[2] : 0;
    seg->n = n - dropped;
    seg->n_in = n;
    if (seg->n > 0) {
        seg->z_lo = (int32_t)hm[0];
        seg->z_hi = (int32_t)hm[1];
    } else {
        seg->z_lo = 0;
        seg->z_hi = -1;
    }
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[9], st));
    // LSD radix passes (a pass whose digit is the same for every key is skipped)
    const size_t ds_smem = (size_t)kTile * 12 + (size_t)kRsWarps * 256 * 4 + 512 * 4;
    XM_CUDA(ctx, cudaFuncSetAttribute(rs_downsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ds_smem));
    unsigned long long *kin = k0, *kout = k1;
    uint32_t *vin = v0, *vout = v1;
    for (int p = 0; p < passes && n > 0; ++p) {
        bool constant = false;
        for (int d = 0; d < 256; ++d)
            if (h[(size_t)p * 256 + d] == n) constant = true;
        if (constant) continue;
        rs_upsweep<<<n_tiles, kRsThreads, 0, st>>>(kin, n, 8 * p, n_tiles, tcnt);
        XM_CUDA(ctx, xm_scan_exclusive_u32(tcnt, toff, (size_t)n_tiles * 256, scan_tmp, st));
        rs_downsweep<<<n_tiles, kRsThreads, ds_smem, st>>>(kin, vin, n, 8 * p, n_tiles, toff, kout, vout);
        launches += 5;
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    XM_CUDA(ctx, cudaGetLastError());
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[10], st));
    if (seg->n > 0) {
        const unsigned long long mask = (1ull << raq_bits) - 1;
        zb_gather<<<grid_for(seg->n, 256, ctx->sm_count, 8), 256, 0, st>>>(kin, vin, objs, seg->n, mask,
                                                                            (long long *)seg->id, seg->radec,
                                                                            seg->xyz);
        launches++;
    }
    XM_CUDA(ctx, cudaMemsetAsync(seg->zone_off, 0xFF, ((size_t)nz + 1) * 4, st));
    if (n > 0) {
        zb_bounds_mark<<<grid_for(n, 256, ctx->sm_count, 8), 256, 0, st>>>(kin, n, raq_bits, nz, seg->zone_off);
        launches++;
    }
    zb_bounds_fill<<<grid_for((uint64_t)nz + 1, 256, ctx->sm_count, 8), 256, 0, st>>>(kin, n, raq_bits, nz,
                                                                                       seg->zone_off);
    launches++;
    if (seg->zbin) {
        zb_bins<<<grid_for((uint64_t)nz, 256, ctx->sm_count, 8), 256, 0, st>>>(seg->xyz, seg->zone_off, nz,
                                                                                seg->bin_log2, seg->zbin);
        launches++;
    }
    XM_CUDA(ctx, cudaGetLastError());
    // dropped count beside the offsets
    seg->dropped_host = (uint32_t)dropped;
    XM_CUDA(ctx, cudaMemcpyAsync(seg->zone_off + nz + 1, &seg->dropped_host, 4, cudaMemcpyHostToDevice, st));
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[11], st));
    XM_CUDA(ctx, cudaStreamSynchronize(st));
    if (stats) {
        float a = 0, b = 0, c = 0, d = 0;
        cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[8]);
        cudaEventElapsedTime(&b, ctx->ev[8], ctx->ev[9]);
        cudaEventElapsedTime(&c, ctx->ev[9], ctx->ev[10]);
        cudaEventElapsedTime(&d, ctx->ev[10], ctx->ev[11]);
        stats->ms_zb_count += a;    // key generation + digit histograms
        stats->ms_zb_scan += b;     // histogram read-back
        stats->ms_zb_scatter += c;  // radix passes
        stats->ms_zb_sort += d;     // gather + zone offsets
        stats->ms_build += a + b + c + d;
        stats->n_launches += launches;
    }
    return XM_OK;
}

// The segment's arrays live in one allocation (fewer, equal-sized blocks keep
// the context's memory pool from fragmenting when segments come and go):
// zone_off, id, radec, xyz, each 256-byte aligned.
void xm_seg_layout(xm_segment *seg, void *base)
{
    char *w = (char *)base;
    seg->zone_off = base ? (uint32_t *)w : nullptr;
    seg->id = base ? (int64_t *)(w + seg->off_id) : nullptr;
    seg->radec = base ? (double2 *)(w + seg->off_radec) : nullptr;
    seg->xyz = base ? (float4 *)(w + seg->off_xyz) : nullptr;
    seg->zbin = base && seg->bin_log2 ? (uint16_t *)(w + seg->off_zbin) : nullptr;
}

// Bins per zone of a segment's index: none below 16 objects per zone on
// average (a bisection of a few steps is as fast), else about one bin per 2
// to 4 objects, at most 32.
static int bin_log2_for(uint64_t n, int32_t n_zones)
{
    const double avg = (double)n / std::max<int32_t>(n_zones, 1);
    if (avg < 16) return 0;
    if (avg < 32) return 3;
    if (avg < 64) return 4;
    return 5;
}

xm_status xm_seg_storage(xm_segment *seg, uint64_t n)
{
    xm_ctx *ctx = seg->ctx;
    if (seg->host_store) {   // a rebuild makes the host copy of an offloaded segment stale
        cudaFreeHost(seg->host_store);
        seg->host_store = nullptr;
    }
    if (seg->store && seg->cap >= n) return XM_OK;
    const uint64_t c = std::max<uint64_t>(n, 1);
    auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
    seg->bin_log2 = bin_log2_for(c, seg->n_zones);
    const size_t bz = al(((size_t)seg->n_zones + 8) * 4), bi = al((c + 2) * 8), br = al(c * 16), bx = al(c * 16),
                 bb = seg->bin_log2 ? al(((size_t)seg->n_zones << seg->bin_log2) * 2) : 0;
    xm_dev_free(ctx, seg->store);
    seg->store = nullptr;
    seg->cap = 0;
    XM_TRY(xm_dev_alloc(ctx, &seg->store, bz + bi + br + bx + bb));
    seg->store_bytes = bz + bi + br + bx + bb;
    seg->off_id = bz;
    seg->off_radec = bz + bi;
    seg->off_xyz = bz + bi + br;
    seg->off_zbin = bz + bi + br + bx;
    xm_seg_layout(seg, seg->store);
    seg->cap = c;
    XM_CUDA(ctx, cudaMemsetAsync(seg->zone_off, 0, bz, ctx->stream));
    return XM_OK;
}

// Zone-bucket build; *fallback is set when a zone holds more than kBlockZone
// objects (the radix-sort build then redoes the segment).
static xm_status build_zones(xm_segment *seg, const xm_obj *objs, uint64_t n, xm_stats *stats, bool *fallback)
{
    xm_ctx *ctx = seg->ctx;
    cudaStream_t st = ctx->stream;
    *fallback = false;
    const int nz = seg->n_zones;
    int raq_bits, passes;
    xm_raq_layout(nz, &raq_bits, &passes);
    seg->raq_bits = raq_bits;
    XM_TRY(xm_seg_storage(seg, n));
    seg->n_in = n;
    if (n == 0) {   // every zone empty
        XM_CUDA(ctx, cudaMemsetAsync(seg->zone_off, 0, ((size_t)nz + 2) * 4, st));
        XM_CUDA(ctx, cudaStreamSynchronize(st));
        seg->n = 0;
        seg->dropped_host = 0;
        seg->z_lo = 0;
        seg->z_hi = -1;
        return XM_OK;
    }
    // buckets of 2^shift zones, at least 4 per SM
    int shift = kBucketMaxShift;
    while (shift > 0 && (nz >> shift) < ctx->sm_count * 4) --shift;
    const int n_buckets = (nz + (1 << shift) - 1) >> shift;
    // scratch: records by bucket, records of large zones in zone order, bucket
    // counts and cursors, large-zone list, scan scratch, misc
    const size_t rb = (n * sizeof(ZRec) + 255) & ~(size_t)255;
    const size_t bb = (((size_t)n_buckets + 1) * 4 + 255) & ~(size_t)255;
    const size_t zb = (((size_t)nz + 1) * 4 + 255) & ~(size_t)255;
    const size_t sb = (xm_scan_tmp_bytes((size_t)n_buckets) + 255) & ~(size_t)255;
    const size_t mb = 256;
    XM_TRY(ensure(ctx, &ctx->build_tmp, &ctx->build_tmp_bytes, 2 * rb + 2 * bb + zb + sb + mb));
    char *w = (char *)ctx->build_tmp;
    ZRec *recs_b = (ZRec *)w; w += rb;
    ZRec *recs_z = (ZRec *)w; w += rb;
    uint32_t *bcnt = (uint32_t *)w; w += bb;
    uint32_t *bcur = (uint32_t *)w; w += bb;
    uint32_t *big = (uint32_t *)w; w += zb;
    void *scan_tmp = w; w += sb;
    uint32_t *misc = (uint32_t *)w;   // z_lo, z_hi, dropped, n_big, largest big zone, error bits
    uint32_t launches = 0;
    static bool attr = false;
    const size_t smem_scatter = sizeof(TileRing), smem_bucket = sizeof(BucketSmem);
    const size_t smem_block = (size_t)kBlockZone * 10;
    if (!attr) {
        XM_CUDA(ctx, cudaFuncSetAttribute(zc_count<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          kHistMax * 4));
        XM_CUDA(ctx, cudaFuncSetAttribute(zc_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_scatter));
        XM_CUDA(ctx, cudaFuncSetAttribute(zs_bucket, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bucket));
        XM_CUDA(ctx, cudaFuncSetAttribute(zs_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_block));
        attr = true;
    }

    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[0], st));
    XM_CUDA(ctx, cudaMemsetAsync(bcnt, 0, (size_t)n_buckets * 4, st));
    XM_CUDA(ctx, cudaMemsetAsync(misc, 0, 32, st));
    XM_CUDA(ctx, cudaMemsetAsync(misc, 0xFF, 4, st));
    KeyParams kp{seg->zh_deg, nz, 32 - raq_bits, raq_bits, passes};
    const uint64_t cgroups = (n + kCountU - 1) / kCountU;
    if (n_buckets <= kHistMax)
        zc_count<true><<<grid_for(cgroups, 256, ctx->sm_count, 2), 256, (size_t)n_buckets * 4, st>>>(
            objs, n, kp, shift, n_buckets, bcnt, misc);
    else
        zc_count<false><<<grid_for(cgroups, 256, ctx->sm_count, 8), 256, 0, st>>>(objs, n, kp, shift, n_buckets,
                                                                                  bcnt, misc);
    launches++;
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[8], st));
    XM_CUDA(ctx, xm_scan_exclusive_u32(bcnt, bcur, (size_t)n_buckets, scan_tmp, st));
    launches += 3;
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[9], st));
    const bool bulk_ok = ((uintptr_t)objs & 15) == 0;
    const uint64_t n_tiles = (n + kTileRecs - 1) / kTileRecs;
    zc_scatter<<<(unsigned)std::min<uint64_t>(n_tiles, (uint64_t)ctx->sm_count * 2), kStageThreads, smem_scatter,
                 st>>>(objs, n, kp, shift, bulk_ok, bcur, recs_b, misc);
    launches++;
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[10], st));
    ZOut o{(long long *)seg->id, seg->radec, seg->xyz, seg->zbin, seg->bin_log2};
    zs_bucket<<<std::min(n_buckets, ctx->sm_count * 2), kBucketThreads, smem_bucket, st>>>(
        recs_b, recs_z, bcur, seg->zone_off, nz, shift, n_buckets, o, big, misc);
    zs_block<<<ctx->sm_count * 2, kZsThreads, smem_block, st>>>(recs_z, seg->zone_off, big, misc, o);
    launches += 2;
    XM_CUDA(ctx, cudaGetLastError());
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[11], st));
    uint32_t hm[8];
    XM_CUDA(ctx, cudaMemcpyAsync(hm, misc, 32, cudaMemcpyDeviceToHost, st));
    XM_CUDA(ctx, cudaStreamSynchronize(st));
    const uint64_t dropped = hm[2];
    seg->n = n - dropped;
    seg->dropped_host = (uint32_t)dropped;
    if (seg->n > 0) {
        seg->z_lo = (int32_t)hm[0];
        seg->z_hi = (int32_t)hm[1];
    } else {
        seg->z_lo = 0;
        seg->z_hi = -1;
    }
    if (hm[5] & 1u) {
        ctx->last_error = "zone build: a record left its bucket";
        return XM_ERR_CUDA;
    }
    if (hm[5] & 2u) {
        ctx->last_error = "zone build: a bounded wait for a bulk copy of records ran out";
        return XM_ERR_TIMEOUT;
    }
    if (hm[4] > (uint32_t)kBlockZone) *fallback = true;
    if (stats) {
        float a = 0, b = 0, c = 0, d = 0;
        cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[8]);
        cudaEventElapsedTime(&b, ctx->ev[8], ctx->ev[9]);
        cudaEventElapsedTime(&c, ctx->ev[9], ctx->ev[10]);
        cudaEventElapsedTime(&d, ctx->ev[10], ctx->ev[11]);
        stats->ms_zb_count += a;    // objects per bucket
        stats->ms_zb_scan += b;     // bucket offsets
        stats->ms_zb_scatter += c;  // records into buckets
        stats->ms_zb_sort += d;     // zone offsets, in-zone sort + SoA output
        stats->ms_build += a + b + c + d;
        stats->n_launches += launches;
    }
    return XM_OK;
}

xm_status xm_build_impl(xm_segment *seg, const xm_obj *objs, uint64_t n, xm_stats *stats)
{
    xm_ctx *ctx = seg->ctx;
    if (n >= 0xFFFFFFF0ull) {
        ctx->last_error = "segment larger than 2^32-16 records";
        return XM_ERR_INVALID;
    }
    bool fallback = false;
    XM_TRY(build_zones(seg, objs, n, stats, &fallback));
    if (!fallback) return XM_OK;
    return build_lsd(seg, objs, n, stats);
}

// ---------------------------------------------------------------------------
// Zone build without allocation (xm_segment_build_noalloc).  The radix-sort
// scratch is this file-scope device array; host code must not use its name
// as a pointer (it is a host-side stand-in), so its device address is looked
// up once per device with cudaGetSymbolAddress.
// ---------------------------------------------------------------------------
namespace {

constexpr uint64_t kNaMax = XM_NOALLOC_MAX_OBJS;
constexpr uint64_t kNaTiles = (kNaMax + kTile - 1) / kTile;
constexpr size_t kNaAlign(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kNaKeys = kNaAlign(kNaMax * 8);
constexpr size_t kNaVals = kNaAlign(kNaMax * 4);
constexpr size_t kNaCnt = kNaAlign(kNaTiles * 256 * 4 + 4);
constexpr size_t kNaScan = kNaAlign(((kNaTiles * 256 + 4095) / 4096 + 1) * 4);
constexpr size_t kNaHist = kNaAlign(kMaxPasses * 256 * 4 + 64);
constexpr size_t kNaBytes = 2 * kNaKeys + 2 * kNaVals + 2 * kNaCnt + kNaScan + kNaHist;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

constexpr int kNaMaxDevices = 64;
void *g_noalloc_ptr[kNaMaxDevices] = {};
std::mutex g_noalloc_mu;

// Makes `device` current for the call and gives the caller's current device
// back on every return path.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int device)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) {
            cudaGetLastError();
            prev = -1;
        }
        ok = cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

extern "C" xm_status xm_segment_build_noalloc(int device, void *stream, const xm_obj *objs, uint64_t n,
                                              double zh_deg, int64_t *out_id, double *out_radec, float *out_xyz,
                                              uint32_t *out_zone_off, uint64_t zone_off_cap, uint64_t *n_kept)
{
    if (n > kNaMax) return XM_ERR_TOO_LARGE;
    if (!(zh_deg > 0) || !std::isfinite(zh_deg) || !out_zone_off || !n_kept || device < 0 ||
        device >= kNaMaxDevices)
        return XM_ERR_INVALID;
    if (n && (!objs || !out_id || !out_radec || !out_xyz)) return XM_ERR_INVALID;
    const double nzd = std::ceil(180 / zh_deg);
    if (nzd > 2.0e9) return XM_ERR_INVALID;
    const int nz = (int)nzd;
    if (zone_off_cap < (uint64_t)nz + 1) return XM_ERR_INVALID;
    int raq_bits, passes;
    xm_raq_layout(nz, &raq_bits, &passes);
    if (passes > kMaxPasses) return XM_ERR_INVALID;
    DeviceGuard dg(device);
    if (!dg.ok) return XM_ERR_CUDA;
    // one-time set-up per device: device address of the scratch array
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[device]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return XM_ERR_CUDA;
            }
            g_noalloc_ptr[device] = p;
        }
        base = g_noalloc_ptr[device];
    }
    int sm_count = 0;
    if (cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return XM_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    char *w = (char *)base;
    unsigned long long *k0 = (unsigned long long *)w; w += kNaKeys;
    unsigned long long *k1 = (unsigned long long *)w; w += kNaKeys;
    uint32_t *v0 = (uint32_t *)w; w += kNaVals;
    uint32_t *v1 = (uint32_t *)w; w += kNaVals;
    uint32_t *tcnt = (uint32_t *)w; w += kNaCnt;
    uint32_t *toff = (uint32_t *)w; w += kNaCnt;
    void *scan_tmp = w; w += kNaScan;
    uint32_t *hist = (uint32_t *)w;
    uint32_t *misc = hist + kMaxPasses * 256;
    const uint32_t n_tiles = (uint32_t)((std::max<uint64_t>(n, 1) + kTile - 1) / kTile);
    // the scratch keeps the previous call's contents: clear what accumulates
    if (cudaMemsetAsync(hist, 0, kMaxPasses * 256 * 4 + 64, st) != cudaSuccess ||
        cudaMemsetAsync(misc, 0xFF, 4, st) != cudaSuccess)
        return XM_ERR_CUDA;
    KeyParams kp{zh_deg, nz, 32 - raq_bits, raq_bits, passes};
    if (n > 0) zb_keys<<<grid_for(n, 256, sm_count, 4), 256, 0, st>>>(objs, n, kp, k0, v0, hist, misc);
    uint32_t h[kMaxPasses * 256 + 16];
    if (cudaMemcpyAsync(h, hist, sizeof(uint32_t) * (kMaxPasses * 256 + 16), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return XM_ERR_CUDA;
    const uint64_t dropped = n ? h[kMaxPasses * 256 + 2] : 0;
    const size_t ds_smem = (size_t)kTile * 12 + (size_t)kRsWarps * 256 * 4 + 512 * 4;
    if (cudaFuncSetAttribute(rs_downsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ds_smem) != cudaSuccess)
        return XM_ERR_CUDA;
    unsigned long long *kin = k0, *kout = k1;
    uint32_t *vin = v0, *vout = v1;
    for (int p = 0; p < passes && n > 0; ++p) {
        bool constant = false;
        for (int d = 0; d < 256; ++d)
            if (h[p * 256 + d] == n) constant = true;
        if (constant) continue;
        rs_upsweep<<<n_tiles, kRsThreads, 0, st>>>(kin, n, 8 * p, n_tiles, tcnt);
        if (xm_scan_exclusive_u32(tcnt, toff, (size_t)n_tiles * 256, scan_tmp, st) != cudaSuccess) return XM_ERR_CUDA;
        rs_downsweep<<<n_tiles, kRsThreads, ds_smem, st>>>(kin, vin, n, 8 * p, n_tiles, toff, kout, vout);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    const uint64_t kept = n - dropped;
    if (kept > 0)
        zb_gather<<<grid_for(kept, 256, sm_count, 8), 256, 0, st>>>(kin, vin, objs, kept, (1ull << raq_bits) - 1,
                                                                    (long long *)out_id, (double2 *)out_radec,
                                                                    (float4 *)out_xyz);
    if (cudaMemsetAsync(out_zone_off, 0xFF, ((size_t)nz + 1) * 4, st) != cudaSuccess) return XM_ERR_CUDA;
    if (n > 0) zb_bounds_mark<<<grid_for(n, 256, sm_count, 8), 256, 0, st>>>(kin, n, raq_bits, nz, out_zone_off);
    zb_bounds_fill<<<grid_for((uint64_t)nz + 1, 256, sm_count, 8), 256, 0, st>>>(kin, n, raq_bits, nz, out_zone_off);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) return XM_ERR_CUDA;
    *n_kept = kept;
    return XM_OK;
}
