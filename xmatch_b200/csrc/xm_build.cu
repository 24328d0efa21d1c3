// xm_build.cu -- device zone builder (replaces Sorter::Sort, Sorter.cu:141-185).
//
// Input: n records {int64 id, f64 ra_deg, f64 dec_deg} in device memory.
// Records with a zone outside [0, n_zones) or a non-finite ra are dropped
// (a non-finite ra can never pass the RA cut of Worker.cu:89-110).
// Output (per segment, sorted by (zone, ra, input index)):
//   zone_off[n_zones + 1]  first object of each zone (zone_off[z+1] = end)
//   id[n]                  int64
//   radec[n]               double2 radians, deg / RAD2DEG (Sorter.cu:52-62)
//   xyz[n]                 float4 (FP32 unit vector, w = zone id bits)
//
// Passes:
//   1. zb_count    zone of every record, histogram (warp-aggregated atomics)
//   2. scan        histogram -> zone offsets
//   3. zb_scatter  32-byte staging record into its zone's slice
//   4. zb_sort_chunks  zone-aligned chunks of <= kSmemCap records sorted by
//                  (zone, ra, index) in shared memory (bitonic network), then
//                  the SoA written in sorted order with unit vectors computed
//   5. oversize chunks (a zone larger than the chunk target; only for dense
//      or degenerate catalogs): runs sorted in shared memory, merged pairwise
//      in global memory, then written like pass 4.
#include <algorithm>
#include <vector>

#include "xm_internal.h"
#include "xm_math.cuh"

namespace {

constexpr int kChunkTarget = 1536;   // records per sort chunk (zone aligned)
constexpr int kSmemCap = 4096;       // largest chunk sorted in shared memory
constexpr int kSortThreads = 512;

struct StageRec {          // 32 bytes: one full sector per scattered write
    double ra_deg;
    double dec_deg;
    long long id;
    unsigned zone;
    unsigned idx;
};
static_assert(sizeof(StageRec) == 32, "staging record must be 32 bytes");

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void zb_count(const xm_obj *__restrict__ objs, unsigned long long n, double zh_deg,
                         int n_zones, uint32_t *__restrict__ cnt)
{
    __shared__ unsigned s_lo, s_hi;
    if (threadIdx.x == 0) {
        s_lo = 0xFFFFFFFFu;
        s_hi = 0u;
    }
    __syncthreads();
    const unsigned lane = threadIdx.x & 31;
    unsigned zlo = 0xFFFFFFFFu, zhi = 0u;   // populated zone range seen by this thread
    unsigned long long warp0 = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull;
    unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = warp0; base < n; base += stride) {
        unsigned long long i = base + lane;
        int bin = -1;
        if (i < n) {
            const xm_obj o = objs[i];
            int z = isfinite(o.ra_deg) ? xm::zone_of(o.dec_deg, zh_deg, n_zones) : -1;
            bin = z < 0 ? n_zones : z;
            if (z >= 0) {
                zlo = min(zlo, (unsigned)z);
                zhi = max(zhi, (unsigned)z);
            }
        }
        unsigned peers = __match_any_sync(0xffffffffu, bin);
        if (bin >= 0 && lane == (unsigned)(__ffs(peers) - 1)) atomicAdd(&cnt[bin], (uint32_t)__popc(peers));
    }
    zlo = __reduce_min_sync(0xffffffffu, zlo);
    zhi = __reduce_max_sync(0xffffffffu, zhi);
    if (lane == 0) {
        atomicMin(&s_lo, zlo);
        atomicMax(&s_hi, zhi);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_lo != 0xFFFFFFFFu) atomicMin(&cnt[n_zones + 2], s_lo);
        atomicMax(&cnt[n_zones + 3], s_hi);
    }
}

__global__ void zb_scatter(const xm_obj *__restrict__ objs, unsigned long long n, double zh_deg,
                           int n_zones, const uint32_t *__restrict__ zone_off,
                           uint32_t *__restrict__ cursor, StageRec *__restrict__ stage)
{
    const unsigned lane = threadIdx.x & 31;
    unsigned long long warp0 = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull;
    unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = warp0; base < n; base += stride) {
        unsigned long long i = base + lane;
        int z = -1;
        xm_obj o;
        if (i < n) {
            o = objs[i];
            z = isfinite(o.ra_deg) ? xm::zone_of(o.dec_deg, zh_deg, n_zones) : -1;
        }
        unsigned peers = __match_any_sync(0xffffffffu, z);
        int leader = __ffs(peers) - 1;
        uint32_t slot = 0;
        if (z >= 0 && (int)lane == leader) slot = atomicAdd(&cursor[z], (uint32_t)__popc(peers));
        slot = __shfl_sync(0xffffffffu, slot, leader);
        if (z >= 0) {
            uint32_t pos = zone_off[z] + slot + __popc(peers & lanemask_lt());
            StageRec r;
            r.ra_deg = o.ra_deg;
            r.dec_deg = o.dec_deg;
            r.id = o.id;
            r.zone = (unsigned)z;
            r.idx = (unsigned)i;
            stage[pos] = r;
        }
    }
}

// Chunk c starts at the first zone whose offset is >= c * kChunkTarget.
__device__ __forceinline__ uint32_t chunk_start(const uint32_t *zone_off, int n_zones, unsigned long long c)
{
    unsigned long long target = c * (unsigned long long)kChunkTarget;
    uint32_t total = zone_off[n_zones];
    if (target >= total) return total;
    int lo = 0, hi = n_zones;  // first z in [0, n_zones] with zone_off[z] >= target
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (zone_off[mid] < target) lo = mid + 1; else hi = mid;
    }
    return zone_off[lo];
}

struct SortKey {
    unsigned long long a, b;   // (zone, ra key high) , (ra key low, input index)
};

__device__ __forceinline__ SortKey make_key(const StageRec &r)
{
    unsigned long long k = xm::order_key(__dadd_rn(r.ra_deg, 0.0));   // -0.0 sorts as +0.0
    SortKey s;
    s.a = ((unsigned long long)r.zone << 32) | (k >> 32);
    s.b = (k << 32) | (unsigned long long)r.idx;
    return s;
}

__device__ __forceinline__ bool key_gt(const SortKey &x, const SortKey &y)
{
    return x.a > y.a || (x.a == y.a && x.b > y.b);
}

__device__ __forceinline__ bool key_lt(const SortKey &x, const SortKey &y)
{
    return x.a < y.a || (x.a == y.a && x.b < y.b);
}

// Bitonic sort of P (power of two) keys with payload in shared memory.
__device__ void smem_bitonic(SortKey *key, uint32_t *pay, int P)
{
    for (int k = 2; k <= P; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                int ixj = i ^ j;
                if (ixj > i) {
                    SortKey ki = key[i], kj = key[ixj];
                    bool up = (i & k) == 0;
                    if (up ? key_gt(ki, kj) : key_lt(ki, kj)) {
                        key[i] = kj;
                        key[ixj] = ki;
                        uint32_t t = pay[i];
                        pay[i] = pay[ixj];
                        pay[ixj] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ void write_sorted(const StageRec &r, uint32_t o, long long *__restrict__ id,
                                             double2 *__restrict__ radec, float4 *__restrict__ xyz)
{
    double ra = __ddiv_rn(r.ra_deg, XM_RAD2DEG);
    double dec = __ddiv_rn(r.dec_deg, XM_RAD2DEG);
    double x, y, z;
    xm::radec2xyz(ra, dec, x, y, z);
    id[o] = r.id;
    radec[o] = make_double2(ra, dec);
    xyz[o] = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z),
                         __uint_as_float(r.zone));
}

__global__ void __launch_bounds__(kSortThreads)
zb_sort_chunks(const StageRec *__restrict__ stage, const uint32_t *__restrict__ zone_off, int n_zones,
               long long *__restrict__ id, double2 *__restrict__ radec, float4 *__restrict__ xyz,
               uint32_t *__restrict__ big, uint32_t big_cap)
{
    extern __shared__ __align__(16) unsigned char smem[];
    SortKey *key = (SortKey *)smem;
    uint32_t *pay = (uint32_t *)(key + kSmemCap);
    __shared__ uint32_t s_range[2];
    if (threadIdx.x == 0) {
        s_range[0] = chunk_start(zone_off, n_zones, blockIdx.x);
        s_range[1] = chunk_start(zone_off, n_zones, (unsigned long long)blockIdx.x + 1);
    }
    __syncthreads();
    const uint32_t s = s_range[0], m = s_range[1] - s_range[0];
    if (m == 0) return;
    if (m > (uint32_t)kSmemCap) {
        if (threadIdx.x == 0) {
            uint32_t k = atomicAdd(&big[0], 1u);
            if (k < big_cap) big[1 + k] = blockIdx.x;
        }
        return;
    }
    int P = 1;
    while (P < (int)m) P <<= 1;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        if (i < (int)m) {
            key[i] = make_key(stage[s + i]);
            pay[i] = (uint32_t)i;
        } else {
            key[i].a = ~0ull;
            key[i].b = ~0ull;
            pay[i] = 0;
        }
    }
    __syncthreads();
    smem_bitonic(key, pay, P);
    for (int j = threadIdx.x; j < (int)m; j += blockDim.x) write_sorted(stage[s + pay[j]], s + j, id, radec, xyz);
}

// ---- oversize chunks ----
// Elements of oversize chunks live in a compact "big space" q in [0, M).
// Chunk k covers q in [boff[k], boff[k+1]) and stage positions starting at bstart[k].
__device__ __forceinline__ int find_chunk(const uint32_t *boff, int nb, uint32_t q)
{
    int lo = 0, hi = nb;  // last k with boff[k] <= q
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (boff[mid] <= q) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void zb_big_load(const StageRec *__restrict__ stage, const uint32_t *__restrict__ boff,
                            const uint32_t *__restrict__ bstart, int nb, uint32_t M,
                            SortKey *__restrict__ K, uint32_t *__restrict__ G)
{
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        int k = find_chunk(boff, nb, q);
        uint32_t g = bstart[k] + (q - boff[k]);
        K[q] = make_key(stage[g]);
        G[q] = g;
    }
}

// Sort runs of kSmemCap consecutive big-space elements (runs never cross chunks:
// run r of chunk k starts at boff[k] + r * kSmemCap).
__global__ void __launch_bounds__(kSortThreads)
zb_big_runs(SortKey *__restrict__ K, uint32_t *__restrict__ G, const uint32_t *__restrict__ run_q,
            const uint32_t *__restrict__ run_len)
{
    extern __shared__ __align__(16) unsigned char smem[];
    SortKey *key = (SortKey *)smem;
    uint32_t *pay = (uint32_t *)(key + kSmemCap);
    const uint32_t q0 = run_q[blockIdx.x], m = run_len[blockIdx.x];
    int P = 1;
    while (P < (int)m) P <<= 1;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        if (i < (int)m) {
            key[i] = K[q0 + i];
            pay[i] = G[q0 + i];
        } else {
            key[i].a = ~0ull;
            key[i].b = ~0ull;
            pay[i] = 0;
        }
    }
    __syncthreads();
    smem_bitonic(key, pay, P);
    for (int i = threadIdx.x; i < (int)m; i += blockDim.x) {
        K[q0 + i] = key[i];
        G[q0 + i] = pay[i];
    }
}

// One merge round: sorted runs of width w inside each chunk are merged pairwise.
__global__ void zb_big_merge(const SortKey *__restrict__ Kin, const uint32_t *__restrict__ Gin,
                             SortKey *__restrict__ Kout, uint32_t *__restrict__ Gout,
                             const uint32_t *__restrict__ boff, int nb, uint32_t M, uint32_t w)
{
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        int k = find_chunk(boff, nb, q);
        uint32_t base = boff[k], L = boff[k + 1] - base, p = q - base;
        uint32_t r = p / w, partner = r ^ 1u;
        uint64_t ps = (uint64_t)partner * w;
        SortKey key = Kin[q];
        uint32_t newp;
        if (ps >= L) {
            newp = p;
        } else {
            uint64_t pe64 = ps + w;
            if (pe64 > L) pe64 = L;
            uint32_t pe = (uint32_t)pe64;
            uint32_t lo = (uint32_t)ps, hi = pe;
            if ((r & 1u) == 0) {   // left run: count partner keys < key
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (key_lt(Kin[base + mid], key)) lo = mid + 1; else hi = mid;
                }
            } else {               // right run: count partner keys <= key
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (!key_gt(Kin[base + mid], key)) lo = mid + 1; else hi = mid;
                }
            }
            uint32_t rank = lo - (uint32_t)ps;
            uint32_t first = min(r, partner) * w;
            newp = first + (p - r * w) + rank;
        }
        Kout[base + newp] = key;
        Gout[base + newp] = Gin[q];
    }
}

__global__ void zb_big_write(const StageRec *__restrict__ stage, const uint32_t *__restrict__ G,
                             const uint32_t *__restrict__ boff, const uint32_t *__restrict__ bstart,
                             int nb, uint32_t M, long long *__restrict__ id, double2 *__restrict__ radec,
                             float4 *__restrict__ xyz)
{
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        int k = find_chunk(boff, nb, q);
        uint32_t o = bstart[k] + (q - boff[k]);
        write_sorted(stage[G[q]], o, id, radec, xyz);
    }
}

int grid_for(unsigned long long n, int threads, int sm_count)
{
    unsigned long long blocks = (n + threads - 1) / threads;
    unsigned long long cap = (unsigned long long)sm_count * 8;
    if (blocks > cap) blocks = cap;
    return (int)std::max<unsigned long long>(blocks, 1);
}

}  // namespace

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

// Host driver of the oversize-chunk path.
static xm_status build_big(xm_segment *seg, const StageRec *stage, const std::vector<uint32_t> &chunks,
                           uint32_t *n_launch)
{
    xm_ctx *ctx = seg->ctx;
    cudaStream_t st = ctx->stream;
    const int nc = (int)chunks.size();
    // chunk ranges from the zone offsets (host copy of the needed entries)
    std::vector<uint32_t> zoff((size_t)seg->n_zones + 1);
    XM_CUDA(ctx, cudaMemcpyAsync(zoff.data(), seg->zone_off, zoff.size() * 4, cudaMemcpyDeviceToHost, st));
    XM_CUDA(ctx, cudaStreamSynchronize(st));
    auto cstart = [&](uint64_t c) -> uint32_t {
        uint64_t target = c * (uint64_t)kChunkTarget;
        uint32_t total = zoff[seg->n_zones];
        if (target >= total) return total;
        auto it = std::lower_bound(zoff.begin(), zoff.end(), (uint32_t)target);
        return *it;
    };
    std::vector<uint32_t> sorted(chunks);
    std::sort(sorted.begin(), sorted.end());
    std::vector<uint32_t> boff(nc + 1), bstart(nc), run_q, run_len;
    uint32_t M = 0, maxlen = 0;
    for (int k = 0; k < nc; ++k) {
        uint32_t s = cstart(sorted[k]), e = cstart((uint64_t)sorted[k] + 1);
        bstart[k] = s;
        boff[k] = M;
        uint32_t L = e - s;
        for (uint32_t r = 0; r < L; r += kSmemCap) {
            run_q.push_back(M + r);
            run_len.push_back(std::min<uint32_t>(kSmemCap, L - r));
        }
        M += L;
        maxlen = std::max(maxlen, L);
    }
    boff[nc] = M;
    size_t bytes = (size_t)M * (2 * sizeof(SortKey) + 2 * sizeof(uint32_t)) + (boff.size() + bstart.size() +
                   2 * run_q.size()) * 4 + 64;
    void *buf = nullptr;
    XM_TRY(xm_dev_alloc(ctx, &buf, bytes));
    char *p = (char *)buf;
    SortKey *K0 = (SortKey *)p; p += (size_t)M * sizeof(SortKey);
    SortKey *K1 = (SortKey *)p; p += (size_t)M * sizeof(SortKey);
    uint32_t *G0 = (uint32_t *)p; p += (size_t)M * 4;
    uint32_t *G1 = (uint32_t *)p; p += (size_t)M * 4;
    uint32_t *d_boff = (uint32_t *)p; p += boff.size() * 4;
    uint32_t *d_bstart = (uint32_t *)p; p += bstart.size() * 4;
    uint32_t *d_runq = (uint32_t *)p; p += run_q.size() * 4;
    uint32_t *d_runl = (uint32_t *)p;
    xm_status rc = XM_OK;
    do {
        if (cudaMemcpyAsync(d_boff, boff.data(), boff.size() * 4, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(d_bstart, bstart.data(), bstart.size() * 4, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(d_runq, run_q.data(), run_q.size() * 4, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(d_runl, run_len.data(), run_len.size() * 4, cudaMemcpyHostToDevice, st)) {
            rc = XM_ERR_CUDA;
            break;
        }
        int g = grid_for(M, 256, ctx->sm_count);
        zb_big_load<<<g, 256, 0, st>>>(stage, d_boff, d_bstart, nc, M, K0, G0);
        size_t smem = (size_t)kSmemCap * (sizeof(SortKey) + 4);
        zb_big_runs<<<(unsigned)run_q.size(), kSortThreads, smem, st>>>(K0, G0, d_runq, d_runl);
        *n_launch += 2;
        for (uint32_t w = kSmemCap; w < maxlen; w *= 2) {
            zb_big_merge<<<g, 256, 0, st>>>(K0, G0, K1, G1, d_boff, nc, M, w);
            std::swap(K0, K1);
            std::swap(G0, G1);
            *n_launch += 1;
        }
        zb_big_write<<<g, 256, 0, st>>>(stage, G0, d_boff, d_bstart, nc, M, (long long *)seg->id, seg->radec,
                                        seg->xyz);
        *n_launch += 1;
        if (cudaGetLastError() != cudaSuccess) rc = XM_ERR_CUDA;
    } while (0);
    cudaStreamSynchronize(st);
    xm_dev_free(ctx, buf);
    if (rc != XM_OK) ctx->last_error = "oversize-zone sort failed";
    return rc;
}

xm_status xm_build_impl(xm_segment *seg, const xm_obj *objs, uint64_t n, xm_stats *stats)
{
    xm_ctx *ctx = seg->ctx;
    cudaStream_t st = ctx->stream;
    if (n >= 0xFFFFFFF0ull) {
        ctx->last_error = "segment larger than 2^32-16 records";
        return XM_ERR_INVALID;
    }
    const int nz = seg->n_zones;
    uint32_t launches = 0;
    // storage
    if (seg->cap < n || !seg->id) {
        xm_dev_free(ctx, seg->id);
        xm_dev_free(ctx, seg->radec);
        xm_dev_free(ctx, seg->xyz);
        seg->id = nullptr; seg->radec = nullptr; seg->xyz = nullptr;
        seg->cap = 0;
        uint64_t c = std::max<uint64_t>(n, 1);
        XM_TRY(xm_dev_alloc(ctx, (void **)&seg->id, (c + 2) * sizeof(int64_t)));
        XM_TRY(xm_dev_alloc(ctx, (void **)&seg->radec, c * sizeof(double2)));
        XM_TRY(xm_dev_alloc(ctx, (void **)&seg->xyz, c * sizeof(float4)));
        seg->cap = c;
    }
    if (!seg->zone_off) {
        XM_TRY(xm_dev_alloc(ctx, (void **)&seg->zone_off, ((size_t)nz + 8) * 4));
        XM_CUDA(ctx, cudaMemsetAsync(seg->zone_off, 0, ((size_t)nz + 8) * 4, st));
    }
    if (!seg->cnt) XM_TRY(xm_dev_alloc(ctx, (void **)&seg->cnt, ((size_t)nz + 4) * 4));
    XM_TRY(ensure(ctx, &seg->tmp, &seg->tmp_bytes, std::max<uint64_t>(n, 1) * sizeof(StageRec)));
    XM_TRY(ensure(ctx, &seg->scan_tmp, &seg->scan_tmp_bytes, xm_scan_tmp_bytes((size_t)nz)));
    const uint32_t big_cap = 4096;
    if (!seg->big) {
        XM_TRY(xm_dev_alloc(ctx, (void **)&seg->big, (big_cap + 1) * 4));
        seg->big_cap = big_cap;
    }
    StageRec *stage = (StageRec *)seg->tmp;

    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[0], st));
    XM_CUDA(ctx, cudaMemsetAsync(seg->cnt, 0, ((size_t)nz + 4) * 4, st));
    XM_CUDA(ctx, cudaMemsetAsync(seg->cnt + nz + 2, 0xFF, 4, st));
    XM_CUDA(ctx, cudaMemsetAsync(seg->big, 0, 4, st));
    const int threads = 256;
    int g = grid_for(n, threads, ctx->sm_count);
    if (n > 0) {
        zb_count<<<g, threads, 0, st>>>(objs, n, seg->zh_deg, nz, seg->cnt);
        launches++;
    }
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[8], st));
    XM_CUDA(ctx, xm_scan_exclusive_u32(seg->cnt, seg->zone_off, (size_t)nz, seg->scan_tmp, st));
    launches += 3;
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[9], st));
    // dropped count travels with the offsets: zone_off[nz + 1] = cnt[nz]
    XM_CUDA(ctx, cudaMemcpyAsync(seg->zone_off + nz + 1, seg->cnt + nz, 4, cudaMemcpyDeviceToDevice, st));
    XM_CUDA(ctx, cudaMemsetAsync(seg->cnt, 0, (size_t)nz * 4, st));
    if (n > 0) {
        zb_scatter<<<g, threads, 0, st>>>(objs, n, seg->zh_deg, nz, seg->zone_off, seg->cnt, stage);
        launches++;
        if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[10], st));
        unsigned long long n_chunks = (n + kChunkTarget - 1) / kChunkTarget;
        size_t smem = (size_t)kSmemCap * (sizeof(SortKey) + 4);
        static bool attr_set = false;
        if (!attr_set) {
            cudaFuncSetAttribute(zb_sort_chunks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            cudaFuncSetAttribute(zb_big_runs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            attr_set = true;
        }
        zb_sort_chunks<<<(unsigned)n_chunks, kSortThreads, smem, st>>>(stage, seg->zone_off, nz, (long long *)seg->id,
                                                                      seg->radec, seg->xyz, seg->big, big_cap);
        launches++;
        XM_CUDA(ctx, cudaGetLastError());
        if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[11], st));
    }
    // kept / dropped counts and the oversize list
    uint32_t h[5];
    XM_CUDA(ctx, cudaMemcpyAsync(&h[0], seg->zone_off + nz, 8, cudaMemcpyDeviceToHost, st));
    XM_CUDA(ctx, cudaMemcpyAsync(&h[2], seg->big, 4, cudaMemcpyDeviceToHost, st));
    XM_CUDA(ctx, cudaMemcpyAsync(&h[3], seg->cnt + nz + 2, 8, cudaMemcpyDeviceToHost, st));
    XM_CUDA(ctx, cudaStreamSynchronize(st));
    seg->n = h[0];
    seg->n_in = n;
    if (seg->n > 0) {
        seg->z_lo = (int32_t)h[3];
        seg->z_hi = (int32_t)h[4];
    } else {
        seg->z_lo = 0;
        seg->z_hi = -1;
    }
    if (h[2] > 0) {
        uint32_t nbig = h[2];
        std::vector<uint32_t> chunks;
        if (nbig <= big_cap) {
            chunks.resize(nbig);
            XM_CUDA(ctx, cudaMemcpy(chunks.data(), seg->big + 1, nbig * 4, cudaMemcpyDeviceToHost));
        } else {
            // more oversize chunks than the list holds: recompute them on the host
            std::vector<uint32_t> zoff((size_t)nz + 1);
            XM_CUDA(ctx, cudaMemcpy(zoff.data(), seg->zone_off, zoff.size() * 4, cudaMemcpyDeviceToHost));
            auto cstart = [&](uint64_t c) -> uint32_t {
                uint64_t target = c * (uint64_t)kChunkTarget;
                if (target >= zoff[nz]) return zoff[nz];
                return *std::lower_bound(zoff.begin(), zoff.end(), (uint32_t)target);
            };
            uint64_t n_chunks = (n + kChunkTarget - 1) / kChunkTarget;
            for (uint64_t c = 0; c < n_chunks; ++c)
                if (cstart(c + 1) - cstart(c) > (uint32_t)kSmemCap) chunks.push_back((uint32_t)c);
        }
        XM_TRY(build_big(seg, stage, chunks, &launches));
    }
    if (stats) {
        XM_CUDA(ctx, cudaEventRecord(ctx->ev[1], st));
        XM_CUDA(ctx, cudaEventSynchronize(ctx->ev[1]));
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        stats->ms_build += ms;
        stats->n_launches += launches;
        if (n > 0) {
            float a = 0, b = 0, c = 0, d = 0;
            cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[8]);
            cudaEventElapsedTime(&b, ctx->ev[8], ctx->ev[9]);
            cudaEventElapsedTime(&c, ctx->ev[9], ctx->ev[10]);
            cudaEventElapsedTime(&d, ctx->ev[10], ctx->ev[11]);
            stats->ms_zb_count += a;
            stats->ms_zb_scan += b;
            stats->ms_zb_scatter += c;
            stats->ms_zb_sort += d;
        }
    }
    return XM_OK;
}
