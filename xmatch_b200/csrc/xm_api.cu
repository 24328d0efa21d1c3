// xm_api.cu -- C ABI of libxmatch_b200: contexts, segments, match calls.
//
// Host-side counterpart of the reference's Worker::Match (Worker.cu:243-428)
// and Sorter::Sort (Sorter.cu:141-185): parameters and the per-zone RA
// half-width are computed here with the host libm exactly as the reference
// host code does (Worker.cu:310-317, 349; Common.cu:7-23), the device work is
// queued on the context's stream, and results are copied back only when the
// caller asks for them.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "xm_internal.h"
#include "xm_match.cuh"
#include "xm_math.cuh"

// ---------------------------------------------------------------------------
// RA half-width per zone, Gray, Nieto & Szalay (2007) as written in
// Common.cu:7-23 (including its parenthesisation atan(sin t) / sqrt(...),
// which is never smaller than the exact half-width).  Host libm on purpose:
// the reference evaluates it on the host (Worker.cu:349).
// ---------------------------------------------------------------------------
static double calc_alpha_dec(double theta, double abs_dec)
{
    if (abs_dec + theta > 89.99) return 180;
    return std::fabs(std::atan(std::sin(theta / XM_RAD2DEG)) /
                     std::sqrt(std::fabs(std::cos((abs_dec - theta) / XM_RAD2DEG) *
                                         std::cos((abs_dec + theta) / XM_RAD2DEG))));
}

static double calc_alpha_zone(double theta, double zh_deg, int zone)
{
    double dec = std::fabs(zone * zh_deg - 90);
    double dec2 = std::fabs((zone + 1) * zh_deg - 90);
    dec = (dec > dec2 ? dec : dec2);
    return calc_alpha_dec(theta, dec + 0.01 * theta);
}

void xm_host_alpha_table(double sr_deg, double zh_deg, int32_t n_zones, double *out)
{
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n_zones < 65536) nt = 1;
    auto work = [&](unsigned t) {
        int64_t a = (int64_t)n_zones * t / nt, b = (int64_t)n_zones * (t + 1) / nt;
        for (int64_t z = a; z < b; ++z) out[z] = calc_alpha_zone(sr_deg, zh_deg, (int)z);
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
}

static int32_t zones_for(double zh_deg) { return (int32_t)std::ceil(180 / zh_deg); }   // Sorter.cu:156

static float round_up_f(double v)
{
    float f = (float)v;
    if ((double)f < v) f = std::nextafter(f, INFINITY);
    return f;
}

static float round_down_f(double v)
{
    float f = (float)v;
    if ((double)f > v) f = std::nextafter(f, -INFINITY);
    return f;
}

// Worker.cu:310-317 plus the FP32 margin bounds.
//
// With X the FP64 unit vectors and X~ = fl32(X): |X~_i - X_i| <= 2^-25, so the
// exact differences satisfy ||D~ - D|| <= delta = sqrt(3) 2^-24.  If the FP64
// chord^2 is below T then ||D|| < sqrt(T)(1 + 8u64) = R, and the FP32 value,
// with one rounding of each difference and three in the fused sum of squares,
// is at most H = ((R + delta)(1 + u32))^2 (1 + u32)^3.  A pair whose FP32
// value exceeds H therefore cannot match.
//
// thr_lo is the mirror bound: an FP32 value below it implies ||D|| < sqrt(T)
// (1 - eta) with eta = 2^-20, so the FP64 chord^2 is under T and the angular
// distance theta of the two (FP64) positions is below r (1 - eta) up to a few
// units of 1e-16.  Such a pair also passes the reference's two cuts whenever
// the A zone has an RA cut (alpha < 3 rad, i.e. not the 180-degree sentinel):
// |dec_a - dec_b| <= theta < r, and the RA offset of a point within theta is at
// most the exact half-width of a cap of radius theta at |dec_a|, which is below
// the zone's alpha (computed for radius r at the zone's largest |dec| plus
// 0.01 r, and never below the exact half-width) by at least (r - theta).  Both
// margins, about r eta, dwarf the FP64 rounding of the cut arithmetic (below
// 64 u64 2 pi) once r eta exceeds that; for smaller radii thr_lo is 0 and every
// pair under thr_hi is decided by the full FP64 predicate.
xm_status xm_make_params(double sr_deg, double zh_deg, xm_match_params *p)
{
    if (!(sr_deg > 0) || !(zh_deg > 0) || !std::isfinite(sr_deg) || !std::isfinite(zh_deg)) return XM_ERR_INVALID;
    p->sr_deg = sr_deg;
    p->nz = (int32_t)std::ceil(sr_deg / zh_deg);
    p->sr_rad = sr_deg / XM_RAD2DEG;
    double d = 2.0 * std::sin(p->sr_rad / 2.0);
    p->sr_dist2 = d * d;
    const double u32 = std::ldexp(1.0, -24), u64 = std::ldexp(1.0, -53);
    const double delta = std::sqrt(3.0) * std::ldexp(1.0, -24) * (1 + 1e-6);
    const double rt = std::sqrt(p->sr_dist2);
    double R = rt * (1 + 8 * u64);
    double H = (R + delta) * (1 + u32);
    H = H * H * std::pow(1 + u32, 3) * (1 + 1e-6);
    p->thr_hi = round_up_f(H);
    const double eta = std::ldexp(1.0, -20);
    double Rl = rt * (1 - eta) - delta;
    double L = 0;
    if (Rl > 0 && p->sr_rad * eta > 64 * u64 * XM_TWO_PI) {
        L = Rl * (1 - u32);
        L = L * L * std::pow(1 - u32, 3) * (1 - 1e-6);
    }
    p->thr_lo = round_down_f(L);
    return XM_OK;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
xm_status xm_dev_alloc(xm_ctx *ctx, void **p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->last_error = std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
                          cudaGetErrorString(e);
        *p = nullptr;
        return XM_ERR_NOMEM;
    }
    return XM_OK;
}

xm_status xm_dev_alloc_on(xm_ctx *ctx, void **p, size_t bytes, cudaStream_t st)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->last_error = std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " +
                          cudaGetErrorString(e);
        *p = nullptr;
        return XM_ERR_NOMEM;
    }
    return XM_OK;
}

void xm_dev_free(xm_ctx *ctx, void *p)
{
    if (p) cudaFreeAsync(p, ctx->stream);
}

extern "C" const char *xm_status_str(xm_status s)
{
    switch (s) {
    case XM_OK: return "ok";
    case XM_ERR_INVALID: return "invalid argument";
    case XM_ERR_CUDA: return "CUDA error";
    case XM_ERR_NOMEM: return "out of memory";
    case XM_ERR_CAPACITY: return "output buffer too small";
    case XM_ERR_MISMATCH: return "segments have different zone heights";
    case XM_ERR_NODEVICE: return "no CUDA device";
    case XM_ERR_IO: return "I/O error";
    case XM_ERR_BUSY: return "busy";
    case XM_ERR_TIMEOUT: return "timed out";
    case XM_ERR_TOO_LARGE: return "input exceeds the fixed capacity of the call";
    default: return "unknown status";
    }
}

extern "C" const char *xm_last_error(const xm_ctx *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

extern "C" xm_status xm_ctx_create(int device, xm_ctx **out)
{
    if (!out) return XM_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return XM_ERR_NODEVICE;
    }
    if (device < 0 || device >= n) return XM_ERR_INVALID;
    xm_ctx *ctx = new xm_ctx();
    ctx->device = device;
    auto fail = [&](cudaError_t e) {
        ctx->last_error = cudaGetErrorString(e);
        delete ctx;
        return XM_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(e);
    if ((e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return fail(e);
    if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaStreamCreateWithFlags(&ctx->stream2, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreate(&ctx->ev_b2)) != cudaSuccess) return fail(e);
    for (auto &ev : ctx->ev_slot)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if ((e = cudaMemPoolCreate(&ctx->pool, &props)) != cudaSuccess) return fail(e);
    uint64_t thr = UINT64_MAX;   // keep freed blocks for reuse by this context
    cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    for (auto &ev : ctx->ev)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&ctx->counters, 16 * sizeof(unsigned long long))) != cudaSuccess) return fail(e);
    if ((e = cudaMallocHost(&ctx->h_counters, 16 * sizeof(unsigned long long))) != cudaSuccess) return fail(e);
    if ((e = cudaMallocHost(&ctx->h_tiles, 2 * sizeof(uint32_t))) != cudaSuccess) return fail(e);
    *out = ctx;
    return XM_OK;
}

static void free_result(xm_ctx *ctx)
{
    xm_dev_free(ctx, ctx->res.pairs);
    xm_dev_free(ctx, ctx->res.dist);
    xm_dev_free(ctx, ctx->res.job);
    xm_dev_free(ctx, ctx->res.pairs_g);
    xm_dev_free(ctx, ctx->res.dist_g);
    ctx->res = xm_result_buf();
}

extern "C" xm_status xm_ctx_destroy(xm_ctx *ctx)
{
    if (!ctx) return XM_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_result(ctx);
    alpha_cache_clear(ctx);
    xm_dev_free(ctx, ctx->d_jobs);
    xm_dev_free(ctx, ctx->d_work);
    xm_dev_free(ctx, ctx->d_plans);
    xm_dev_free(ctx, ctx->build_tmp);
    xm_dev_free(ctx, ctx->stage);
    xm_dev_free(ctx, ctx->stage2);
    cudaStreamSynchronize(ctx->stream);
    if (ctx->stream2) {
        cudaStreamSynchronize(ctx->stream2);
        cudaStreamDestroy(ctx->stream2);
    }
    if (ctx->ev_b2) cudaEventDestroy(ctx->ev_b2);
    for (auto &ev : ctx->ev_slot)
        if (ev) cudaEventDestroy(ev);
    if (ctx->counters) cudaFree(ctx->counters);
    if (ctx->h_counters) cudaFreeHost(ctx->h_counters);
    if (ctx->h_tiles) cudaFreeHost(ctx->h_tiles);
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    for (auto &ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return XM_OK;
}

extern "C" xm_status xm_ctx_info(const xm_ctx *ctx, int *device, int *sm_count, uint64_t *free_bytes,
                                 uint64_t *total_bytes)
{
    if (!ctx) return XM_ERR_INVALID;
    cudaSetDevice(ctx->device);
    size_t f = 0, t = 0;
    cudaMemGetInfo(&f, &t);
    if (device) *device = ctx->device;
    if (sm_count) *sm_count = ctx->sm_count;
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return XM_OK;
}

extern "C" xm_status xm_ctx_stream(const xm_ctx *ctx, void **stream)
{
    if (!ctx || !stream) return XM_ERR_INVALID;
    *stream = (void *)ctx->stream;
    return XM_OK;
}

extern "C" xm_status xm_ctx_synchronize(xm_ctx *ctx)
{
    if (!ctx) return XM_ERR_INVALID;
    XM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return XM_OK;
}

static constexpr size_t kAlphaCacheBytes = 512ull << 20;   // cached tables per context, at most

static xm_alpha_key alpha_key(const xm_alpha_req &r)
{
    xm_alpha_key k;
    std::memcpy(&k.sr, &r.sr_deg, 8);
    std::memcpy(&k.zh, &r.zh_deg, 8);
    k.z0 = r.z0;
    k.z1 = r.z1;
    return k;
}

void alpha_cache_clear(xm_ctx *ctx)
{
    for (auto &kv : ctx->alpha_cache) xm_dev_free(ctx, kv.second.dev);
    ctx->alpha_cache.clear();
    ctx->alpha_bytes = 0;
}

// Tables missing from the cache are computed on the host (libm, as the
// reference does), all of them together over a pool of threads in chunks of
// zones, then copied to the device.
xm_status xm_get_alpha_ranges(xm_ctx *ctx, xm_alpha_req *req, size_t n)
{
    std::vector<xm_alpha_key> miss;
    size_t miss_bytes = 0;
    for (size_t i = 0; i < n; ++i) {
        const xm_alpha_key k = alpha_key(req[i]);
        if (ctx->alpha_cache.count(k)) continue;
        bool dup = false;
        for (size_t j = 0; j < miss.size() && !dup; ++j)   // few misses per call in practice
            dup = !(miss[j] < k) && !(k < miss[j]);
        if (dup) continue;
        miss.push_back(k);
        miss_bytes += (size_t)(k.z1 - k.z0 + 1) * 8;
    }
    if (!miss.empty() && ctx->alpha_bytes + miss_bytes > kAlphaCacheBytes) {
        alpha_cache_clear(ctx);
        miss.clear();
        miss_bytes = 0;
        for (size_t i = 0; i < n; ++i) {
            const xm_alpha_key k = alpha_key(req[i]);
            bool dup = false;
            for (size_t j = 0; j < miss.size() && !dup; ++j) dup = !(miss[j] < k) && !(k < miss[j]);
            if (dup) continue;
            miss.push_back(k);
            miss_bytes += (size_t)(k.z1 - k.z0 + 1) * 8;
        }
    }
    if (!miss.empty()) {
        std::vector<size_t> off(miss.size() + 1, 0);
        for (size_t j = 0; j < miss.size(); ++j) off[j + 1] = off[j] + (size_t)(miss[j].z1 - miss[j].z0 + 1);
        std::vector<double> h(off.back());
        // tasks: (table, first zone) chunks of at most 8192 zones
        struct Task { size_t t; int32_t za, zb; };
        std::vector<Task> tasks;
        for (size_t j = 0; j < miss.size(); ++j)
            for (int64_t z = miss[j].z0; z <= miss[j].z1; z += 8192)
                tasks.push_back({j, (int32_t)z, (int32_t)std::min<int64_t>(z + 8191, miss[j].z1)});
        std::atomic<size_t> next{0};
        auto work = [&]() {
            for (size_t q; (q = next.fetch_add(1)) < tasks.size();) {
                const Task &T = tasks[q];
                double sr, zh;
                std::memcpy(&sr, &miss[T.t].sr, 8);
                std::memcpy(&zh, &miss[T.t].zh, 8);
                double *dst = h.data() + off[T.t] - miss[T.t].z0;
                for (int32_t z = T.za; z <= T.zb; ++z) dst[z] = calc_alpha_zone(sr, zh, z);
            }
        };
        const unsigned nt = (unsigned)std::min<size_t>(tasks.size(),
                                                       std::max(1u, std::min(32u, std::thread::hardware_concurrency())));
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; ++t) th.emplace_back(work);
        work();
        for (auto &x : th) x.join();
        for (size_t j = 0; j < miss.size(); ++j) {
            xm_alpha_entry e;
            e.bytes = (off[j + 1] - off[j] + 2) * 8;   // 2 spare entries: the pair kernel copies in 16-byte units
            XM_TRY(xm_dev_alloc(ctx, (void **)&e.dev, e.bytes));
            XM_CUDA(ctx, cudaMemsetAsync(e.dev, 0, e.bytes, ctx->stream));
            XM_CUDA(ctx, cudaMemcpyAsync(e.dev, h.data() + off[j], (off[j + 1] - off[j]) * 8, cudaMemcpyHostToDevice,
                                         ctx->stream));
            ctx->alpha_cache[miss[j]] = e;
            ctx->alpha_bytes += e.bytes;
        }
        XM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));   // h goes out of scope
    }
    for (size_t i = 0; i < n; ++i) req[i].dev = ctx->alpha_cache.at(alpha_key(req[i])).dev;
    return XM_OK;
}

// ---------------------------------------------------------------------------
// segments
// ---------------------------------------------------------------------------

static xm_status new_segment(xm_ctx *ctx, uint32_t seg_id, double zh_deg, xm_segment **out)
{
    if (!(zh_deg > 0) || !std::isfinite(zh_deg)) return XM_ERR_INVALID;
    double nzd = std::ceil(180 / zh_deg);
    if (nzd > 2.0e9) {
        ctx->last_error = "zone height too small";
        return XM_ERR_INVALID;
    }
    xm_segment *s = new xm_segment();
    s->ctx = ctx;
    s->seg_id = seg_id;
    s->zh_deg = zh_deg;
    s->n_zones = zones_for(zh_deg);
    *out = s;
    return XM_OK;
}

extern "C" xm_status xm_segment_build_device(xm_ctx *ctx, uint32_t seg_id, const xm_obj *dev_objs, uint64_t n,
                                             double zh_deg, xm_segment **out, xm_stats *stats)
{
    if (!ctx || !out || (n && !dev_objs)) return XM_ERR_INVALID;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    xm_segment *s = nullptr;
    XM_TRY(new_segment(ctx, seg_id, zh_deg, &s));
    xm_status rc = xm_build_impl(s, dev_objs, n, stats);
    if (rc != XM_OK) {
        xm_segment_free(s);
        return rc;
    }
    *out = s;
    return XM_OK;
}

extern "C" xm_status xm_segment_rebuild_device(xm_segment *seg, const xm_obj *dev_objs, uint64_t n,
                                               xm_stats *stats)
{
    if (!seg || (n && !dev_objs)) return XM_ERR_INVALID;
    cudaSetDevice(seg->ctx->device);
    return xm_build_impl(seg, dev_objs, n, stats);
}

extern "C" xm_status xm_segment_build(xm_ctx *ctx, uint32_t seg_id, const xm_obj *host_objs, uint64_t n,
                                      double zh_deg, xm_segment **out, xm_stats *stats)
{
    if (!ctx || !out || (n && !host_objs)) return XM_ERR_INVALID;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    xm_segment *s = nullptr;
    XM_TRY(new_segment(ctx, seg_id, zh_deg, &s));
    // host records land in the context's staging buffer (grown, never shrunk)
    xm_status rc = XM_OK;
    const size_t need = std::max<uint64_t>(n, 1) * sizeof(xm_obj);
    if (ctx->stage_bytes < need) {
        xm_dev_free(ctx, ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_bytes = 0;
        rc = xm_dev_alloc(ctx, &ctx->stage, need);
        if (rc == XM_OK) ctx->stage_bytes = need;
    }
    void *d = ctx->stage;
    if (rc == XM_OK && n) {
        if (stats) cudaEventRecord(ctx->ev[12], ctx->stream);
        cudaError_t e = cudaMemcpyAsync(d, host_objs, n * sizeof(xm_obj), cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) {
            ctx->last_error = cudaGetErrorString(e);
            rc = XM_ERR_CUDA;
        }
        if (stats) cudaEventRecord(ctx->ev[13], ctx->stream);
    }
    if (rc == XM_OK) rc = xm_build_impl(s, (const xm_obj *)d, n, stats);
    if (rc == XM_OK && n && stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[12], ctx->ev[13]);   // build_impl synchronised the stream
        stats->ms_h2d += ms;
    }
    if (rc != XM_OK) {
        xm_segment_free(s);
        return rc;
    }
    *out = s;
    return XM_OK;
}

extern "C" xm_status xm_segment_free(xm_segment *seg)
{
    if (!seg) return XM_OK;
    xm_ctx *ctx = seg->ctx;
    cudaSetDevice(ctx->device);
    if (seg->ready_pending) cudaStreamWaitEvent(ctx->stream, seg->ready, 0);
    xm_dev_free(ctx, seg->store);
    if (seg->host_store || seg->ready) {
        cudaStreamSynchronize(ctx->stream2);   // a page-in copy may still read the host copy
        if (seg->host_store) cudaFreeHost(seg->host_store);
        if (seg->ready) cudaEventDestroy(seg->ready);
    }
    delete seg;
    return XM_OK;
}

// ---- segments in host memory (replaces the reference's per-job copies of
// host-resident segments to the GPU, Worker.cu:251-292, for catalogs larger
// than device memory) ----

extern "C" xm_status xm_segment_offload(xm_segment *seg)
{
    if (!seg) return XM_ERR_INVALID;
    xm_ctx *ctx = seg->ctx;
    cudaSetDevice(ctx->device);
    if (!seg->store) return XM_OK;   // already offloaded
    if (seg->ready_pending) XM_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, seg->ready, 0));
    seg->ready_pending = false;
    if (!seg->host_store) {
        if (cudaMallocHost(&seg->host_store, seg->store_bytes) != cudaSuccess) {
            cudaGetLastError();
            seg->host_store = nullptr;
            ctx->last_error = "pinned host allocation of " + std::to_string(seg->store_bytes) + " bytes failed";
            return XM_ERR_NOMEM;
        }
        XM_CUDA(ctx, cudaMemcpyAsync(seg->host_store, seg->store, seg->store_bytes, cudaMemcpyDeviceToHost,
                                     ctx->stream));
        XM_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    xm_dev_free(ctx, seg->store);   // after the work queued on the segment
    seg->store = nullptr;
    xm_seg_layout(seg, nullptr);
    return XM_OK;
}

extern "C" xm_status xm_segment_page_in(xm_segment *seg)
{
    if (!seg) return XM_ERR_INVALID;
    xm_ctx *ctx = seg->ctx;
    cudaSetDevice(ctx->device);
    if (seg->store) return XM_OK;
    if (!seg->host_store) return XM_ERR_INVALID;
    if (!seg->ready) XM_CUDA(ctx, cudaEventCreateWithFlags(&seg->ready, cudaEventDisableTiming));
    void *p = nullptr;
    XM_TRY(xm_dev_alloc_on(ctx, &p, seg->store_bytes, ctx->stream2));
    XM_CUDA(ctx, cudaMemcpyAsync(p, seg->host_store, seg->store_bytes, cudaMemcpyHostToDevice, ctx->stream2));
    XM_CUDA(ctx, cudaEventRecord(seg->ready, ctx->stream2));
    seg->ready_pending = true;
    seg->store = p;
    xm_seg_layout(seg, p);
    return XM_OK;
}

extern "C" xm_status xm_segment_page_out(xm_segment *seg)
{
    if (!seg) return XM_ERR_INVALID;
    if (!seg->store) return XM_OK;
    if (!seg->host_store) return xm_segment_offload(seg);
    xm_ctx *ctx = seg->ctx;
    cudaSetDevice(ctx->device);
    if (seg->ready_pending) XM_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, seg->ready, 0));
    seg->ready_pending = false;
    xm_dev_free(ctx, seg->store);   // stream-ordered after the work queued on the segment
    seg->store = nullptr;
    xm_seg_layout(seg, nullptr);
    return XM_OK;
}

extern "C" xm_status xm_segment_resident(const xm_segment *seg, int *on_device, uint64_t *bytes)
{
    if (!seg) return XM_ERR_INVALID;
    if (on_device) *on_device = seg->store != nullptr;
    if (bytes) *bytes = seg->store_bytes;
    return XM_OK;
}

extern "C" xm_status xm_segment_info(const xm_segment *seg, uint32_t *seg_id, uint64_t *n_kept, int32_t *n_zones,
                                     double *zh_deg)
{
    if (!seg) return XM_ERR_INVALID;
    if (seg_id) *seg_id = seg->seg_id;
    if (n_kept) *n_kept = seg->n;
    if (n_zones) *n_zones = seg->n_zones;
    if (zh_deg) *zh_deg = seg->zh_deg;
    return XM_OK;
}

extern "C" xm_status xm_segment_export(const xm_segment *seg, int64_t *id, double *radec, int32_t *zone_begin,
                                       int32_t *zone_end)
{
    if (!seg) return XM_ERR_INVALID;
    xm_ctx *ctx = seg->ctx;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    if (!seg->store && !seg->host_store) return XM_ERR_INVALID;
    if (seg->ready_pending) XM_CUDA(ctx, cudaStreamWaitEvent(st, seg->ready, 0));
    // the device arrays, or the host copy of an offloaded segment
    const char *base = seg->store ? (const char *)seg->store : (const char *)seg->host_store;
    const void *s_id = base + seg->off_id, *s_radec = base + seg->off_radec, *s_zoff = base;
    if (id && seg->n) XM_CUDA(ctx, cudaMemcpyAsync(id, s_id, seg->n * 8, cudaMemcpyDefault, st));
    if (radec && seg->n) XM_CUDA(ctx, cudaMemcpyAsync(radec, s_radec, seg->n * 16, cudaMemcpyDefault, st));
    if (zone_begin || zone_end) {
        std::vector<uint32_t> z((size_t)seg->n_zones + 1);
        XM_CUDA(ctx, cudaMemcpyAsync(z.data(), s_zoff, z.size() * 4, cudaMemcpyDefault, st));
        XM_CUDA(ctx, cudaStreamSynchronize(st));
        for (int32_t k = 0; k < seg->n_zones; ++k) {
            if (zone_begin) zone_begin[k] = (int32_t)z[k];
            if (zone_end) zone_end[k] = (int32_t)z[k + 1];
        }
    }
    XM_CUDA(ctx, cudaStreamSynchronize(st));
    return XM_OK;
}

// ---------------------------------------------------------------------------
// matching
// ---------------------------------------------------------------------------
namespace {

xm_status ensure_result(xm_ctx *ctx, uint64_t cap, bool want_job)
{
    xm_result_buf &r = ctx->res;
    if (r.cap >= cap && r.pairs && (!want_job || r.job)) return XM_OK;
    uint64_t c = std::max<uint64_t>(cap, r.cap);
    xm_dev_free(ctx, r.pairs);
    xm_dev_free(ctx, r.dist);
    xm_dev_free(ctx, r.job);
    r.pairs = nullptr; r.dist = nullptr; r.job = nullptr; r.cap = 0;
    XM_TRY(xm_dev_alloc(ctx, (void **)&r.pairs, c * 16));
    XM_TRY(xm_dev_alloc(ctx, (void **)&r.dist, c * 8));
    XM_TRY(xm_dev_alloc(ctx, (void **)&r.job, c * 4));
    r.cap = c;
    return XM_OK;
}

struct Prepared {
    std::vector<xm::JobDev> jobs;
    uint32_t n_items = 0;
    uint64_t cap_guess = 0;
};

xm_status prepare_jobs(xm_ctx *ctx, const xm_job *jobs, uint32_t n_jobs, uint32_t zc, Prepared &P)
{
    P.jobs.resize(n_jobs);
    uint64_t items = 0, guess = 0;
    std::vector<xm_alpha_req> areq;   // RA half-widths of every job's A zones
    std::vector<uint32_t> ajob;
    for (uint32_t j = 0; j < n_jobs; ++j) {
        const xm_segment *A = jobs[j].A, *B = jobs[j].B;
        if (!A || !B || A->ctx->device != ctx->device || B->ctx->device != ctx->device) {
            ctx->last_error = "job " + std::to_string(j) + ": missing segment or segment on another device";
            return XM_ERR_INVALID;
        }
        if (A->zh_deg != B->zh_deg || A->n_zones != B->n_zones) {
            ctx->last_error = "job " + std::to_string(j) + ": zone heights differ";
            return XM_ERR_MISMATCH;
        }
        if (!A->store || !B->store) {
            ctx->last_error = "job " + std::to_string(j) + ": a segment is offloaded (xm_segment_page_in it first)";
            return XM_ERR_INVALID;
        }
        for (const xm_segment *s : {A, B})   // a page-in copy of the segment must land first
            if (s->ready_pending) XM_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, s->ready, 0));
        xm_match_params p;
        if (xm_make_params(jobs[j].sr_deg, A->zh_deg, &p) != XM_OK) {
            ctx->last_error = "job " + std::to_string(j) + ": invalid radius";
            return XM_ERR_INVALID;
        }
        xm::JobDev &d = P.jobs[j];
        std::memset(&d, 0, sizeof(d));
        d.a_id = (const long long *)A->id;
        d.a_radec = A->radec;
        d.a_xyz = A->xyz;
        d.a_zoff = A->zone_off;
        d.b_id = (const long long *)B->id;
        d.b_radec = B->radec;
        d.b_xyz = B->xyz;
        d.b_bins = B->zbin;
        d.b_bin_log2 = B->zbin ? B->bin_log2 : 0;
        d.b_zoff = B->zone_off;
        d.sr_rad = p.sr_rad;
        d.sr_dist2 = p.sr_dist2;
        d.thr_hi = p.thr_hi;
        d.thr_lo = p.thr_lo;
        d.n_zones = A->n_zones;
        d.nz = p.nz;
        d.z_lo = A->z_lo;
        d.z_hi = A->z_hi;
        d.raq_shift = 32 - B->raq_bits;
        d.nA = (uint32_t)A->n;
        d.item_begin = (uint32_t)items;
        if (A->n > 0 && B->n > 0 && A->z_hi >= A->z_lo) {
            items += ((uint64_t)(A->z_hi - A->z_lo) + zc) / zc;
            areq.push_back({p.sr_deg, A->zh_deg, A->z_lo, A->z_hi, nullptr});
            ajob.push_back(j);
        }
        // first output size: 2 min(nA, nB) per job (Worker.cu:296-297 uses the max,
        // which for a small query against a large catalog would reserve the
        // catalog's size); an overflow reruns at the exact count
        guess += 2 * std::min(A->n, B->n);
        if (items >= 0xFFFFFF00ull) {
            ctx->last_error = "too many work items in one launch";
            return XM_ERR_INVALID;
        }
    }
    XM_TRY(xm_get_alpha_ranges(ctx, areq.data(), areq.size()));
    for (size_t q = 0; q < areq.size(); ++q) {
        P.jobs[ajob[q]].alpha = areq[q].dev;
        P.jobs[ajob[q]].alpha_z0 = areq[q].z0;
    }
    P.n_items = (uint32_t)items;
    P.cap_guess = std::max<uint64_t>(guess, 1 << 16);
    return XM_OK;
}

}  // namespace

// Runs the pair kernel over the jobs; on return ctx->res holds the matches
// (ungrouped) and ctx->h_counters the statistics.
xm_status xm_run_jobs(xm_ctx *ctx, const xm_job *jobs, uint32_t n_jobs, uint32_t flags, const xm_tuning *tuning,
                      bool want_job, xm_stats *stats, float *kernel_ms, const xm_pairs *direct, bool *direct_used)
{
    if (direct_used) *direct_used = false;
    cudaStream_t st = ctx->stream;
    xm::LaunchCfg L;
    L.sm_count = ctx->sm_count;
    L.variant = (flags & XM_PLAIN64) ? 1 : 0;
    L.count_cand = (flags & XM_COUNT_CAND) != 0;
    L.dist = (flags & XM_NO_DIST) == 0;
    // Default geometry.  Where A's populated zones hold 48 or more objects on average, a
    // zone is split into tiles anyway, so the wider tile of 256 objects (8 consumer warps)
    // packs two to three zones and keeps its lanes busy, with items of 32 zones: at 50M x 50M
    // (77 objects per zone) 3.43 against 3.92 ms for tiles of 128.
    {
        uint64_t objs = 0, zones = 0;
        for (uint32_t j = 0; j < n_jobs; ++j)
            if (jobs[j].A && jobs[j].A->n > 0 && jobs[j].A->z_hi >= jobs[j].A->z_lo) {
                objs += jobs[j].A->n;
                zones += (uint64_t)(jobs[j].A->z_hi - jobs[j].A->z_lo + 1);
            }
        if (zones && objs >= 48 * zones) {
            L.tile = 256;
            L.zc = 32;
        }
    }
    if (tuning) {
        if (tuning->tile) L.tile = (int)tuning->tile;
        if (tuning->chunk) L.chunk = tuning->chunk;
        if (tuning->blocks_per_sm) L.blocks_per_sm = (int)tuning->blocks_per_sm;
        if (tuning->zones) L.zc = tuning->zones;
    }
    if (L.tile != 64 && L.tile != 128 && L.tile != 256) return XM_ERR_INVALID;
    if (L.zc < 1 || L.zc > 64 || L.chunk < 1 || L.chunk > 32) return XM_ERR_INVALID;
    Prepared P;
    XM_TRY(prepare_jobs(ctx, jobs, n_jobs, L.zc, P));
    size_t jb = P.jobs.size() * sizeof(xm::JobDev);
    if (ctx->d_jobs_bytes < jb) {
        xm_dev_free(ctx, ctx->d_jobs);
        ctx->d_jobs = nullptr;
        ctx->d_jobs_bytes = 0;
        XM_TRY(xm_dev_alloc(ctx, &ctx->d_jobs, jb));
        ctx->d_jobs_bytes = jb;
    }
    XM_CUDA(ctx, cudaMemcpyAsync(ctx->d_jobs, P.jobs.data(), jb, cudaMemcpyHostToDevice, st));
    XM_TRY(ensure_result(ctx, std::max<uint64_t>(ctx->res.cap, P.cap_guess), want_job));
    // tile pre-pass: count tiles per work item, read the totals back, size the plans
    const size_t cnt_b = ((size_t)P.n_items * 8 + 255) & ~(size_t)255;
    const size_t off_b = ((size_t)(P.n_items + 1) * 8 + 255) & ~(size_t)255;
    const size_t scan_b = (xm_scan_tmp_bytes(P.n_items) + 255) & ~(size_t)255;
    const size_t need = cnt_b + off_b + scan_b;
    if (ctx->d_work_bytes < need) {
        xm_dev_free(ctx, ctx->d_work);
        ctx->d_work = nullptr;
        ctx->d_work_bytes = 0;
        XM_TRY(xm_dev_alloc(ctx, &ctx->d_work, need + need / 4));
        ctx->d_work_bytes = need + need / 4;
    }
    char *wp = (char *)ctx->d_work;
    uint32_t *tile_cnt = (uint32_t *)wp;
    uint32_t *tile_off = (uint32_t *)(wp + cnt_b);
    void *scan_tmp = wp + cnt_b + off_b;
    uint32_t n_normal = 0, n_heavy = 0;
    XM_CUDA(ctx, cudaEventRecord(ctx->ev[14], st));
    if (P.n_items > 0) {
        XM_CUDA(ctx, xm::plan_count(L, (const xm::JobDev *)ctx->d_jobs, (int)n_jobs, P.n_items, tile_cnt, tile_off,
                                    scan_tmp, st));
        XM_CUDA(ctx, cudaMemcpyAsync(ctx->h_tiles, tile_off + P.n_items, 4, cudaMemcpyDeviceToHost, st));
        XM_CUDA(ctx, cudaMemcpyAsync(ctx->h_tiles + 1, tile_off + 2 * P.n_items + 1, 4, cudaMemcpyDeviceToHost, st));
        XM_CUDA(ctx, cudaStreamSynchronize(st));
        n_normal = ctx->h_tiles[0];
        n_heavy = ctx->h_tiles[1];
        if ((uint64_t)n_normal + n_heavy >= 0xFFFFFF00ull) {
            ctx->last_error = "too many tiles in one launch";
            return XM_ERR_INVALID;
        }
        const size_t pb = xm::plan_bytes((uint64_t)n_normal + n_heavy) + 256;
        if (ctx->d_plans_bytes < pb) {
            xm_dev_free(ctx, ctx->d_plans);
            ctx->d_plans = nullptr;
            ctx->d_plans_bytes = 0;
            XM_TRY(xm_dev_alloc(ctx, &ctx->d_plans, pb + pb / 4));
            ctx->d_plans_bytes = pb + pb / 4;
        }
    }
    uint32_t retries = 0;
    float ms = 0, plan_ms = 0;
    const bool use_graph = (flags & XM_NO_GRAPH) == 0;
    for (;;) {
        xm::MatchOut out;
        out.pairs = (long long *)ctx->res.pairs;
        out.dist = L.dist ? ctx->res.dist : nullptr;
        out.job = want_job ? ctx->res.job : nullptr;
        out.cap = ctx->res.cap;
        const bool to_host = direct && retries == 0 && !want_job;
        if (to_host) {   // straight into the caller's pinned buffers
            out.pairs = (long long *)direct->pairs;
            out.dist = L.dist ? (double *)direct->dist : nullptr;
            out.cap = direct->capacity;
        }
        out.counters = ctx->counters;
        // counters cleared, tile plans, pair kernel, counters read back
        auto enqueue = [&](unsigned ev_flags) -> cudaError_t {
            cudaError_t e = cudaMemsetAsync(ctx->counters, 0, 16 * sizeof(unsigned long long), st);
            if (e == cudaSuccess && P.n_items > 0)
                e = xm::plan_make(L, (const xm::JobDev *)ctx->d_jobs, (int)n_jobs, P.n_items, tile_off, n_normal,
                                  n_heavy, ctx->d_plans, ctx->counters + 7, st);
            if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev[2], st, ev_flags);
            if (e == cudaSuccess && P.n_items > 0)
                e = xm::run_pairs(L, (const xm::JobDev *)ctx->d_jobs, ctx->d_plans, n_normal, n_heavy, out, st);
            if (e == cudaSuccess) e = cudaEventRecordWithFlags(ctx->ev[3], st, ev_flags);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(ctx->h_counters, ctx->counters, 16 * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, st);
            return e;
        };
        if (use_graph) {
            // captured into a graph; the context's executable graph is updated
            // in place when the launch sequence keeps its shape, else rebuilt
            XM_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            cudaError_t e = enqueue(cudaEventRecordExternal);
            cudaGraph_t g = nullptr;
            cudaError_t e2 = cudaStreamEndCapture(st, &g);
            if (e == cudaSuccess) e = e2;
            if (e == cudaSuccess && ctx->graph_exec) {
                cudaGraphExecUpdateResultInfo info;
                if (cudaGraphExecUpdate(ctx->graph_exec, g, &info) != cudaSuccess) {
                    cudaGetLastError();   // an update that does not fit is not an error
                    cudaGraphExecDestroy(ctx->graph_exec);
                    ctx->graph_exec = nullptr;
                }
            }
            if (e == cudaSuccess && !ctx->graph_exec) e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e == cudaSuccess) e = cudaGraphLaunch(ctx->graph_exec, st);
            XM_CUDA(ctx, e);
            ctx->graph_launches++;
        } else {
            XM_CUDA(ctx, enqueue(cudaEventRecordDefault));
        }
        XM_CUDA(ctx, cudaStreamSynchronize(st));
        cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]);
        if (retries == 0) cudaEventElapsedTime(&plan_ms, ctx->ev[14], ctx->ev[2]);
        if (ctx->h_counters[7]) {
            ctx->last_error = "pair kernel: a bounded wait for staged data ran out, or the tile plan overflowed";
            return XM_ERR_TIMEOUT;
        }
        uint64_t found = ctx->h_counters[0];
        if (to_host && found <= direct->capacity) {
            if (direct_used) *direct_used = true;
            break;
        }
        if (!to_host && found <= ctx->res.cap) break;
        if (to_host) {   // did not fit the caller's buffers: again into device buffers
            retries++;
            XM_TRY(ensure_result(ctx, found + found / 16 + 1024, want_job));
            continue;
        }
        // never truncate: grow to the exact count and run again
        retries++;
        uint64_t want = found + found / 16 + 1024;
        xm_dev_free(ctx, ctx->res.pairs);
        xm_dev_free(ctx, ctx->res.dist);
        xm_dev_free(ctx, ctx->res.job);
        ctx->res.pairs = nullptr; ctx->res.dist = nullptr; ctx->res.job = nullptr; ctx->res.cap = 0;
        XM_TRY(ensure_result(ctx, want, want_job));
    }
    ctx->res.count = ctx->h_counters[0];
    ctx->res.grouped = false;
    ctx->res.has_dist = L.dist;
    if (kernel_ms) *kernel_ms = ms;
    if (stats) {
        stats->n_match += ctx->h_counters[0];
        stats->n_tested += ctx->h_counters[2];
        stats->n_cand += ctx->h_counters[3];
        stats->n_border += ctx->h_counters[4];
        stats->n_exact += ctx->h_counters[5];
        stats->n_tiles += (uint64_t)n_normal + n_heavy;
        stats->n_launches += P.n_items > 0 ? 9 + retries : 0;   // count, 2 x 3 scan, plans, pairs
        stats->ms_plan += plan_ms;
        stats->n_retries += retries;
        stats->ms_match += ms;
    }
    return XM_OK;
}

static xm_status copy_out(xm_ctx *ctx, const int64_t *dpairs, const double *ddist, uint64_t count, xm_pairs *out,
                          xm_stats *stats)
{
    out->count = count;
    if (!out->pairs && !out->dist) return XM_OK;
    if (out->capacity < count) return XM_ERR_CAPACITY;
    cudaStream_t st = ctx->stream;
    XM_CUDA(ctx, cudaEventRecord(ctx->ev[4], st));
    if (out->pairs && count) XM_CUDA(ctx, cudaMemcpyAsync(out->pairs, dpairs, count * 16, cudaMemcpyDeviceToHost, st));
    if (out->dist && count) {
        if (!ctx->res.has_dist) {
            ctx->last_error = "distances asked for, but the match ran with XM_NO_DIST";
            return XM_ERR_INVALID;
        }
        XM_CUDA(ctx, cudaMemcpyAsync(out->dist, ddist, count * 8, cudaMemcpyDeviceToHost, st));
    }
    XM_CUDA(ctx, cudaEventRecord(ctx->ev[5], st));
    XM_CUDA(ctx, cudaStreamSynchronize(st));
    if (stats) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]);
        stats->ms_d2h += ms;
    }
    return XM_OK;
}

extern "C" xm_status xm_match(xm_ctx *ctx, const xm_segment *A, const xm_segment *B, double sr_deg, uint32_t flags,
                              xm_pairs *out, xm_stats *stats)
{
    if (!ctx || !A || !B) return XM_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    xm_job job = {A, B, sr_deg};
    XM_CUDA(ctx, cudaEventRecord(ctx->ev[6], ctx->stream));
    XM_TRY(xm_run_jobs(ctx, &job, 1, flags, nullptr, false, stats, nullptr));
    if (out) XM_TRY(copy_out(ctx, ctx->res.pairs, ctx->res.dist, ctx->res.count, out, stats));
    if (stats) {
        XM_CUDA(ctx, cudaEventRecord(ctx->ev[7], ctx->stream));
        XM_CUDA(ctx, cudaEventSynchronize(ctx->ev[7]));
        cudaEventElapsedTime(&stats->ms_total, ctx->ev[6], ctx->ev[7]);
    }
    return XM_OK;
}

extern "C" xm_status xm_fetch_pairs(xm_ctx *ctx, xm_pairs *out)
{
    if (!ctx || !out) return XM_ERR_INVALID;
    cudaSetDevice(ctx->device);
    const int64_t *p = ctx->res.grouped ? ctx->res.pairs_g : ctx->res.pairs;
    const double *d = ctx->res.grouped ? ctx->res.dist_g : ctx->res.dist;
    uint64_t n = std::min<uint64_t>(ctx->res.count, out->capacity);
    uint64_t total = ctx->res.count;
    xm_status rc = copy_out(ctx, p, d, n, out, nullptr);
    out->count = total;
    return rc;
}

// Device-accessible address of a pinned host buffer, or null for pageable memory.
static void *pinned_device_ptr(const void *p)
{
    if (!p) return nullptr;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

static xm_status grow(xm_ctx *ctx, void **p, size_t *have, size_t need)
{
    if (*have >= need && *p) return XM_OK;
    xm_dev_free(ctx, *p);
    *p = nullptr;
    *have = 0;
    XM_TRY(xm_dev_alloc(ctx, p, need));
    *have = need;
    return XM_OK;
}

// Both catalogs from host memory to matches in host memory.
//
// With pinned output buffers (device-accessible) the work is pipelined:
// B is copied and zone-built first; then A is streamed in chunks through two
// staging slots, each chunk copied on the second stream while the previous one
// is built and matched against B, its matches written by the pair kernel
// straight into the caller's buffers (device-to-host traffic that overlaps the
// next chunk's host-to-device copy).  Any subset of A can be matched against
// the whole of B, so the pair set is that of one match.  If the matches do not
// fit the buffers, or the buffers are pageable, the catalogs are built whole
// and matched once (XM_ERR_CAPACITY then reports the count and leaves the
// matches for xm_fetch_pairs).
namespace {
// Chunks of A.  A chunk is a slice of A's records in input order, so it spans
// all of A's zones and its match walks all of B's: few large chunks balance that
// against the overlap.  Their sizes fall towards the end, so that the work left
// after the last chunk's copy (its build, its match and its matches over the
// link) is short, while every earlier chunk is still matched before the next one
// has landed: n chunks of relative sizes n + 1, n, ..., 2, n = nA / 10M (5 at
// 50M: 48.9 ms at 50M x 50M against 50.1 ms for 4 equal chunks and 59 ms for
// one).  Environment XMATCH_CHUNK_OBJS sets the objects per chunk that fix n,
// XMATCH_CHUNK_WEIGHTS (comma-separated relative sizes, at most kMaxChunks) the
// whole schedule.
constexpr uint64_t kMaxChunks = 16;   // = the context's staging-slot events

uint64_t chunk_objs()
{
    const char *e = std::getenv("XMATCH_CHUNK_OBJS");
    const unsigned long long v = e ? std::strtoull(e, nullptr, 10) : 0ull;
    return v ? (uint64_t)v : 10000000ull;
}

// Staging slots of A's chunks (environment XMATCH_CHUNK_SLOTS, at least 2).
uint64_t chunk_slots()
{
    const char *e = std::getenv("XMATCH_CHUNK_SLOTS");
    const unsigned long long v = e ? std::strtoull(e, nullptr, 10) : 0ull;
    return v ? std::max<uint64_t>(2, std::min<uint64_t>(kMaxChunks, v)) : 2;
}

// Chunk boundaries of A: bounds[c] .. bounds[c + 1] is chunk c.
std::vector<uint64_t> chunk_bounds(uint64_t nA, uint64_t n_chunks)
{
    std::vector<double> w;
    if (const char *e = std::getenv("XMATCH_CHUNK_WEIGHTS")) {
        for (const char *p = e; *p;) {
            char *end = nullptr;
            const double v = std::strtod(p, &end);
            if (end == p) break;
            if (v > 0 && std::isfinite(v)) w.push_back(v);
            p = *end == ',' ? end + 1 : end;
        }
    }
    double sum = 0;
    for (double v : w) sum += v;
    if (w.size() > kMaxChunks || !std::isfinite(sum)) w.clear();
    if (w.empty()) {
        sum = 0;
        for (uint64_t c = 0; c < n_chunks; ++c) {
            w.push_back((double)(n_chunks + 1 - c));
            sum += w.back();
        }
    }
    std::vector<uint64_t> b(1, 0);
    double acc = 0;
    for (size_t c = 0; c < w.size(); ++c) {
        acc += w[c];
        const uint64_t e = c + 1 == w.size() ? nA : std::min<uint64_t>(nA, (uint64_t)((double)nA * (acc / sum)));
        b.push_back(std::max(e, b.back()));
    }
    return b;
}
}

static xm_status crossmatch_whole(xm_ctx *ctx, const xm_obj *A, uint64_t nA, xm_segment *sb, double sr_deg,
                                  double zh_deg, uint32_t flags, xm_pairs *out, xm_stats *stats)
{
    cudaStream_t st = ctx->stream;
    XM_TRY(grow(ctx, &ctx->stage, &ctx->stage_bytes, std::max<uint64_t>(nA, 1) * sizeof(xm_obj)));
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[12], st));
    if (nA) XM_CUDA(ctx, cudaMemcpyAsync(ctx->stage, A, nA * sizeof(xm_obj), cudaMemcpyHostToDevice, st));
    if (stats) XM_CUDA(ctx, cudaEventRecord(ctx->ev[13], st));
    xm_segment *sa = nullptr;
    xm_status rc = new_segment(ctx, 0, zh_deg, &sa);
    if (rc == XM_OK) rc = xm_build_impl(sa, (const xm_obj *)ctx->stage, nA, stats);
    if (rc == XM_OK && stats) {
        float t = 0;
        cudaEventElapsedTime(&t, ctx->ev[12], ctx->ev[13]);
        stats->ms_h2d += t;
    }
    if (rc == XM_OK) {
        xm_job job = {sa, sb, sr_deg};
        rc = xm_run_jobs(ctx, &job, 1, flags, nullptr, false, stats, nullptr);
        if (rc == XM_OK && out) rc = copy_out(ctx, ctx->res.pairs, ctx->res.dist, ctx->res.count, out, stats);
    }
    xm_segment_free(sa);
    return rc;
}

extern "C" xm_status xm_crossmatch(xm_ctx *ctx, const xm_obj *A, uint64_t nA, const xm_obj *B, uint64_t nB,
                                   double sr_deg, double zh_deg, uint32_t flags, xm_pairs *out, xm_stats *stats)
{
    if (!ctx || (nA && !A) || (nB && !B) || !(zh_deg > 0)) return XM_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    cudaStream_t st = ctx->stream, s2 = ctx->stream2;
    XM_CUDA(ctx, cudaEventRecord(ctx->ev[6], st));
    // B: copied and built whole
    XM_TRY(grow(ctx, &ctx->stage2, &ctx->stage2_bytes, std::max<uint64_t>(nB, 1) * sizeof(xm_obj)));
    XM_CUDA(ctx, cudaEventRecord(ctx->ev[1], st));
    if (nB) XM_CUDA(ctx, cudaMemcpyAsync(ctx->stage2, B, nB * sizeof(xm_obj), cudaMemcpyHostToDevice, st));
    XM_CUDA(ctx, cudaEventRecord(ctx->ev_b2, st));
    // the output route
    const bool want_dist = (flags & XM_NO_DIST) == 0;
    xm_pairs direct = {nullptr, nullptr, 0, 0};
    if (out && out->pairs && (!out->dist || want_dist)) {
        direct.pairs = (int64_t *)pinned_device_ptr(out->pairs);
        direct.dist = want_dist ? (double *)pinned_device_ptr(out->dist) : nullptr;
        direct.capacity = out->capacity;
    }
    const bool streamed = direct.pairs && (!want_dist || direct.dist);
    const uint64_t n_even = streamed ? std::max<uint64_t>(1, std::min<uint64_t>(kMaxChunks, nA / chunk_objs())) : 1;
    const std::vector<uint64_t> bounds = n_even > 1 ? chunk_bounds(nA, n_even) : std::vector<uint64_t>{0, nA};
    const uint64_t n_chunks = bounds.size() - 1;
    uint64_t chunk = 0;   // the largest chunk: the size of a staging slot
    for (uint64_t c = 0; c < n_chunks; ++c) chunk = std::max(chunk, bounds[c + 1] - bounds[c]);
    // A's chunks land in a ring of staging slots, copied on the second stream: chunk
    // c + n_slots is copied once chunk c's build has read its slot
    const uint64_t n_slots = std::min<uint64_t>(n_chunks, chunk_slots());
    const uint64_t slot_objs = std::max<uint64_t>(chunk, 1);
    XM_TRY(grow(ctx, &ctx->stage, &ctx->stage_bytes, n_slots * slot_objs * sizeof(xm_obj)));
    auto slot = [&](uint64_t c) { return (xm_obj *)ctx->stage + (c % n_slots) * slot_objs; };
    cudaEvent_t *landed = ctx->ev_slot;   // recorded only here
    auto copy_chunk = [&](uint64_t c) -> xm_status {
        const uint64_t first = bounds[c], n = bounds[c + 1] - bounds[c];
        if (n) XM_CUDA(ctx, cudaMemcpyAsync(slot(c), A + first, n * sizeof(xm_obj), cudaMemcpyHostToDevice, s2));
        XM_CUDA(ctx, cudaEventRecord(landed[c % n_slots], s2));
        return XM_OK;
    };
    xm_segment *sb = nullptr, *sa = nullptr;
    xm_status rc = new_segment(ctx, 1, zh_deg, &sb);
    if (rc == XM_OK && streamed) {
        // A's first n_slots chunks follow B on the link
        if (cudaStreamWaitEvent(s2, ctx->ev_b2, 0) != cudaSuccess) rc = XM_ERR_CUDA;
        for (uint64_t c = 0; rc == XM_OK && c < n_slots; ++c) rc = copy_chunk(c);
    }
    if (rc == XM_OK) rc = xm_build_impl(sb, (const xm_obj *)ctx->stage2, nB, stats);
    if (rc == XM_OK && stats) {
        float t = 0;
        cudaEventElapsedTime(&t, ctx->ev[1], ctx->ev_b2);
        stats->ms_h2d += t;
    }
    if (rc == XM_OK && !streamed) {
        rc = crossmatch_whole(ctx, A, nA, sb, sr_deg, zh_deg, flags, out, stats);
    } else if (rc == XM_OK) {
        uint64_t found = 0;
        bool overflow = false;
        rc = new_segment(ctx, 0, zh_deg, &sa);
        for (uint64_t c = 0; rc == XM_OK && c < n_chunks; ++c) {
            const uint64_t n = bounds[c + 1] - bounds[c];
            if (cudaStreamWaitEvent(st, landed[c % n_slots], 0) != cudaSuccess) {
                rc = XM_ERR_CUDA;
                break;
            }
            rc = xm_build_impl(sa, slot(c), n, stats);   // returns with the slot read (stream synchronised)
            if (rc == XM_OK && c + n_slots < n_chunks) rc = copy_chunk(c + n_slots);
            if (rc != XM_OK) break;
            xm_job job = {sa, sb, sr_deg};
            xm_pairs dc = direct;
            dc.pairs = direct.pairs + 2 * found;
            dc.dist = direct.dist ? direct.dist + found : nullptr;
            dc.capacity = direct.capacity - found;
            bool used = false;
            rc = xm_run_jobs(ctx, &job, 1, flags, nullptr, false, stats, nullptr, &dc, &used);
            if (rc != XM_OK) break;
            if (!used) {   // this chunk's matches did not fit: redo the whole match into device buffers
                overflow = true;
                break;
            }
            found += ctx->h_counters[0];
        }
        if (rc == XM_OK && overflow) {
            cudaStreamSynchronize(s2);
            rc = crossmatch_whole(ctx, A, nA, sb, sr_deg, zh_deg, flags, out, stats);
        } else if (rc == XM_OK) {
            out->count = found;
            ctx->res.count = 0;   // nothing left on the device for xm_fetch_pairs
            if (stats) stats->n_match = found;
        }
    }
    cudaStreamSynchronize(s2);
    xm_segment_free(sa);
    xm_segment_free(sb);
    if (rc == XM_OK && stats) {
        XM_CUDA(ctx, cudaEventRecord(ctx->ev[7], st));
        XM_CUDA(ctx, cudaEventSynchronize(ctx->ev[7]));
        cudaEventElapsedTime(&stats->ms_total, ctx->ev[6], ctx->ev[7]);
    }
    return rc;
}

// ---------------------------------------------------------------------------
// utilities
// ---------------------------------------------------------------------------
namespace {
__global__ void unit_vectors_kernel(const double *ra_deg, const double *dec_deg, uint64_t n, double *xyz)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        double x, y, z;
        xm::radec2xyz(__ddiv_rn(ra_deg[i], XM_RAD2DEG), __ddiv_rn(dec_deg[i], XM_RAD2DEG), x, y, z);
        xyz[3 * i] = x;
        xyz[3 * i + 1] = y;
        xyz[3 * i + 2] = z;
    }
}
}  // namespace

extern "C" xm_status xm_unit_vectors(xm_ctx *ctx, const double *ra_deg, const double *dec_deg, uint64_t n,
                                     double *xyz)
{
    if (!ctx || (n && (!ra_deg || !dec_deg || !xyz))) return XM_ERR_INVALID;
    if (!n) return XM_OK;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    void *buf = nullptr;
    XM_TRY(xm_dev_alloc(ctx, &buf, n * 40));
    double *dra = (double *)buf, *dde = dra + n, *dx = dde + n;
    xm_status rc = XM_OK;
    if (cudaMemcpyAsync(dra, ra_deg, n * 8, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dde, dec_deg, n * 8, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        rc = XM_ERR_CUDA;
    } else {
        unit_vectors_kernel<<<(unsigned)std::min<uint64_t>((n + 255) / 256, 4096), 256, 0, st>>>(dra, dde, n, dx);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(xyz, dx, n * 24, cudaMemcpyDeviceToHost, st) != cudaSuccess)
            rc = XM_ERR_CUDA;
    }
    cudaStreamSynchronize(st);
    xm_dev_free(ctx, buf);
    cudaStreamSynchronize(st);
    return rc;
}

extern "C" xm_status xm_alpha_table(double sr_deg, double zh_deg, double *alpha, int32_t n_zones)
{
    if (!alpha || !(sr_deg > 0) || !(zh_deg > 0) || n_zones < 0) return XM_ERR_INVALID;
    xm_host_alpha_table(sr_deg, zh_deg, n_zones, alpha);
    return XM_OK;
}

extern "C" xm_status xm_filter_bounds(double sr_deg, float *thr_hi, float *thr_lo)
{
    if (!thr_hi || !thr_lo) return XM_ERR_INVALID;
    xm_match_params p;
    const xm_status s = xm_make_params(sr_deg, 1.0, &p);
    if (s != XM_OK) return s;
    *thr_hi = p.thr_hi;
    *thr_lo = p.thr_lo;
    return XM_OK;
}
