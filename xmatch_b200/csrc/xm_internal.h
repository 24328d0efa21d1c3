// xm_internal.h -- library-private types of libxmatch_b200.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <map>
#include <unordered_map>
#include <vector>

#include "../../include/xmatch.h"

// RA half-widths of one zone range for one (radius, zone height).
struct xm_alpha_key {
    uint64_t sr, zh;         // bit patterns of the doubles
    int32_t z0, z1;          // zones [z0, z1]
    bool operator<(const xm_alpha_key &o) const
    {
        if (sr != o.sr) return sr < o.sr;
        if (zh != o.zh) return zh < o.zh;
        if (z0 != o.z0) return z0 < o.z0;
        return z1 < o.z1;
    }
};
struct xm_alpha_entry {
    double *dev = nullptr;   // [z1 - z0 + 1] radians (180 = no cut)
    size_t bytes = 0;
};
// One request of xm_get_alpha_ranges; dev is filled in.
struct xm_alpha_req {
    double sr_deg, zh_deg;
    int32_t z0, z1;
    const double *dev;
};

// Device result of the last match call (library-owned, grown on demand).
struct xm_result_buf {
    int64_t *pairs = nullptr;   // [2 * cap] (idA, idB)
    double *dist = nullptr;     // [cap]
    uint32_t *job = nullptr;    // [cap] job index (batches)
    uint64_t cap = 0;
    uint64_t count = 0;         // matches of the last call
    // batch grouping
    int64_t *pairs_g = nullptr;
    double *dist_g = nullptr;
    uint64_t cap_g = 0;
    std::vector<uint64_t> job_off;  // host copy, n_jobs + 1
    bool grouped = false;
    bool has_dist = true;
};

struct xm_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    cudaEvent_t ev[16] = {};
    std::string last_error;
    // counters: [0] matches, [1] tiles claimed, [2..] statistics
    unsigned long long *counters = nullptr;   // device, 16 entries
    unsigned long long *h_counters = nullptr; // pinned host mirror
    std::map<xm_alpha_key, xm_alpha_entry> alpha_cache;
    size_t alpha_bytes = 0;
    xm_result_buf res;
    // job table and tile pre-pass buffers
    void *d_jobs = nullptr;
    size_t d_jobs_bytes = 0;
    void *d_work = nullptr;      // tile counts, offsets, scan scratch
    size_t d_work_bytes = 0;
    void *d_plans = nullptr;     // tile plans
    size_t d_plans_bytes = 0;
    uint32_t *h_tiles = nullptr; // pinned: tile totals read back after the count pass
    void *build_tmp = nullptr;   // zone-build scratch, shared by the context's builds
    void *stage = nullptr;       // host records copied here by xm_segment_build (and A of xm_crossmatch)
    size_t stage_bytes = 0;
    void *stage2 = nullptr;      // B of xm_crossmatch
    size_t stage2_bytes = 0;
    cudaStream_t stream2 = nullptr;   // copies that overlap work on stream
    cudaEvent_t ev_b2 = nullptr;
    cudaEvent_t ev_slot[16] = {};   // xm_crossmatch: a chunk of A has landed in a staging slot
    size_t build_tmp_bytes = 0;
    cudaGraphExec_t graph_exec = nullptr;   // the pair-kernel launch sequence (see xm_run_jobs)
    uint64_t graph_launches = 0;
};

struct xm_segment {
    xm_ctx *ctx = nullptr;
    uint32_t seg_id = 0;
    uint64_t n_in = 0;        // records given
    uint64_t n = 0;           // objects kept (valid zone)
    uint64_t cap = 0;         // capacity of the SoA arrays (id has 2 spare entries)
    double zh_deg = 0;
    int32_t n_zones = 0;
    int32_t z_lo = 0, z_hi = -1;   // first / last zone holding an object
    int raq_bits = 32;             // leading bits of the quantised ra kept in xyz.w
    uint32_t dropped_host = 0;
    void *store = nullptr;         // one device allocation holding the arrays below (null when offloaded)
    size_t store_bytes = 0;        // its size, and the offsets of id, radec, xyz in it
    size_t off_id = 0, off_radec = 0, off_xyz = 0, off_zbin = 0;
    int bin_log2 = 0;              // 2^bin_log2 quantised-ra bins per zone in zbin (0 = no index)
    void *host_store = nullptr;    // pinned host copy of the store (xm_segment_offload)
    cudaEvent_t ready = nullptr;   // recorded after a page-in copy (xm_segment_page_in)
    bool ready_pending = false;    // work on ctx->stream must wait for `ready` first
    uint32_t *zone_off = nullptr;  // [n_zones + 8]; [n_zones + 1] = dropped count; the rest
                                   // pads 16-byte bulk copies of zone-offset slices
    int64_t *id = nullptr;
    double2 *radec = nullptr;      // radians
    float4 *xyz = nullptr;         // FP32 unit vector; w = quantised-ra bits
    uint16_t *zbin = nullptr;      // [n_zones << bin_log2] per-zone bin index (see xm_build.cu)
};
// Points the segment's arrays into a store of its layout at base (null clears them).
void xm_seg_layout(xm_segment *seg, void *base);
// Allocates (or keeps, when large enough) the segment's arrays for n objects.
xm_status xm_seg_storage(xm_segment *seg, uint64_t n);

// ---- error plumbing ----
#define XM_CUDA(ctx, call)                                                       \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            if (ctx) (ctx)->last_error = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return (e_ == cudaErrorMemoryAllocation) ? XM_ERR_NOMEM : XM_ERR_CUDA; \
        }                                                                        \
    } while (0)

#define XM_TRY(call)                        \
    do {                                    \
        xm_status s_ = (call);              \
        if (s_ != XM_OK) return s_;         \
    } while (0)

// ---- internal entry points shared between translation units ----
xm_status xm_dev_alloc(xm_ctx *ctx, void **p, size_t bytes);
// The same, stream-ordered on another stream of the context.
xm_status xm_dev_alloc_on(xm_ctx *ctx, void **p, size_t bytes, cudaStream_t st);
void xm_dev_free(xm_ctx *ctx, void *p);
// Runs the pair kernel over the jobs; ctx->res holds the (ungrouped) matches.
// direct (optional): pinned host buffers (device-accessible pointers) the pair
// kernel writes the matches into when they hold them all; *direct_used tells
// whether they did (else the matches are in ctx->res).
xm_status xm_run_jobs(xm_ctx *ctx, const xm_job *jobs, uint32_t n_jobs, uint32_t flags, const xm_tuning *tuning,
                      bool want_job, xm_stats *stats, float *kernel_ms, const xm_pairs *direct = nullptr,
                      bool *direct_used = nullptr);
// Groups ctx->res by job (res.pairs_g, res.dist_g, res.job_off).
xm_status xm_group_by_job(xm_ctx *ctx, uint32_t n_jobs, uint32_t *n_launch);
// Device tables of RA half-widths for each request's zone range (cached).
xm_status xm_get_alpha_ranges(xm_ctx *ctx, xm_alpha_req *req, size_t n);
void alpha_cache_clear(xm_ctx *ctx);
void xm_host_alpha_table(double sr_deg, double zh_deg, int32_t n_zones, double *out);

// exclusive scan of n uint32 values (out[n] = total); tmp from xm_scan_tmp_bytes
size_t xm_scan_tmp_bytes(size_t n);
cudaError_t xm_scan_exclusive_u32(const uint32_t *in, uint32_t *out, size_t n, void *tmp,
                                  cudaStream_t s);

xm_status xm_build_impl(xm_segment *seg, const xm_obj *dev_objs, uint64_t n, xm_stats *st);
// Sort-key layout of a segment with n_zones zones: raq bits kept, radix passes.
void xm_raq_layout(int32_t n_zones, int *raq_bits, int *passes);

// Match parameters derived on the host (Worker.cu:310-317).
struct xm_match_params {
    double sr_deg, sr_rad, sr_dist2;
    float thr_hi;       // FP32 reject threshold: c32 > thr_hi => chord^2 >= sr_dist2
    float thr_lo;       // c32 < thr_lo => chord^2 < sr_dist2 and, with alpha < 3, both cuts hold
    int32_t nz;
};
xm_status xm_make_params(double sr_deg, double zh_deg, xm_match_params *p);
