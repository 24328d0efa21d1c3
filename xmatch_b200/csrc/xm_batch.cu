// xm_batch.cu -- many segment-pair jobs in one persistent launch.
//
// Replaces the reference's job loop: JobManager holds the cross product of
// A segments x B segments (JobManager.cpp:5-14) and one host thread per GPU
// pulls jobs under a mutex (NextPreferredJob, JobManager.cpp:16-41;
// Worker::operator(), Worker.cu:430-485), launching one kernel per zone pair
// for each.  Here all jobs' tiles form one work list that the persistent
// pair kernel drains with an atomic counter (heavy pieces first, then tiles
// in chunks); matches carry their job index and are grouped by job with a
// counting sort afterwards.  After the host has read the tile totals, the
// launch sequence (counters cleared, tile plans, pair kernel, counters read
// back) runs as a CUDA graph held by the context: captured on every call and
// applied to the executable graph by an in-place update, so a batch of
// thousands of jobs is one graph launch (xm_run_jobs, xm_api.cu).
#include <algorithm>
#include <cstring>
#include <vector>

#include "xm_internal.h"
#include "xm_match.cuh"

namespace {

constexpr int kHistSmem = 8192;

__global__ void job_hist(const uint32_t *__restrict__ job, unsigned long long n, uint32_t *__restrict__ cnt,
                         int n_jobs)
{
    __shared__ uint32_t h[kHistSmem];
    const bool use_smem = n_jobs <= kHistSmem;
    if (use_smem)
        for (int k = threadIdx.x; k < n_jobs; k += blockDim.x) h[k] = 0;
    __syncthreads();
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        uint32_t j = job[i];
        if (use_smem) atomicAdd(&h[j], 1u); else atomicAdd(&cnt[j], 1u);
    }
    __syncthreads();
    if (use_smem)
        for (int k = threadIdx.x; k < n_jobs; k += blockDim.x)
            if (h[k]) atomicAdd(&cnt[k], h[k]);
}

__device__ __forceinline__ unsigned lanemask_lt_b()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void job_scatter(const uint32_t *__restrict__ job, const longlong2 *__restrict__ pairs,
                            const double *__restrict__ dist, unsigned long long n, const uint32_t *__restrict__ off,
                            uint32_t *__restrict__ cursor, longlong2 *__restrict__ pairs_g, double *__restrict__ dist_g)
{
    const unsigned lane = threadIdx.x & 31;
    unsigned long long warp0 = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) & ~31ull;
    unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = warp0; base < n; base += stride) {
        unsigned long long i = base + lane;
        int j = i < n ? (int)job[i] : -1;
        unsigned peers = __match_any_sync(0xffffffffu, j);
        int leader = __ffs(peers) - 1;
        uint32_t slot = 0;
        if (j >= 0 && (int)lane == leader) slot = atomicAdd(&cursor[j], (uint32_t)__popc(peers));
        slot = __shfl_sync(0xffffffffu, slot, leader);
        if (j >= 0) {
            uint32_t pos = off[j] + slot + __popc(peers & lanemask_lt_b());
            pairs_g[pos] = pairs[i];
            if (dist) dist_g[pos] = dist[i];
        }
    }
}

}  // namespace

// Groups ctx->res by job into pairs_g/dist_g and fills res.job_off.
xm_status xm_group_by_job(xm_ctx *ctx, uint32_t n_jobs, uint32_t *n_launch)
{
    xm_result_buf &r = ctx->res;
    cudaStream_t st = ctx->stream;
    const uint64_t n = r.count;
    if (r.cap_g < std::max<uint64_t>(n, 1)) {
        xm_dev_free(ctx, r.pairs_g);
        xm_dev_free(ctx, r.dist_g);
        r.pairs_g = nullptr; r.dist_g = nullptr; r.cap_g = 0;
        uint64_t c = std::max<uint64_t>(n, 1);
        XM_TRY(xm_dev_alloc(ctx, (void **)&r.pairs_g, c * 16));
        XM_TRY(xm_dev_alloc(ctx, (void **)&r.dist_g, c * 8));
        r.cap_g = c;
    }
    void *tmp = nullptr;
    size_t scan_b = xm_scan_tmp_bytes(n_jobs);
    XM_TRY(xm_dev_alloc(ctx, &tmp, (size_t)(n_jobs + 1) * 8 + scan_b + 16));
    uint32_t *cnt = (uint32_t *)tmp;
    uint32_t *off = cnt + n_jobs + 1;
    void *scan_tmp = off + n_jobs + 1;
    xm_status rc = XM_OK;
    do {
        if (cudaMemsetAsync(cnt, 0, (size_t)(n_jobs + 1) * 4, st) != cudaSuccess) { rc = XM_ERR_CUDA; break; }
        unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->sm_count * 4);
        if (n) job_hist<<<std::max(g, 1u), 256, 0, st>>>(r.job, n, cnt, (int)n_jobs);
        if (xm_scan_exclusive_u32(cnt, off, n_jobs, scan_tmp, st) != cudaSuccess) { rc = XM_ERR_CUDA; break; }
        if (cudaMemsetAsync(cnt, 0, (size_t)n_jobs * 4, st) != cudaSuccess) { rc = XM_ERR_CUDA; break; }
        if (n)
            job_scatter<<<std::max(g, 1u), 256, 0, st>>>(r.job, (const longlong2 *)r.pairs,
                                                         r.has_dist ? r.dist : nullptr, n, off, cnt,
                                                         (longlong2 *)r.pairs_g, r.dist_g);
        *n_launch += (n ? 2 : 0) + 3;
        std::vector<uint32_t> h(n_jobs + 1);
        if (cudaMemcpyAsync(h.data(), off, (size_t)(n_jobs + 1) * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = XM_ERR_CUDA;
            break;
        }
        r.job_off.assign(h.begin(), h.end());
        r.grouped = true;
    } while (0);
    if (rc != XM_OK) ctx->last_error = "grouping matches by job failed";
    xm_dev_free(ctx, tmp);
    return rc;
}

extern "C" xm_status xm_match_batch(xm_ctx *ctx, const xm_job *jobs, uint32_t n_jobs, uint32_t flags,
                                    const xm_tuning *tuning, xm_pairs *outs, uint64_t *job_counts, xm_stats *stats)
{
    if (!ctx || (n_jobs && !jobs)) return XM_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (n_jobs == 0) return XM_OK;
    XM_CUDA(ctx, cudaEventRecord(ctx->ev[6], ctx->stream));
    XM_TRY(xm_run_jobs(ctx, jobs, n_jobs, flags, tuning, n_jobs > 1, stats, nullptr));
    uint32_t launches = 0;
    if (n_jobs > 1) {
        XM_TRY(xm_group_by_job(ctx, n_jobs, &launches));
    } else {
        ctx->res.job_off = {0ull, (uint64_t)ctx->res.count};
        ctx->res.grouped = false;
    }
    const std::vector<uint64_t> &off = ctx->res.job_off;
    if (job_counts)
        for (uint32_t j = 0; j < n_jobs; ++j) job_counts[j] = off[j + 1] - off[j];
    if (outs) {
        const int64_t *P = ctx->res.grouped ? ctx->res.pairs_g : ctx->res.pairs;
        const double *D = ctx->res.grouped ? ctx->res.dist_g : ctx->res.dist;
        // one bulk copy into pinned staging, then per-job host copies
        uint64_t n = ctx->res.count;
        bool any_dist = false, too_small = false;
        for (uint32_t j = 0; j < n_jobs; ++j) {
            uint64_t c = off[j + 1] - off[j];
            outs[j].count = c;
            if ((outs[j].pairs || outs[j].dist) && outs[j].capacity < c) too_small = true;
            any_dist |= outs[j].dist != nullptr;
        }
        if (too_small) return XM_ERR_CAPACITY;
        if (any_dist && !ctx->res.has_dist) return XM_ERR_INVALID;
        int64_t *hp = nullptr;
        double *hd = nullptr;
        if (n) {
            XM_CUDA(ctx, cudaMallocHost(&hp, n * 16));
            if (any_dist && cudaMallocHost(&hd, n * 8) != cudaSuccess) {
                cudaFreeHost(hp);
                return XM_ERR_NOMEM;
            }
            cudaStream_t st = ctx->stream;
            XM_CUDA(ctx, cudaEventRecord(ctx->ev[4], st));
            cudaMemcpyAsync(hp, P, n * 16, cudaMemcpyDeviceToHost, st);
            if (hd) cudaMemcpyAsync(hd, D, n * 8, cudaMemcpyDeviceToHost, st);
            XM_CUDA(ctx, cudaEventRecord(ctx->ev[5], st));
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                cudaFreeHost(hp);
                if (hd) cudaFreeHost(hd);
                ctx->last_error = cudaGetErrorString(e);
                return XM_ERR_CUDA;
            }
            if (stats) {
                float ms = 0;
                cudaEventElapsedTime(&ms, ctx->ev[4], ctx->ev[5]);
                stats->ms_d2h += ms;
            }
            for (uint32_t j = 0; j < n_jobs; ++j) {
                uint64_t c = off[j + 1] - off[j];
                if (!c) continue;
                if (outs[j].pairs) std::memcpy(outs[j].pairs, hp + 2 * off[j], c * 16);
                if (outs[j].dist) std::memcpy(outs[j].dist, hd + off[j], c * 8);
            }
            cudaFreeHost(hp);
            if (hd) cudaFreeHost(hd);
        }
    }
    if (stats) {
        stats->n_launches += launches;
        XM_CUDA(ctx, cudaEventRecord(ctx->ev[7], ctx->stream));
        XM_CUDA(ctx, cudaEventSynchronize(ctx->ev[7]));
        cudaEventElapsedTime(&stats->ms_total, ctx->ev[6], ctx->ev[7]);
    }
    return XM_OK;
}

extern "C" xm_status xm_autotune_batch(xm_ctx *ctx, const xm_job *jobs, uint32_t n_jobs, uint32_t flags,
                                       xm_tuning *best, float *best_ms, float *fixed_ms)
{
    if (!ctx || !best || (n_jobs && !jobs)) return XM_ERR_INVALID;
    cudaSetDevice(ctx->device);
    const uint32_t tiles[] = {64, 128, 256};
    const uint32_t chunks[] = {4, 16};
    const uint32_t zones[] = {4, 16, 64};
    // fixed-tile reference point: tile 128, 16 zones per item, 16 tiles per claim;
    // it is the starting best, so the setting returned is never slower than it
    // as measured here
    xm_tuning b = {128, 16, 0, 16};
    float fixed = 0;
    {
        float ms = 0;
        XM_TRY(xm_run_jobs(ctx, jobs, n_jobs, flags, &b, n_jobs > 1, nullptr, &ms));   // warm (and size the output)
        XM_TRY(xm_run_jobs(ctx, jobs, n_jobs, flags, &b, n_jobs > 1, nullptr, &ms));
        fixed = ms;
    }
    float bms = fixed;
    for (uint32_t tl : tiles)
        for (uint32_t ch : chunks)
            for (uint32_t zn : zones) {
            xm_tuning t = {tl, ch, 0, zn};
            float m1 = 0, m2 = 0;
            XM_TRY(xm_run_jobs(ctx, jobs, n_jobs, flags, &t, n_jobs > 1, nullptr, &m1));
            XM_TRY(xm_run_jobs(ctx, jobs, n_jobs, flags, &t, n_jobs > 1, nullptr, &m2));
            float ms = std::min(m1, m2);
            if (ms < bms) {
                bms = ms;
                b = t;
            }
        }
    *best = b;
    if (best_ms) *best_ms = bms;
    if (fixed_ms) *fixed_ms = fixed;
    return XM_OK;
}
