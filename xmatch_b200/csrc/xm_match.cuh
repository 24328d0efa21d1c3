// xm_match.cuh -- job table and launch description of the pair kernel.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace xm {

// One segment-pair job (Job.h:16-29) as the pair kernel sees it.
struct JobDev {
    const long long *a_id;
    const double2 *a_radec;
    const float4 *a_xyz;
    const uint32_t *a_zoff;    // [n_zones + 1]
    const long long *b_id;
    const double2 *b_radec;
    const float4 *b_xyz;
    const uint16_t *b_bins;    // B's per-zone bin index, or null (xm_segment::zbin)
    int b_bin_log2;
    const uint32_t *b_zoff;    // [n_zones + 1]
    const double *alpha;       // RA half-width of A's zone z at alpha[z - alpha_z0], z in [z_lo, z_hi]
    double sr_rad, sr_dist2;
    float thr_hi, thr_lo;
    int n_zones, nz;
    int z_lo, z_hi;            // populated zone range of A
    uint32_t nA;               // objects of A
    uint32_t item_begin;       // first global work item of this job
    int raq_shift;             // xyz.w holds raq32(ra) >> raq_shift
    int alpha_z0;
};

struct MatchOut {
    long long *pairs;          // [2 * cap]
    double *dist;              // [cap] or null
    uint32_t *job;             // [cap] or null
    unsigned long long cap;
    // [0] matches, [1] next normal tile, [2] tested, [3] candidates, [4] in margin band,
    // [5] FP64 decisions, [6] next heavy piece, [7] error flag (a bounded wait ran out)
    unsigned long long *counters;
};

struct LaunchCfg {
    int tile = 128;            // A objects per tile = threads per block
    uint32_t zc = 16;          // zones per work item
    uint32_t chunk = 16;       // tiles per work-stealing claim (<= 32)
    int blocks_per_sm = 0;     // 0 = occupancy limit
    int sm_count = 148;
    int variant = 0;           // 0 FP32 reject + FP64 decision, 1 plain FP64
    bool count_cand = false;
    bool dist = true;
};

size_t plan_bytes(uint64_t n_plans);

// Tile pre-pass, part 1: tiles per work item.  cnt: [2 n_items] (normal, heavy),
// off: [2 (n_items + 1)] exclusive scans of both halves (totals at off[n_items]
// and off[2 n_items + 1]), scan_tmp: xm_scan_tmp_bytes(n_items).
cudaError_t plan_count(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_items, uint32_t *cnt,
                       uint32_t *off, void *scan_tmp, cudaStream_t st);
// Part 2: plans for n_heavy heavy pieces (first) and n_normal tiles; an
// overflow sets *err.
cudaError_t plan_make(const LaunchCfg &L, const JobDev *jobs, int n_jobs, uint32_t n_items, const uint32_t *off,
                      uint32_t n_normal, uint32_t n_heavy, void *plans, unsigned long long *err, cudaStream_t st);
// The pair kernel over the plans (counters[6] and counters[1] must be zero).
cudaError_t run_pairs(const LaunchCfg &L, const JobDev *jobs, const void *plans, uint32_t n_normal, uint32_t n_heavy,
                      const MatchOut &out, cudaStream_t st);

}  // namespace xm
