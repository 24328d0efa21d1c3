// ref_harness.cu -- runs the REFERENCE's own pair kernel (TEST INFRASTRUCTURE).
//
// Links against BoostXmatch/Worker.cu and BoostXmatch/Common.cu compiled
// unmodified for sm_100a (recipe: oracle/ref_kernel.mk, output in
// oracle/_ref/).  It does not call Worker::Match, whose host-to-device
// copies are short (Worker.cu:284,289 copy vRadec.size() bytes): it copies
// the whole arrays itself and then runs the reference zone loop of
// Worker.cu:310-366 -- nz = ceil(r/zh), sr_rad, sr_dist2, calc_alpha per
// (zid1, zid2) on the host, one xmatch_kernel launch per zone pair with
// 16x16 blocks -- collecting the segment-local index pairs it appends.
// The caller passes A and B already grouped by zone (any order inside a
// zone: the kernel tests all pairs of a zone pair).
//
// The kernel's block compaction (Worker.cu:157-233) also reads the shared
// slots of threads that left at Worker.cu:125 (outside the zone ranges), so
// a partial block compacts stale shared memory: it drops tested matches and
// appends pairs that were never tested.  Two modes:
//   pad = 0  the reference launch geometry; with `validate` the harness
//            synchronises after every launch and counts appended pairs that
//            fall outside that launch's index ranges (evidence of the defect);
//   pad = 1  every launch covers whole 16x16 blocks: the index ranges are
//            extended to multiples of 16 (into the next zone's objects, or 16
//            dummy records appended to each array that can never match), so
//            no thread leaves early and the compaction is sound; only pairs
//            inside the true ranges are kept.  This is the reference
//            predicate evaluated by the reference's own code.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <ostream>
#include <vector>

#include <cuda_runtime.h>

#include "Common.h"
#include "Obj.h"

namespace xmatch {
__global__ void xmatch_kernel(const dbl2 *p_radec1, int i1s, int i1e, const dbl2 *p_radec2, int i2s, int i2e,
                              double sr_rad, double alpha_rad, double sr_dist2, uint2 *m_idx, unsigned int m_size,
                              unsigned int *m_end);
}

// Symbols Worker.o references from the reference's host classes (logging,
// CUDA context, job manager).  The harness never runs that host code; these
// definitions only satisfy the linker.
#include "CudaContext.h"
#include "Job.h"
#include "JobManager.h"
#include "Log.h"
namespace xmatch {
Log::~Log() {}
std::ostream &Log::Get(LogLevel) { return buffer; }
CudaContext::CudaContext(CudaManagerPtr) : id(-1) {}
CudaContext::~CudaContext() {}
JobPtr JobManager::NextPreferredJob(JobPtr) { return JobPtr(); }
void JobManager::SetStatus(JobPtr, JobStatus) {}
std::ostream &operator<<(std::ostream &o, const Job &) { return o; }
}

extern "C" {

// radec_*: [2 n] radians (ra, dec) grouped by zone; zbeg/zend: [n_zones].
// Writes up to cap (iA, iB) pairs of segment-local indices, returns the
// number of matches the kernel counted (may exceed cap), or -1 on error.
// ms_loop (optional): device time of the zone loop.
long long ref_xmatch(const double *radec_a, long long na, const int *zbeg_a, const int *zend_a,
                     const double *radec_b, long long nb, const int *zbeg_b, const int *zend_b, int n_zones,
                     double sr_deg, double zh_deg, unsigned int *pairs, unsigned int cap, int *launches,
                     int validate, long long *outside, int pad, float *ms_loop)
{
    using namespace xmatch;
    dbl2 *da = nullptr, *db = nullptr;
    uint2 *dm = nullptr;
    unsigned int *dn = nullptr;
    long long result = -1;
    int nl = 0;
    unsigned int kept = 0;
    long long out_n = 0;
    bool failed = false;
    const long long padn = 16;   // dummy records after each array
    if (cudaMalloc(&da, sizeof(dbl2) * (na + padn)) != cudaSuccess) return -1;
    if (cudaMalloc(&db, sizeof(dbl2) * (nb + padn)) != cudaSuccess) { cudaFree(da); return -1; }
    if (cudaMalloc(&dm, sizeof(uint2) * (cap > 0 ? cap : 1)) != cudaSuccess) { cudaFree(da); cudaFree(db); return -1; }
    if (cudaMalloc(&dn, sizeof(unsigned int)) != cudaSuccess) { cudaFree(da); cudaFree(db); cudaFree(dm); return -1; }
    do {
        if (na && cudaMemcpy(da, radec_a, sizeof(dbl2) * na, cudaMemcpyHostToDevice) != cudaSuccess) break;
        if (nb && cudaMemcpy(db, radec_b, sizeof(dbl2) * nb, cudaMemcpyHostToDevice) != cudaSuccess) break;
        {   // dummies: dec far outside [-pi/2, pi/2] and of opposite sign in A and B, so no pair
            // involving one passes the dec cut of Worker.cu:88
            dbl2 dummy_a[16], dummy_b[16];
            for (int q = 0; q < 16; ++q) {
                dummy_a[q].x = 0.0; dummy_a[q].y = 1000.0;
                dummy_b[q].x = 0.0; dummy_b[q].y = -1000.0;
            }
            if (cudaMemcpy(da + na, dummy_a, sizeof(dummy_a), cudaMemcpyHostToDevice) != cudaSuccess) break;
            if (cudaMemcpy(db + nb, dummy_b, sizeof(dummy_b), cudaMemcpyHostToDevice) != cudaSuccess) break;
        }
        if (cudaMemset(dn, 0, sizeof(unsigned int)) != cudaSuccess) break;
        // Worker.cu:310-317
        const int nz = (int)ceil(sr_deg / zh_deg);
        const double sr_rad = sr_deg / RAD2DEG;
        double sr_dist2 = 2.0 * sin(sr_rad / 2.0);
        sr_dist2 *= sr_dist2;
        // Worker.cu:330-366; timed with events around the whole zone loop (launch gaps included)
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        if (ms_loop) {
            cudaEventCreate(&ev0);
            cudaEventCreate(&ev1);
            cudaEventRecord(ev0);
        }
        for (int zid1 = 0; zid1 < n_zones; zid1++) {
            const int i1s = zbeg_a[zid1], i1e = zend_a[zid1], n1 = i1e - i1s;
            if (n1 < 1) continue;
            const int zid2start = zid1 - nz > 0 ? zid1 - nz : 0;
            const int zid2end = zid1 + nz < n_zones - 1 ? zid1 + nz : n_zones - 1;
            for (int zid2 = zid2start; zid2 <= zid2end; zid2++) {
                const int i2s = zbeg_b[zid2], i2e = zend_b[zid2], n2 = i2e - i2s;
                if (n2 < 1) continue;
                const double alpha_rad = calc_alpha(sr_deg, zh_deg, zid1);
                dim3 dimBlock(16, 256 / 16);
                dim3 dimGrid((n1 + dimBlock.x - 1) / dimBlock.x, (n2 + dimBlock.y - 1) / dimBlock.y);
                // padded ranges end on a block edge (at most 15 past the zone, within the dummies)
                const int e1 = pad ? i1s + (int)(dimGrid.x * dimBlock.x) : i1e;
                const int e2 = pad ? i2s + (int)(dimGrid.y * dimBlock.y) : i2e;
                xmatch_kernel<<<dimGrid, dimBlock>>>(da, i1s, e1, db, i2s, e2, sr_rad, alpha_rad, sr_dist2,
                                                     validate ? dm + kept : dm, validate ? cap - kept : cap, dn);
                ++nl;
                if (validate) {
                    // take this launch's pairs, keep those inside its ranges
                    unsigned int c = 0;
                    if (cudaMemcpy(&c, dn, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess) { failed = true; break; }
                    if (c > cap - kept) { failed = true; break; }
                    std::vector<uint2> h(c);
                    if (c && cudaMemcpy(h.data(), dm + kept, sizeof(uint2) * c, cudaMemcpyDeviceToHost) != cudaSuccess) {
                        failed = true;
                        break;
                    }
                    for (unsigned int q = 0; q < c; ++q) {
                        if ((int)h[q].x >= i1s && (int)h[q].x < i1e && (int)h[q].y >= i2s && (int)h[q].y < i2e) {
                            pairs[2 * kept] = h[q].x;
                            pairs[2 * kept + 1] = h[q].y;
                            ++kept;
                        } else {
                            ++out_n;
                        }
                    }
                    if (cudaMemset(dn, 0, sizeof(unsigned int)) != cudaSuccess) { failed = true; break; }
                }
            }
            if (failed) break;
        }
        if (ms_loop) cudaEventRecord(ev1);
        if (failed) break;
        if (cudaDeviceSynchronize() != cudaSuccess) break;
        if (ms_loop) {
            cudaEventElapsedTime(ms_loop, ev0, ev1);
            cudaEventDestroy(ev0);
            cudaEventDestroy(ev1);
        }
        if (validate) {
            result = (long long)kept;
            if (outside) *outside = out_n;
            break;
        }
        unsigned int count = 0;
        if (cudaMemcpy(&count, dn, sizeof(count), cudaMemcpyDeviceToHost) != cudaSuccess) break;
        const unsigned int keep = count < cap ? count : cap;
        if (keep && cudaMemcpy(pairs, dm, sizeof(uint2) * keep, cudaMemcpyDeviceToHost) != cudaSuccess) break;
        result = (long long)count;
    } while (0);
    cudaFree(da);
    cudaFree(db);
    cudaFree(dm);
    cudaFree(dn);
    if (launches) *launches = nl;
    return result;
}

}  // extern "C"
