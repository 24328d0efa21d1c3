/*
 * xmatch.h -- C ABI of the B200 zone crossmatch (libxmatch_b200.so).
 *
 * The reference (matthiaslee/Xmatch, BoostXmatch) has no plugin or FFI
 * surface; it is one executable whose internal boundary is the Segment data
 * contract, the Job contract and the Worker::Match / Sorter::Sort operators.
 * Each entry point below replaces one of those; the comment names the
 * reference interface (file:line, paths inside the BoostXmatch project).
 *
 * Conventions: every call returns an xm_status (XM_OK == 0), never throws,
 * and never aborts.  Host buffers are owned by the caller.  Device data
 * (segments, match results) is owned by the library and lives on the
 * context's GPU.  One xm_ctx per GPU; a context is not thread-safe (use one
 * per host thread), different contexts are independent.  Angles: degrees for
 * inputs (as in the .idradec file), radians for the reported distance.
 */
#ifndef XMATCH_B200_H
#define XMATCH_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int xm_status;
enum {
    XM_OK = 0,
    XM_ERR_INVALID = 1,      /* bad argument */
    XM_ERR_CUDA = 2,         /* CUDA runtime error (see xm_last_error) */
    XM_ERR_NOMEM = 3,        /* device or host allocation failed */
    XM_ERR_CAPACITY = 4,     /* output buffer too small; count holds the size needed */
    XM_ERR_MISMATCH = 5,     /* segments built with different zone heights */
    XM_ERR_NODEVICE = 6,     /* no usable CUDA device */
    XM_ERR_IO = 7,           /* file could not be read or written */
    XM_ERR_BUSY = 8,         /* serving queue full / request not finished */
    XM_ERR_TIMEOUT = 9,      /* a bounded wait ran out */
    XM_ERR_TOO_LARGE = 10    /* input exceeds a fixed capacity (xm_segment_build_noalloc) */
};

/* One .idradec record: 24 bytes, little endian (Obj.h:21-25). */
typedef struct xm_obj {
    int64_t id;
    double ra_deg;
    double dec_deg;
} xm_obj;

typedef struct xm_ctx xm_ctx;
typedef struct xm_segment xm_segment;

/* Pair-kernel variants (xm_match flags). */
enum {
    XM_FILTER32 = 0,          /* default: FP32 chord^2 reject with a proven margin,
                                 every surviving pair decided by the FP64 predicate */
    XM_PLAIN64 = 1u << 0,     /* all-FP64: FP64 cuts, unit vectors by sincos per pair */
    XM_COUNT_CAND = 1u << 1,  /* also count reference-prefilter candidates (stats.n_cand) */
    XM_NO_DIST = 1u << 2,     /* do not compute distances (16-byte output) */
    XM_NO_GRAPH = 1u << 3     /* launch the match kernels directly, not through the context's CUDA graph */
};

/* Stats may be NULL everywhere; when given, the call accumulates into it. */

/* Result buffers in HOST memory.  pairs holds (idA, idB) interleaved, i.e.
 * exactly the 16-byte records the reference writes (Worker.cu:407-420);
 * dist (radians, 2 asin(chord/2)) may be NULL.  If both pointers are NULL the
 * result stays on the device and only count is returned. */
typedef struct xm_pairs {
    int64_t *pairs;     /* [2 * capacity] */
    double *dist;       /* [capacity] or NULL */
    uint64_t capacity;  /* records the arrays can hold */
    uint64_t count;     /* out: number of matches */
} xm_pairs;

typedef struct xm_stats {
    uint64_t n_tested;     /* pairs the pair loop evaluated */
    uint64_t n_cand;       /* pairs passing dec + RA cuts (XM_COUNT_CAND) */
    uint64_t n_border;     /* FP32 value inside the margin band */
    uint64_t n_exact;      /* pairs decided by the FP64 predicate */
    uint64_t n_match;
    uint64_t n_tiles;
    uint32_t n_launches;   /* kernels launched by the call */
    uint32_t n_retries;    /* output-buffer growth re-runs */
    float ms_total;        /* device time of the call (CUDA events) */
    float ms_match;        /* device time of the pair kernel alone */
    float ms_build;        /* zone build (xm_segment_build*) */
    float ms_h2d, ms_d2h;
    /* zone-build passes: sort keys + digit histograms, histogram read-back,
       radix passes, gather into zone order + zone bounds */
    float ms_zb_count, ms_zb_scan, ms_zb_scatter, ms_zb_sort;
    float ms_plan;         /* tile pre-pass of the pair kernel (count, scans, plans) */
} xm_stats;

/* Tuning of the persistent pair kernel (0 = default / autotuned).  A work
 * item of `zones` consecutive A zones is cut into tiles of at most `tile`
 * objects; a block claims `chunk` tiles at a time. */
typedef struct xm_tuning {
    uint32_t tile;        /* A objects per tile (= consumer threads per block): 64, 128, 256 */
    uint32_t chunk;       /* tiles claimed per work-stealing step (1..32) */
    uint32_t blocks_per_sm;
    uint32_t zones;       /* zones per work item (1..64) */
} xm_tuning;

/* ---- context (replaces CudaManager / CudaContext, CudaManager.cpp:8-65) ---- */
xm_status xm_ctx_create(int device, xm_ctx **out);
xm_status xm_ctx_destroy(xm_ctx *ctx);
const char *xm_status_str(xm_status s);
const char *xm_last_error(const xm_ctx *ctx);
/* Library and device description, e.g. for logs. */
xm_status xm_ctx_info(const xm_ctx *ctx, int *device, int *sm_count, uint64_t *free_bytes,
                      uint64_t *total_bytes);
xm_status xm_ctx_synchronize(xm_ctx *ctx);
/* The cudaStream_t all work of this context is queued on (for callers that
 * time or order their own work against the library's). */
xm_status xm_ctx_stream(const xm_ctx *ctx, void **stream);

/* ---- zone builder (replaces Sorter::Sort, Sorter.cu:141-185) ----
 * Assigns dec zones of height zh_deg, sorts each zone by ra on the GPU and
 * keeps the sorted SoA (id, ra/dec radians, FP32 unit vector) resident.
 * Objects whose zone is outside [0, ceil(180/zh)) are dropped, except
 * dec = +90 which is kept in the last zone.  seg_id mirrors Segment::mId. */
xm_status xm_segment_build(xm_ctx *ctx, uint32_t seg_id, const xm_obj *host_objs,
                           uint64_t n, double zh_deg, xm_segment **out, xm_stats *stats);
/* Same, from records already in this context's device memory. */
xm_status xm_segment_build_device(xm_ctx *ctx, uint32_t seg_id, const xm_obj *dev_objs,
                                  uint64_t n, double zh_deg, xm_segment **out, xm_stats *stats);
/* Re-use seg's device storage for new records (no allocation if they fit). */
xm_status xm_segment_rebuild_device(xm_segment *seg, const xm_obj *dev_objs, uint64_t n,
                                    xm_stats *stats);
xm_status xm_segment_free(xm_segment *seg);
/* Segment fields (Segment.h:24-26): kept objects, zone count, zone height. */
xm_status xm_segment_info(const xm_segment *seg, uint32_t *seg_id, uint64_t *n_kept,
                          int32_t *n_zones, double *zh_deg);
/* ---- segments held in host memory (catalogs larger than device memory) ----
 * The reference keeps every segment in host RAM and copies the two of a job to
 * the GPU when the job runs (Worker.cu:251-292, BoostXmatch.cpp:247-274).
 * Here a built segment can be moved to pinned host memory and paged back in
 * per job; xm_match / xm_match_batch refuse an offloaded segment
 * (XM_ERR_INVALID).
 *   xm_segment_offload   copy the sorted arrays to pinned host memory (kept by
 *                        the segment) and free the device copy
 *   xm_segment_page_in   queue the copy back to device memory on the
 *                        context's second stream and return at once; work
 *                        queued on a context after that waits for the copy, so
 *                        paging the next job's segment in overlaps the current
 *                        match
 *   xm_segment_page_out  free the device copy (after the work already queued on
 *                        it), keeping the host copy
 *   xm_segment_resident  whether the arrays are in device memory, and their size
 * Rebuilding a segment drops its host copy. */
xm_status xm_segment_offload(xm_segment *seg);
xm_status xm_segment_page_in(xm_segment *seg);
xm_status xm_segment_page_out(xm_segment *seg);
xm_status xm_segment_resident(const xm_segment *seg, int *on_device, uint64_t *bytes);
/* Copy the sorted segment to the host, as Sorter.cu:178-182 fills
 * Segment::vId, vRadec, vZoneBegin, vZoneEnd.  Any pointer may be NULL.
 * radec: [2*n_kept] radians; zone_begin/zone_end: [n_zones]. */
xm_status xm_segment_export(const xm_segment *seg, int64_t *id, double *radec,
                            int32_t *zone_begin, int32_t *zone_end);

/* ---- match one job (replaces Worker::Match, Worker.cu:243-428, and the
 * kernel xmatch_kernel, Worker.cu:65-241) ----
 * Finds every (a in A, b in B) with b's zone within ceil(r/zh) zones of a's,
 * |dec_a - dec_b| < r, |ra_a - ra_b| (mod 2 pi branches) < alpha(zone_a) and
 * chord^2 < (2 sin(r/2))^2, all in FP64, each pair once, self-pairs kept. */
xm_status xm_match(xm_ctx *ctx, const xm_segment *A, const xm_segment *B, double sr_deg,
                   uint32_t flags, xm_pairs *out, xm_stats *stats);
/* Copy the device-resident result of the last xm_match / xm_match_batch of
 * this context to the host (first `out->capacity` records). */
xm_status xm_fetch_pairs(xm_ctx *ctx, xm_pairs *out);

/* ---- many jobs in one persistent launch (replaces JobManager + the worker
 * threads, JobManager.cpp:5-47, Worker.cu:430-485) ---- */
typedef struct xm_job {
    const xm_segment *A;
    const xm_segment *B;
    double sr_deg;
} xm_job;
/* outs[j] receives job j's pairs (host); job_counts[j] its count.  With
 * outs == NULL the results stay on the device, grouped by job. */
xm_status xm_match_batch(xm_ctx *ctx, const xm_job *jobs, uint32_t n_jobs, uint32_t flags,
                         const xm_tuning *tuning, xm_pairs *outs, uint64_t *job_counts,
                         xm_stats *stats);
/* Times the batch under the fixed tuning {tile 128, chunk 16, zones 16}
 * (*fixed_ms) and under 18 tile / chunk / zones settings, and returns the
 * fastest of all of them (*best, *best_ms <= *fixed_ms).  Replaces the
 * reference's fixed 16 x 16 launch geometry (Worker.cu:351-359). */
xm_status xm_autotune_batch(xm_ctx *ctx, const xm_job *jobs, uint32_t n_jobs, uint32_t flags,
                            xm_tuning *best, float *best_ms, float *fixed_ms);

/* Crossmatch of two catalogs in host memory (the whole of _main for one pair,
 * BoostXmatch.cpp:247-330, in one call): both are zone-built, B's host-to-device
 * copy overlapping A's copy and build, then matched.  If out's buffers are
 * pinned (cudaHostAlloc / cudaHostRegister) and hold every match, the pair
 * kernel writes the matches straight into them; otherwise they are copied.
 * XM_ERR_CAPACITY (out->count = matches) leaves the matches for xm_fetch_pairs. */
xm_status xm_crossmatch(xm_ctx *ctx, const xm_obj *A, uint64_t nA, const xm_obj *B, uint64_t nB, double sr_deg,
                        double zh_deg, uint32_t flags, xm_pairs *out, xm_stats *stats);

/* ---- serving: a resident catalog answering a stream of query catalogs ----
 * Replaces the reference's run-to-completion driver (_main,
 * BoostXmatch.cpp:247-330, which loads, sorts and matches one catalog pair
 * per process) with a request loop: the catalog segment stays in HBM, query
 * catalogs are queued by xm_serve_submit, admitted while their estimated
 * device memory fits the budget, zone-built on a second stream while the
 * previous batch is matched, and matched together in one persistent launch
 * (the xm_match_batch path, query = A side, catalog = B side).  Results are
 * the same as xm_match of the query segment against the catalog. */
typedef struct xm_server xm_server;
typedef struct xm_serve_cfg {
    uint64_t mem_budget;   /* device bytes for queries in flight; 0 = half the free memory at open */
    uint32_t max_batch;    /* queries per batch at most; 0 = 1024 */
    uint32_t flags;        /* match flags of every query (XM_FILTER32, XM_NO_DIST, ...) */
} xm_serve_cfg;
typedef struct xm_serve_info {
    double t_submit_ms;    /* host clock (ms since the server opened) at submit */
    double t_admit_ms;     /* admitted (memory reserved, build started) */
    double t_built_ms;     /* zone build finished, waiting for a batch */
    double t_batch_ms;     /* its batch taken by the matcher (pair kernel queued) */
    double t_matched_ms;   /* pair kernel of the batch finished, matches grouped */
    double t_done_ms;      /* results ready on the host */
    uint32_t batch;        /* batch number that matched it */
    uint32_t batch_size;   /* queries in that batch */
    uint64_t count;        /* matches */
} xm_serve_info;
/* Opens a server on a catalog built on ctx's device; the catalog must outlive
 * the server.  The server owns a second context (stream) for query builds and
 * two host threads; ctx must not be used by the caller until xm_serve_close. */
xm_status xm_serve_open(xm_ctx *ctx, const xm_segment *catalog, const xm_serve_cfg *cfg, xm_server **out);
/* Queues a query catalog (host records, copied) with its radius; returns at
 * once with a ticket.  XM_ERR_TOO_LARGE if the query alone exceeds the budget. */
xm_status xm_serve_submit(xm_server *srv, const xm_obj *objs, uint64_t n, double sr_deg, uint64_t *ticket);
/* Result of a ticket.  wait != 0 blocks until it is ready; otherwise XM_ERR_BUSY
 * while it is pending.  With out NULL or without buffers only out->count and
 * info are filled and the result is kept; XM_ERR_CAPACITY (out->count set,
 * result kept) when the buffers are too small; otherwise the matches are
 * copied and the ticket is released.  A failed query returns its error once. */
xm_status xm_serve_poll(xm_server *srv, uint64_t ticket, int wait, xm_pairs *out, xm_serve_info *info);
/* Message of the last failed query this server returned from xm_serve_poll,
 * copied into buf (at most cap bytes, NUL-terminated); safe to call from any
 * thread while the server runs. */
xm_status xm_serve_last_error(xm_server *srv, char *buf, uint64_t cap);
/* Finishes every queued query, stops the threads and frees the server. */
xm_status xm_serve_close(xm_server *srv);

/* ---- formats (Segment::Load, Segment.cpp:14-22; output, Worker.cu:407-420) ---- */
/* Number of 24-byte records in a .idradec file. */
xm_status xm_idradec_count(const char *path, uint64_t *n);
/* Read records [first, first + n) of a .idradec file into host memory. */
xm_status xm_idradec_read(const char *path, uint64_t first, uint64_t n, xm_obj *out);
xm_status xm_idradec_write(const char *path, const xm_obj *objs, uint64_t n);
/* Append pairs to a file: mode 16 = reference records {idA, idB};
 * mode 24 = {idA, idB, dist}; mode 0 = ASCII "idA idB dist\n". */
xm_status xm_pairs_write(const char *path, const xm_pairs *pairs, int mode, int append);

/* ---- zone build without any allocation ----
 * No counterpart in the reference.  For callers that may not allocate
 * device memory once they are running: a serving process that reserved its
 * HBM budget at start-up, or a host application whose device memory is owned
 * by another allocator.  Same result as xm_segment_build_device +
 * xm_segment_export (same sorted order), written to caller-owned device
 * arrays; the sort scratch is a fixed array inside the library
 * (XM_NOALLOC_MAX_OBJS records, about 25 MB of device memory, held by every
 * GPU that loads the library until the process exits).  Calls no cudaMalloc
 * or cudaFree and allocates nothing on the host heap.
 *   device        GPU to run on (current during the call; the caller's
 *                 current device is restored before it returns)
 *   stream        cudaStream_t to queue on (NULL = default stream); the call
 *                 returns after the work on it has completed
 *   dev_objs      n records in device memory, n <= XM_NOALLOC_MAX_OBJS,
 *                 larger n returns XM_ERR_TOO_LARGE
 *   out_id        int64  [n]      (first *n_kept used)
 *   out_radec     double [2 n]    ra, dec radians
 *   out_xyz       float  [4 n]    FP32 unit vector, w = quantised-ra bits
 *   out_zone_off  uint32 [n_zones + 1], n_zones = ceil(180 / zh_deg), given
 *                 in zone_off_cap; zone z holds [out_zone_off[z], out_zone_off[z+1])
 * The first call on a device looks up the scratch array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * Every call uses the same scratch: calls that overlap on the GPU (from
 * several host threads or streams) race, so serialise them per device. */
#define XM_NOALLOC_MAX_OBJS (1u << 20)
xm_status xm_segment_build_noalloc(int device, void *stream, const xm_obj *dev_objs, uint64_t n,
                                   double zh_deg, int64_t *out_id, double *out_radec, float *out_xyz,
                                   uint32_t *out_zone_off, uint64_t zone_off_cap, uint64_t *n_kept);

/* ---- utilities ---- */
/* FP64 unit vectors of (ra, dec) in degrees computed on the GPU exactly as
 * the zone builder does (xyz: [3*n] host). */
xm_status xm_unit_vectors(xm_ctx *ctx, const double *ra_deg, const double *dec_deg, uint64_t n,
                          double *xyz);
/* RA half-width of Common.cu:17-23 for every zone, as the library uses it. */
xm_status xm_alpha_table(double sr_deg, double zh_deg, double *alpha, int32_t n_zones);
/* The FP32 chord^2 thresholds XM_FILTER32 uses at radius sr_deg: a pair whose
 * FP32 chord^2 (from the FP32 unit vectors, fused sum of squares) exceeds
 * *thr_hi cannot match; one below *thr_lo matches whenever the RA half-width
 * of A's zone is below 3 rad (0 when the radius is too small for that). */
xm_status xm_filter_bounds(double sr_deg, float *thr_hi, float *thr_lo);

#ifdef __cplusplus
}
#endif
#endif /* XMATCH_B200_H */
