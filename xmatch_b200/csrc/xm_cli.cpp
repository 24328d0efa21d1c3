// xm_cli.cpp -- command-line driver on the C ABI with the options and the flow
// of BoostXmatch.x (options BoostXmatch.cpp:102-118, flow _main :218-330):
//
//   xmatch [-r arcsec] [-z arcsec] [-n objects] [-t gpus] [-m maxout]
//          [-o outdir] [-x] [-v [level]] [--dist] fileA fileB
//
// fileA (the file held in memory; pass the smaller one first) is cut into
// segments of -n objects and zone-built on every GPU used; fileB is read in
// rounds of one segment per GPU.  On each GPU a worker thread matches every A
// segment against its B segment and writes the pairs of the round to
// outdir/<wid> (wid counts workers over rounds, as BoostXmatch.cpp:312-320),
// 16-byte {idA, idB} records as Worker.cu:413-417 (--dist: 24-byte records
// with the distance in radians).  While a round is matched, the worker's
// second context reads and zone-builds its next B segment, so file reads,
// host-to-device copies and builds overlap the matching.
//
// A's segments stay in device memory when they fit --resident-mb (default:
// 60 % of the GPU's free memory); the round is then one batch launch of all
// of them.  Otherwise, as the reference does with its host-resident segments
// (BoostXmatch.cpp:247-274, Worker.cu:251-292), they are kept in pinned host
// memory and paged in one job at a time, the next A segment's copy
// overlapping the current match; rounds alternate the order of the A segments
// so that the last one of a round is still on the device for the first job of
// the next (the reference's job affinity, JobManager.cpp:16-41).
//
// Differences: the output directory must not exist unless -x is given (the
// reference asks on the terminal); -m caps the pairs written per job and
// reports any cut on stderr (the reference drops them silently when its
// buffer is full); without -n every file is one segment.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <string>
#include <thread>
#include <vector>

#include "xmatch.h"

namespace {

struct Options {
    double r_arcsec = 5, zh_arcsec = 0;
    uint64_t numobj = 0, maxout = 0;
    double resident_mb = -1;   // device MiB for fileA's segments; < 0 = 60 % of the free memory
    uint32_t threads = 0;
    int verbose = 0;
    bool overwrite = false, dist = false;
    std::string outdir;
    std::vector<std::string> inputs;
};

void usage(FILE *f)
{
    std::fprintf(f,
                 "usage: xmatch [options] fileA fileB\n"
                 "  -r, --radius ARCSEC      search radius (default 5)\n"
                 "  -z, --zoneheight ARCSEC  zone height (default: the radius)\n"
                 "  -n, --numobj N           objects per segment (default: the whole file)\n"
                 "  -t, --threads N          GPUs to use (default: all)\n"
                 "  -m, --maxout N           at most N pairs written per job (default: all)\n"
                 "  -o, --outdir DIR         write pairs to DIR/<worker id>\n"
                 "  -x, --overwrite          allow an existing output directory\n"
                 "  -v, --verbose [LEVEL]    progress on stderr\n"
                 "      --dist               24-byte records {idA, idB, distance}\n"
                 "      --resident-mb MIB    device memory fileA's segments may hold (default: 60%% of the\n"
                 "                           free memory); beyond it they are paged in from host memory per job\n"
                 "  -h, --help\n"
                 "fileA is held in memory (pass the smaller file first), fileB is looped over.\n");
}

bool parse(int argc, char **argv, Options &o, int &rc)
{
    auto value = [&](int &i, const char *name) -> const char * {
        if (i + 1 >= argc) {
            std::fprintf(stderr, "xmatch: %s needs a value\n", name);
            return nullptr;
        }
        return argv[++i];
    };
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        const char *v = nullptr;
        if (a == "-h" || a == "--help") {
            usage(stdout);
            rc = 0;
            return false;
        } else if (a == "-r" || a == "--radius") {
            if (!(v = value(i, "-r"))) break;
            o.r_arcsec = std::atof(v);
        } else if (a == "-z" || a == "--zoneheight") {
            if (!(v = value(i, "-z"))) break;
            o.zh_arcsec = std::atof(v);
        } else if (a == "-n" || a == "--numobj") {
            if (!(v = value(i, "-n"))) break;
            o.numobj = std::strtoull(v, nullptr, 10);
        } else if (a == "-t" || a == "--threads") {
            if (!(v = value(i, "-t"))) break;
            o.threads = (uint32_t)std::strtoul(v, nullptr, 10);
        } else if (a == "-m" || a == "--maxout") {
            if (!(v = value(i, "-m"))) break;
            o.maxout = std::strtoull(v, nullptr, 10);
        } else if (a == "-o" || a == "--outdir") {
            if (!(v = value(i, "-o"))) break;
            o.outdir = v;
        } else if (a.rfind("--outdir=", 0) == 0) {
            o.outdir = a.substr(9);
        } else if (a == "-x" || a == "--overwrite") {
            o.overwrite = true;
        } else if (a == "--dist") {
            o.dist = true;
        } else if (a == "--resident-mb") {
            if (!(v = value(i, "--resident-mb"))) break;
            o.resident_mb = std::atof(v);
        } else if (a == "-v" || a == "--verbose") {
            o.verbose = 9;
            if (i + 1 < argc && argv[i + 1][0] >= '0' && argv[i + 1][0] <= '9') o.verbose = std::atoi(argv[++i]);
        } else if (!a.empty() && a[0] == '-') {
            std::fprintf(stderr, "xmatch: unknown option %s\n", a.c_str());
            rc = 1;
            return false;
        } else {
            o.inputs.push_back(a);
        }
    }
    if (o.inputs.size() != 2) {
        usage(stderr);
        rc = 1;
        return false;
    }
    if (!(o.r_arcsec > 0) || o.zh_arcsec < 0) {
        std::fprintf(stderr, "xmatch: the radius must be positive and the zone height not negative\n");
        rc = 1;
        return false;
    }
    if (o.zh_arcsec == 0) o.zh_arcsec = o.r_arcsec;   // BoostXmatch.cpp:158
    return true;
}

bool check(xm_status s, const char *what, xm_ctx *ctx = nullptr)
{
    if (s == XM_OK) return true;
    std::fprintf(stderr, "xmatch: %s: %s%s%s\n", what, xm_status_str(s), ctx ? ": " : "", ctx ? xm_last_error(ctx) : "");
    return false;
}

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Reads records [first, first + n) of a file and zone-builds them on ctx.
xm_status load_segment(xm_ctx *ctx, const std::string &path, uint64_t first, uint64_t n, uint32_t id, double zh_deg,
                       xm_segment **out)
{
    std::vector<xm_obj> h(n);
    xm_status s = xm_idradec_read(path.c_str(), first, n, h.data());
    if (s != XM_OK) return s;
    return xm_segment_build(ctx, id, h.data(), n, zh_deg, out, nullptr);
}

struct Worker {
    int device = 0;
    xm_ctx *mctx = nullptr, *bctx = nullptr;   // matching, building the next B segment
    std::vector<xm_segment *> A;               // resident A segments
    int rc = 0;
    uint64_t matches = 0;
};

}  // namespace

int main(int argc, char **argv)
{
    Options o;
    int rc = 1;
    if (!parse(argc, argv, o, rc)) return rc;
    const double r_deg = o.r_arcsec / 3600, zh_deg = o.zh_arcsec / 3600;
    const std::string &fa = o.inputs[0], &fb = o.inputs[1];
    uint64_t na = 0, nb = 0;
    if (!check(xm_idradec_count(fa.c_str(), &na), fa.c_str()) || !check(xm_idradec_count(fb.c_str(), &nb), fb.c_str()))
        return 1;
    if (nb < na)
        std::fprintf(stderr, "xmatch: warning: fileA (%s) is the larger file; it is the one held in memory, pass "
                     "the smaller file first to hold less\n", fa.c_str());
    const uint64_t seg_a = o.numobj ? o.numobj : std::max<uint64_t>(na, 1);
    const uint64_t seg_b = o.numobj ? o.numobj : std::max<uint64_t>(nb, 1);
    if (!o.outdir.empty()) {
        struct stat sb;
        if (stat(o.outdir.c_str(), &sb) == 0 && !o.overwrite) {
            std::fprintf(stderr, "xmatch: output directory %s exists (use -x to overwrite)\n", o.outdir.c_str());
            return 1;
        }
        if (mkdir(o.outdir.c_str(), 0777) != 0 && stat(o.outdir.c_str(), &sb) != 0) {
            std::fprintf(stderr, "xmatch: cannot create %s\n", o.outdir.c_str());
            return 1;
        }
    }
    // one worker per GPU (BoostXmatch.cpp:225-227: threads default to the GPU count)
    std::vector<Worker> W;
    for (int d = 0;; ++d) {
        if (o.threads && W.size() >= o.threads) break;
        xm_ctx *m = nullptr, *b = nullptr;
        if (xm_ctx_create(d, &m) != XM_OK) break;
        if (xm_ctx_create(d, &b) != XM_OK) {
            xm_ctx_destroy(m);
            break;
        }
        Worker w;
        w.device = d;
        w.mctx = m;
        w.bctx = b;
        W.push_back(w);
    }
    if (W.empty()) {
        std::fprintf(stderr, "xmatch: no usable GPU\n");
        return 1;
    }
    const uint32_t T = (uint32_t)W.size();
    const double t0 = now_s();
    // A: all segments on every GPU (BoostXmatch.cpp:246-272), in device memory
    // when they fit the budget, else in pinned host memory
    uint64_t free_b = 0;
    xm_ctx_info(W[0].mctx, nullptr, nullptr, &free_b, nullptr);
    const double budget = o.resident_mb >= 0 ? o.resident_mb * 1048576.0 : 0.6 * (double)free_b;
    const uint64_t n_aseg = na ? (na + seg_a - 1) / seg_a : 1;
    const double a_bytes = 40.0 * (double)na + 4.0 * (std::ceil(180 / zh_deg) + 8) * (double)n_aseg;
    const bool paged = a_bytes > budget;
    uint32_t sid = 0;
    for (uint64_t first = 0; first < na || (na == 0 && first == 0); first += seg_a) {
        const uint64_t n = std::min<uint64_t>(seg_a, na - first);
        for (Worker &w : W) {
            xm_segment *s = nullptr;
            if (!check(load_segment(w.mctx, fa, first, n, sid, zh_deg, &s), "building a segment of fileA", w.mctx))
                return 1;
            if (paged && !check(xm_segment_offload(s), "moving a segment of fileA to host memory", w.mctx)) return 1;
            w.A.push_back(s);
        }
        ++sid;
        if (na == 0) break;
    }
    if (o.verbose)
        std::fprintf(stderr, "xmatch: %s: %zu segment(s) of at most %llu objects on %u GPU(s) (%s), %.3f s\n",
                     fa.c_str(), W[0].A.size(), (unsigned long long)seg_a, T,
                     paged ? "in host memory, paged in per job" : "resident in device memory", now_s() - t0);
    // B: rounds of one segment per GPU (BoostXmatch.cpp:278-327)
    const uint64_t n_bseg = nb ? (nb + seg_b - 1) / seg_b : 0;
    const uint64_t rounds = (n_bseg + T - 1) / T;
    auto work = [&](uint32_t g) {
        Worker &w = W[g];
        auto build = [&](uint64_t k) -> std::pair<xm_status, xm_segment *> {   // B segment k on the build context
            xm_segment *s = nullptr;
            const uint64_t first = k * seg_b, n = std::min<uint64_t>(seg_b, nb - first);
            xm_status st = load_segment(w.bctx, fb, first, n, (uint32_t)(sid + k), zh_deg, &s);
            return {st, s};
        };
        std::future<std::pair<xm_status, xm_segment *>> next;
        if (g < n_bseg) next = std::async(std::launch::async, build, (uint64_t)g);
        for (uint64_t round = 0; round < rounds; ++round) {
            const uint64_t k = round * T + g;
            if (k >= n_bseg) break;
            auto got = next.get();
            if (!check(got.first, "building a segment of fileB", w.bctx)) {
                w.rc = 1;
                return;
            }
            xm_segment *B = got.second;
            if (k + T < n_bseg) next = std::async(std::launch::async, build, k + T);
            const std::string path = o.outdir.empty() ? std::string() : o.outdir + "/" + std::to_string(round * T + g);
            bool first_write = true;
            uint64_t total = 0;
            // one batch launch of the given A segments against B; pairs appended to the round's file
            auto run = [&](const std::vector<size_t> &aseg) -> bool {
                std::vector<xm_job> jobs;
                for (size_t a : aseg) jobs.push_back({w.A[a], B, r_deg});
                std::vector<uint64_t> cnt(jobs.size());
                xm_status st = xm_match_batch(w.mctx, jobs.data(), (uint32_t)jobs.size(),
                                              o.dist ? XM_FILTER32 : XM_FILTER32 | XM_NO_DIST, nullptr, nullptr,
                                              cnt.data(), nullptr);
                if (!check(st, "matching", w.mctx)) return false;
                uint64_t n_b = 0;
                for (uint64_t c : cnt) n_b += c;
                // the batch's matches stay on the device grouped by job; one copy brings them over
                std::vector<int64_t> pairs(2 * std::max<uint64_t>(n_b, 1));
                std::vector<double> dist(o.dist ? std::max<uint64_t>(n_b, 1) : 0);
                xm_pairs all = {pairs.data(), o.dist ? dist.data() : nullptr, n_b, 0};
                if (n_b && !check(xm_fetch_pairs(w.mctx, &all), "fetching matches", w.mctx)) return false;
                total += n_b;
                if (path.empty()) return true;
                uint64_t off = 0;
                for (size_t j = 0; j < jobs.size(); ++j) {
                    xm_pairs p = {pairs.data() + 2 * off, o.dist ? dist.data() + off : nullptr, cnt[j], cnt[j]};
                    off += cnt[j];
                    if (o.maxout && p.count > o.maxout) {
                        std::fprintf(stderr, "xmatch: job (A %zu, B %llu): %llu pairs, %llu written (-m)\n",
                                     aseg[j], (unsigned long long)k, (unsigned long long)p.count,
                                     (unsigned long long)o.maxout);
                        p.count = o.maxout;
                    }
                    if (!check(xm_pairs_write(path.c_str(), &p, o.dist ? 24 : 16, first_write ? 0 : 1),
                               path.c_str()))
                        return false;
                    first_write = false;
                }
                return true;
            };
            const size_t S = w.A.size();
            bool ok = true;
            if (!paged) {
                std::vector<size_t> all(S);
                for (size_t a = 0; a < S; ++a) all[a] = a;
                ok = run(all);
            } else {
                // one A segment at a time, the next one's page-in queued before the current match;
                // odd rounds walk the A segments backwards, so the first job reuses the last one
                std::vector<size_t> order(S);
                for (size_t q = 0; q < S; ++q) order[q] = (round & 1) ? S - 1 - q : q;
                ok = check(xm_segment_page_in(w.A[order[0]]), "paging in a segment of fileA", w.mctx);
                for (size_t q = 0; ok && q < S; ++q) {
                    if (q + 1 < S)
                        ok = check(xm_segment_page_in(w.A[order[q + 1]]), "paging in a segment of fileA", w.mctx);
                    ok = ok && run({order[q]});
                    if (ok && q + 1 < S)
                        ok = check(xm_segment_page_out(w.A[order[q]]), "paging out a segment of fileA", w.mctx);
                }
            }
            if (!ok) {
                w.rc = 1;
                return;
            }
            w.matches += total;
            xm_segment_free(B);
            if (o.verbose)
                std::fprintf(stderr, "xmatch: GPU %d round %llu: %llu pairs\n", w.device, (unsigned long long)round,
                             (unsigned long long)total);
        }
    };
    std::vector<std::thread> th;
    for (uint32_t g = 0; g < T; ++g) th.emplace_back(work, g);
    for (auto &t : th) t.join();
    uint64_t matches = 0;
    rc = 0;
    for (Worker &w : W) {
        matches += w.matches;
        rc |= w.rc;
        for (xm_segment *s : w.A) xm_segment_free(s);
        xm_ctx_destroy(w.mctx);
        xm_ctx_destroy(w.bctx);
    }
    if (o.verbose)
        std::fprintf(stderr, "xmatch: %llu pairs in %.3f s\n", (unsigned long long)matches, now_s() - t0);
    return rc;
}
