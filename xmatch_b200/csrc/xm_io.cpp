// xm_io.cpp -- the reference's file formats.
//   .idradec : headerless 24-byte records {int64 id; f64 ra; f64 dec}
//              (Obj.h:21-25, read raw by Segment::Load, Segment.cpp:14-22)
//   pairs    : headerless 16-byte records {int64 idA; int64 idB}
//              (Worker.cu:407-420), or 24-byte {idA, idB, f64 dist}, or ASCII
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <unistd.h>

#include "../../include/xmatch.h"

extern "C" xm_status xm_idradec_count(const char *path, uint64_t *n)
{
    if (!path || !n) return XM_ERR_INVALID;
    FILE *f = std::fopen(path, "rb");
    if (!f) return XM_ERR_IO;
    if (std::fseek(f, 0, SEEK_END) != 0) {
        std::fclose(f);
        return XM_ERR_IO;
    }
    long long sz = ftello(f);
    std::fclose(f);
    if (sz < 0) return XM_ERR_IO;
    *n = (uint64_t)sz / sizeof(xm_obj);
    return XM_OK;
}

// Records [first, first + n) straight into the caller's buffer (pinned memory
// included) with pread(2) in 64 MB pieces, by up to 8 threads at once for a
// large read: from the page cache one thread copies a few GB/s, below what the
// link to the GPU takes.
extern "C" xm_status xm_idradec_read(const char *path, uint64_t first, uint64_t n, xm_obj *out)
{
    if (!path || (n && !out)) return XM_ERR_INVALID;
    const int fd = ::open(path, O_RDONLY | O_CLOEXEC);
    if (fd < 0) return XM_ERR_IO;
    const uint64_t bytes = n * sizeof(xm_obj);
    const off_t base = (off_t)(first * sizeof(xm_obj));
    constexpr uint64_t kPiece = 64ull << 20;
    const uint64_t pieces = (bytes + kPiece - 1) / kPiece;
    std::atomic<uint64_t> next{0};
    std::atomic<bool> ok{true};
    auto work = [&] {
        for (uint64_t k; ok.load(std::memory_order_relaxed) && (k = next.fetch_add(1)) < pieces;) {
            uint64_t done = k * kPiece;
            const uint64_t end = std::min(bytes, done + kPiece);
            while (done < end) {
                const ssize_t r = ::pread(fd, reinterpret_cast<char *>(out) + done, end - done, base + (off_t)done);
                if (r < 0 && errno == EINTR) continue;
                if (r <= 0) {   // error, or the file ends before the records asked for
                    ok = false;
                    break;
                }
                done += (uint64_t)r;
            }
        }
    };
    const unsigned nt = (unsigned)std::min<uint64_t>(8, pieces);
    if (nt <= 1) {
        work();
    } else {
        std::vector<std::thread> th;
        for (unsigned i = 0; i < nt; ++i) th.emplace_back(work);
        for (auto &t : th) t.join();
    }
    ::close(fd);
    return ok ? XM_OK : XM_ERR_IO;
}

extern "C" xm_status xm_idradec_write(const char *path, const xm_obj *objs, uint64_t n)
{
    if (!path || (n && !objs)) return XM_ERR_INVALID;
    FILE *f = std::fopen(path, "wb");
    if (!f) return XM_ERR_IO;
    size_t put = std::fwrite(objs, sizeof(xm_obj), n, f);
    int rc = std::fclose(f);
    return (put == n && rc == 0) ? XM_OK : XM_ERR_IO;
}

extern "C" xm_status xm_pairs_write(const char *path, const xm_pairs *p, int mode, int append)
{
    if (!path || !p || (p->count && !p->pairs)) return XM_ERR_INVALID;
    if (mode != 16 && mode != 24 && mode != 0) return XM_ERR_INVALID;
    if (mode != 16 && p->count && !p->dist) return XM_ERR_INVALID;
    if (p->count > p->capacity) return XM_ERR_CAPACITY;
    FILE *f = std::fopen(path, append ? "ab" : "wb");
    if (!f) return XM_ERR_IO;
    bool ok = true;
    if (mode == 16) {
        // identical bytes to the reference's per-record writes (Worker.cu:413-417)
        ok = std::fwrite(p->pairs, 16, p->count, f) == p->count;
    } else if (mode == 24) {
        const uint64_t B = 1 << 16;
        std::vector<unsigned char> buf(B * 24);
        for (uint64_t s = 0; s < p->count && ok; s += B) {
            uint64_t m = std::min<uint64_t>(B, p->count - s);
            for (uint64_t i = 0; i < m; ++i) {
                std::memcpy(&buf[i * 24], &p->pairs[2 * (s + i)], 16);
                std::memcpy(&buf[i * 24 + 16], &p->dist[s + i], 8);
            }
            ok = std::fwrite(buf.data(), 24, m, f) == m;
        }
    } else {
        for (uint64_t i = 0; i < p->count && ok; ++i)
            ok = std::fprintf(f, "%lld %lld %.17g\n", (long long)p->pairs[2 * i], (long long)p->pairs[2 * i + 1],
                              p->dist[i]) > 0;
    }
    if (std::fclose(f) != 0) ok = false;
    return ok ? XM_OK : XM_ERR_IO;
}
