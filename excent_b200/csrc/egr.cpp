// egr.cpp -- EgrFile (egr.h) and its C entry points.
#include "egr.h"

#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstring>

#include "common.h"

namespace excent {

EgrFile::~EgrFile() {
    if (map_ && map_ != MAP_FAILED) munmap(map_, map_size_);
    if (fd_ >= 0) ::close(fd_);
}

int EgrFile::read_exact(void* dst, size_t bytes, size_t off) const {
    char* p = (char*)dst;
    while (bytes) {
        const ssize_t r = pread(fd_, p, bytes, (off_t)off);
        if (r < 0 && errno == EINTR) continue;
        if (r <= 0) return EXCENT_ERR_IO;
        p += r;
        off += (size_t)r;
        bytes -= (size_t)r;
    }
    return EXCENT_OK;
}

// 8 MiB pieces over up to io_threads threads (include/StaticGraph.h:160-170).
int EgrFile::read_parallel(void* dst, size_t bytes, size_t off) const {
    const size_t piece = 8ull << 20;
    const long long pieces = (long long)((bytes + piece - 1) / piece);
    const int threads = (int)std::min<long long>(io_threads_, std::max<long long>(1, pieces));
    std::atomic<int> bad{0};
#pragma omp parallel for num_threads(threads) schedule(static, 1)
    for (long long i = 0; i < pieces; i++) {
        const size_t b = (size_t)i * piece;
        if (read_exact((char*)dst + b, std::min(piece, bytes - b), off + b) != EXCENT_OK) bad = 1;
    }
    return bad ? EXCENT_ERR_IO : EXCENT_OK;
}

int EgrFile::open(const char* path, int io_threads, bool offsets_in_ram, bool validate) {
    io_threads_ = std::max(1, io_threads);
    fd_ = ::open(path, O_RDONLY);
    if (fd_ < 0) EX_FAIL(EXCENT_ERR_IO, "%s: %s", path, strerror(errno));
    struct stat st;
    if (fstat(fd_, &st) != 0) EX_FAIL(EXCENT_ERR_IO, "%s: %s", path, strerror(errno));
    const size_t fsize = (size_t)st.st_size;
    int32_t hdr[2];
    if (fsize < sizeof hdr || read_exact(hdr, sizeof hdr, 0) != EXCENT_OK)
        EX_FAIL(EXCENT_ERR_IO, "%s: short header", path);
    n = hdr[0];
    size_t off = sizeof hdr;
    wide = hdr[1] == -1;
    if (wide) {
        int64_t mm = 0;
        if (read_exact(&mm, sizeof mm, off) != EXCENT_OK) EX_FAIL(EXCENT_ERR_IO, "%s: short header", path);
        if (mm < 0) EX_FAIL(EXCENT_ERR_IO, "%s: bad header (negative edge count)", path);
        m = (ull)mm;
        off += sizeof mm;
    } else {
        if (hdr[1] < 0) EX_FAIL(EXCENT_ERR_IO, "%s: bad header (edge count %d)", path, hdr[1]);
        m = (ull)hdr[1];
    }
    if (n < 1) EX_FAIL(EXCENT_ERR_IO, "StaticGraph: bad header in %s", path);
    idx_off_ = off;
    const size_t ib = ((size_t)n + 1) * (wide ? sizeof(ull) : sizeof(int32_t));
    nlist_off_ = off + ib;
    if (fsize < nlist_off_ + m * sizeof(int32_t))
        EX_FAIL(EXCENT_ERR_IO, "%s: truncated (%zu bytes, header needs %llu)", path, fsize,
                (ull)(nlist_off_ + m * sizeof(int32_t)));
    if (!wide) offsets_in_ram = true;
    if (offsets_in_ram) {
        ram_off_.resize((size_t)n + 1);
        if (wide) {
            if (read_parallel(ram_off_.data(), ib, off) != EXCENT_OK) EX_FAIL(EXCENT_ERR_IO, "%s: pread of offsets failed", path);
        } else {
            std::vector<uint32_t> tmp((size_t)n + 1);
            if (read_parallel(tmp.data(), ib, off) != EXCENT_OK) EX_FAIL(EXCENT_ERR_IO, "%s: pread of offsets failed", path);
            for (size_t i = 0; i < tmp.size(); i++) ram_off_[i] = tmp[i];
        }
    }
    map_size_ = fsize;
    map_ = mmap(nullptr, map_size_, PROT_READ, MAP_SHARED, fd_, 0);
    if (map_ == MAP_FAILED) { map_ = nullptr; EX_FAIL(EXCENT_ERR_IO, "mmap %s: %s", path, strerror(errno)); }
    madvise(map_, map_size_, MADV_RANDOM);
    posix_fadvise(fd_, 0, 0, POSIX_FADV_SEQUENTIAL);
    nlist_ = (const int32_t*)((const char*)map_ + nlist_off_);
    off_ = offsets_in_ram ? ram_off_.data() : (const ull*)((const char*)map_ + idx_off_);
    if (validate) {
        if (off_[0] != 0 || off_[n] != m) EX_FAIL(EXCENT_ERR_IO, "%s: offsets do not span [0, m]", path);
        std::atomic<long long> bad{-1};
#pragma omp parallel for num_threads(io_threads_) schedule(static)
        for (long long v = 0; v < n; v++)
            if (off_[v] > off_[v + 1]) bad = v;
        if (bad >= 0) EX_FAIL(EXCENT_ERR_IO, "%s: offsets decrease at vertex %lld", path, (long long)bad);
    }
    return EXCENT_OK;
}

int EgrFile::read_offsets(size_t v0, size_t cnt, ull* dst) const {
    if (v0 + cnt > (size_t)n + 1) EX_FAIL(EXCENT_ERR_ARG, "offsets out of range");
    if (!ram_off_.empty()) { memcpy(dst, ram_off_.data() + v0, cnt * sizeof(ull)); return EXCENT_OK; }
    if (read_parallel(dst, cnt * sizeof(ull), idx_off_ + v0 * sizeof(ull)) != EXCENT_OK)
        EX_FAIL(EXCENT_ERR_IO, "pread of offsets failed");
    return EXCENT_OK;
}

int EgrFile::read_edges(ull e0, ull e1, int32_t* dst) const {
    if (e0 > e1 || e1 > m) EX_FAIL(EXCENT_ERR_ARG, "edge range out of bounds");
    if (read_parallel(dst, (e1 - e0) * sizeof(int32_t), nlist_off_ + e0 * sizeof(int32_t)) != EXCENT_OK)
        EX_FAIL(EXCENT_ERR_IO, "pread of edges [%llu, %llu) failed", e0, e1);
    return EXCENT_OK;
}

// Merge each part's page runs and request them once (include/StaticGraph.h:90-114).
void EgrFile::prefetch_lists(const int32_t* vids, int k, ull* pages, ull* runs) const {
    const size_t P = (size_t)sysconf(_SC_PAGESIZE);
    ull np = 0, nr = 0;
    const int parts = std::max(1, std::min(io_threads_, k / 1024));
#pragma omp parallel for num_threads(parts) reduction(+ : np, nr) schedule(static, 1)
    for (int t = 0; t < parts; t++) {
        const int i0 = (int)((long long)k * t / parts), i1 = (int)((long long)k * (t + 1) / parts);
        size_t r0 = 0, r1 = 0;
        bool open = false;
        auto flush = [&]() {
            if (!open) return;
            madvise((char*)map_ + r0 * P, (r1 - r0) * P, MADV_WILLNEED);
            np += r1 - r0;
            nr++;
        };
        for (int i = i0; i < i1; i++) {
            const ull d = degree(vids[i]);
            if (!d) continue;
            const size_t b0 = nlist_off_ + off_[vids[i]] * sizeof(int32_t), b1 = b0 + d * sizeof(int32_t);
            const size_t p0 = b0 / P, p1 = (b1 + P - 1) / P;
            if (open && p0 <= r1) r1 = std::max(r1, p1);
            else { flush(); r0 = p0; r1 = p1; open = true; }
        }
        flush();
    }
    *pages = np;
    *runs = nr;
}

// Unmap our pages and drop them from the page cache (include/StaticGraph.h:116-126).
void EgrFile::drop_cache(ull e0, ull e1, size_t v0, size_t v1) const {
    const size_t P = (size_t)sysconf(_SC_PAGESIZE);
    auto drop = [&](size_t b0, size_t b1) {
        const size_t a0 = b0 / P * P, a1 = std::min(map_size_, (b1 + P - 1) / P * P);
        if (a1 <= a0) return;
        madvise((char*)map_ + a0, a1 - a0, MADV_DONTNEED);
        posix_fadvise(fd_, (off_t)a0, (off_t)(a1 - a0), POSIX_FADV_DONTNEED);
    };
    drop(nlist_off_ + e0 * sizeof(int32_t), nlist_off_ + e1 * sizeof(int32_t));
    const size_t w = wide ? sizeof(ull) : sizeof(int32_t);
    drop(idx_off_ + v0 * w, idx_off_ + (v1 + 1) * w);
}

}  // namespace excent

using namespace excent;

struct excent_egr { EgrFile f; };

extern "C" int excent_egr_open(const char* path, int io_threads, int offsets_in_ram, excent_egr** out) {
    EX_CHECK_ARG(path && out, "null argument");
    *out = nullptr;
    excent_egr* g = new excent_egr();
    const int rc = g->f.open(path, io_threads, offsets_in_ram != 0, true);
    if (rc != EXCENT_OK) { delete g; return rc; }
    *out = g;
    return EXCENT_OK;
}
extern "C" int excent_egr_close(excent_egr* g) { delete g; return EXCENT_OK; }
extern "C" int excent_egr_info(excent_egr* g, int* n, unsigned long long* m, int* wide) {
    EX_CHECK_ARG(g, "null file");
    if (n) *n = g->f.n;
    if (m) *m = g->f.m;
    if (wide) *wide = g->f.wide;
    return EXCENT_OK;
}
extern "C" int excent_egr_read_offsets(excent_egr* g, unsigned long long v0, unsigned long long count,
                                       unsigned long long* dst) {
    EX_CHECK_ARG(g && dst, "null argument");
    return g->f.read_offsets(v0, count, dst);
}
extern "C" int excent_egr_read_edges(excent_egr* g, unsigned long long e0, unsigned long long e1, int32_t* dst) {
    EX_CHECK_ARG(g && (dst || e0 == e1), "null argument");
    return g->f.read_edges(e0, e1, dst);
}
extern "C" int excent_egr_prefetch(excent_egr* g, const int32_t* vids, int k, unsigned long long* pages,
                                   unsigned long long* runs) {
    EX_CHECK_ARG(g && pages && runs && (vids || k == 0), "null argument");
    for (int i = 0; i < k; i++) EX_CHECK_ARG(vids[i] >= 0 && vids[i] < g->f.n, "vertex %d out of range", vids[i]);
    g->f.prefetch_lists(vids, k, pages, runs);
    return EXCENT_OK;
}
extern "C" int excent_egr_drop_cache(excent_egr* g, unsigned long long e0, unsigned long long e1,
                                     unsigned long long v0, unsigned long long v1) {
    EX_CHECK_ARG(g && e0 <= e1 && e1 <= g->f.m && v0 <= v1 && v1 <= (ull)g->f.n, "bad range");
    g->f.drop_cache(e0, e1, v0, v1);
    return EXCENT_OK;
}
