// egr.cpp -- GraphFile (egr.h) and the excent_egr_* C entry points.
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

namespace {

constexpr size_t kPiece = size_t(8) << 20;   // bytes per positional read of a bulk range

// What the first bytes of an EGR file say, before anything is mapped.
struct Header {
    int32_t n = 0;
    ull m = 0;
    bool wide = false;
    size_t offsets_at = 0, entries_at = 0;
};

size_t page_bytes() { return (size_t)sysconf(_SC_PAGESIZE); }

}  // namespace

GraphFile::~GraphFile() {
    if (map_.base) munmap(map_.base, map_.bytes);
    if (fd_ >= 0) ::close(fd_);
}

// One positional read of exactly `bytes` (retried on short reads and EINTR).
int GraphFile::pread_all(void* dst, size_t bytes, size_t at) const {
    char* out = static_cast<char*>(dst);
    size_t done = 0;
    while (done < bytes) {
        const ssize_t got = pread(fd_, out + done, bytes - done, (off_t)(at + done));
        if (got < 0 && errno == EINTR) continue;
        if (got <= 0) return EXCENT_ERR_IO;
        done += (size_t)got;
    }
    return EXCENT_OK;
}

// A bulk range: the reader team claims 8 MiB pieces from a shared cursor
// until none is left, so a slow piece does not hold back a fixed share.
int GraphFile::pread_team(void* dst, size_t bytes, size_t at) const {
    if (bytes == 0) return EXCENT_OK;
    const size_t pieces = (bytes + kPiece - 1) / kPiece;
    const int team = (int)std::min<size_t>((size_t)team_, pieces);
    std::atomic<size_t> cursor{0};
    std::atomic<bool> failed{false};
#pragma omp parallel num_threads(team)
    {
        for (size_t p = cursor.fetch_add(1); p < pieces && !failed.load(std::memory_order_relaxed);
             p = cursor.fetch_add(1)) {
            const size_t b = p * kPiece, len = std::min(kPiece, bytes - b);
            if (pread_all(static_cast<char*>(dst) + b, len, at + b) != EXCENT_OK) failed = true;
        }
    }
    return failed ? EXCENT_ERR_IO : EXCENT_OK;
}

int GraphFile::open(const char* path, int io_threads, bool offsets_in_ram, bool check_offsets) {
    team_ = std::max(1, io_threads);
    fd_ = ::open(path, O_RDONLY);
    if (fd_ < 0) EX_FAIL(EXCENT_ERR_IO, "%s: %s", path, strerror(errno));
    struct stat st;
    if (fstat(fd_, &st) != 0) EX_FAIL(EXCENT_ERR_IO, "%s: %s", path, strerror(errno));
    const size_t file_bytes = (size_t)st.st_size;

    // header: 8 bytes, 16 for the wide form
    Header h;
    int32_t head[2] = {0, 0};
    if (file_bytes < sizeof head || pread_all(head, sizeof head, 0) != EXCENT_OK)
        EX_FAIL(EXCENT_ERR_IO, "%s: short header", path);
    h.n = head[0];
    h.wide = head[1] == -1;
    if (h.wide) {
        int64_t m64 = -1;
        if (file_bytes < 16 || pread_all(&m64, sizeof m64, sizeof head) != EXCENT_OK)
            EX_FAIL(EXCENT_ERR_IO, "%s: short header", path);
        if (m64 < 0) EX_FAIL(EXCENT_ERR_IO, "%s: bad header (negative edge count)", path);
        h.m = (ull)m64;
        h.offsets_at = 16;
    } else {
        if (head[1] < 0) EX_FAIL(EXCENT_ERR_IO, "%s: bad header (edge count %d)", path, head[1]);
        h.m = (ull)head[1];
        h.offsets_at = 8;
    }
    if (h.n < 1) EX_FAIL(EXCENT_ERR_IO, "StaticGraph: bad header in %s", path);
    const size_t offset_width = h.wide ? sizeof(ull) : sizeof(uint32_t);
    const size_t offsets_bytes = ((size_t)h.n + 1) * offset_width;
    h.entries_at = h.offsets_at + offsets_bytes;
    const size_t need = h.entries_at + h.m * sizeof(int32_t);
    if (file_bytes < need)
        EX_FAIL(EXCENT_ERR_IO, "%s: truncated (%zu bytes, header needs %llu)", path, file_bytes, (ull)need);
    n = h.n;
    m = h.m;
    wide = h.wide;
    offsets_at_ = h.offsets_at;
    entries_at_ = h.entries_at;

    // offsets into RAM: narrow ones widened, wide ones when asked
    if (!wide) {
        std::vector<uint32_t> narrow((size_t)n + 1);
        if (pread_team(narrow.data(), offsets_bytes, offsets_at_) != EXCENT_OK)
            EX_FAIL(EXCENT_ERR_IO, "%s: pread of offsets failed", path);
        ram_offsets_.assign(narrow.begin(), narrow.end());
    } else if (offsets_in_ram) {
        ram_offsets_.resize((size_t)n + 1);
        if (pread_team(ram_offsets_.data(), offsets_bytes, offsets_at_) != EXCENT_OK)
            EX_FAIL(EXCENT_ERR_IO, "%s: pread of offsets failed", path);
    }

    void* base = mmap(nullptr, file_bytes, PROT_READ, MAP_SHARED, fd_, 0);
    if (base == MAP_FAILED) EX_FAIL(EXCENT_ERR_IO, "mmap %s: %s", path, strerror(errno));
    map_.base = base;
    map_.bytes = file_bytes;
    // lists are touched in demand order: no kernel readahead on their faults
    // (the bulk preads still stream sequentially); the offsets are read front
    // to back (the check below, the upload), so they are read ahead at once
    const size_t page = (size_t)sysconf(_SC_PAGESIZE);
    const size_t lists_from = entries_at_ / page * page;
    madvise(static_cast<char*>(base) + lists_from, file_bytes - lists_from, MADV_RANDOM);
    madvise(base, lists_from, MADV_SEQUENTIAL);
    madvise(base, lists_from, MADV_WILLNEED);
    posix_fadvise(fd_, 0, 0, POSIX_FADV_SEQUENTIAL);
    const char* bytes = static_cast<const char*>(base);
    entries_ = reinterpret_cast<const int32_t*>(bytes + entries_at_);
    off_ = ram_offsets_.empty() ? reinterpret_cast<const ull*>(bytes + offsets_at_) : ram_offsets_.data();

    if (check_offsets) {
        if (off_[0] != 0 || off_[n] != m) EX_FAIL(EXCENT_ERR_IO, "%s: offsets do not span [0, m]", path);
        long long first_bad = -1;
#pragma omp parallel num_threads(team_)
        {
            long long mine = -1;
#pragma omp for schedule(static) nowait
            for (long long v = 0; v < n; v++)
                if (mine < 0 && off_[v] > off_[v + 1]) mine = v;
#pragma omp critical
            if (mine >= 0 && (first_bad < 0 || mine < first_bad)) first_bad = mine;
        }
        if (first_bad >= 0) EX_FAIL(EXCENT_ERR_IO, "%s: offsets decrease at vertex %lld", path, first_bad);
    }
    return EXCENT_OK;
}

int GraphFile::fetch_offsets(size_t v0, size_t count, ull* dst) const {
    if (v0 + count > (size_t)n + 1) EX_FAIL(EXCENT_ERR_ARG, "offsets out of range");
    if (!ram_offsets_.empty()) {
        std::copy(ram_offsets_.begin() + v0, ram_offsets_.begin() + v0 + count, dst);
        return EXCENT_OK;
    }
    if (pread_team(dst, count * sizeof(ull), offsets_at_ + v0 * sizeof(ull)) != EXCENT_OK)
        EX_FAIL(EXCENT_ERR_IO, "pread of offsets failed");
    return EXCENT_OK;
}

int GraphFile::fetch_entries(ull e0, ull e1, int32_t* dst) const {
    if (e0 > e1 || e1 > m) EX_FAIL(EXCENT_ERR_ARG, "edge range out of bounds");
    if (pread_team(dst, (e1 - e0) * sizeof(int32_t), entries_at_ + e0 * sizeof(int32_t)) != EXCENT_OK)
        EX_FAIL(EXCENT_ERR_IO, "pread of edges [%llu, %llu) failed", e0, e1);
    return EXCENT_OK;
}

void GraphFile::readahead_lists(const int32_t* vids, int k, ull* pages, ull* runs) const {
    const size_t page = page_bytes();
    const int parts = std::max(1, std::min(team_, k / 1024));
    std::vector<ull> part_pages(parts, 0), part_runs(parts, 0);
#pragma omp parallel for num_threads(parts) schedule(static, 1)
    for (int t = 0; t < parts; t++) {
        const int lo = (int)((long long)k * t / parts), hi = (int)((long long)k * (t + 1) / parts);
        // page runs of this part, in list order: [first page, end page)
        std::vector<std::pair<size_t, size_t>> run;
        for (int i = lo; i < hi; i++) {
            const int v = vids[i];
            const ull len = degree(v);
            if (len == 0) continue;
            const size_t b0 = entries_at_ + off_[v] * sizeof(int32_t);
            const size_t first = b0 / page, end = (b0 + len * sizeof(int32_t) + page - 1) / page;
            if (!run.empty() && first <= run.back().second) run.back().second = std::max(run.back().second, end);
            else run.emplace_back(first, end);
        }
        for (const auto& r : run) {
            madvise(static_cast<char*>(map_.base) + r.first * page, (r.second - r.first) * page, MADV_WILLNEED);
            part_pages[t] += r.second - r.first;
        }
        part_runs[t] = run.size();
    }
    ull np = 0, nr = 0;
    for (int t = 0; t < parts; t++) { np += part_pages[t]; nr += part_runs[t]; }
    *pages = np;
    *runs = nr;
}

// Page-aligned [b0, b1) of the file out of the mapping and the page cache.
void GraphFile::drop_bytes(size_t b0, size_t b1) const {
    const size_t page = page_bytes();
    const size_t lo = b0 - b0 % page, hi = std::min(map_.bytes, (b1 + page - 1) / page * page);
    if (hi <= lo) return;
    madvise(static_cast<char*>(map_.base) + lo, hi - lo, MADV_DONTNEED);   // or fadvise keeps our pages
    posix_fadvise(fd_, (off_t)lo, (off_t)(hi - lo), POSIX_FADV_DONTNEED);
}

void GraphFile::evict(ull e0, ull e1, size_t v0, size_t v1) const {
    drop_bytes(entries_at_ + e0 * sizeof(int32_t), entries_at_ + e1 * sizeof(int32_t));
    const size_t w = wide ? sizeof(ull) : sizeof(uint32_t);
    drop_bytes(offsets_at_ + v0 * w, offsets_at_ + (v1 + 1) * w);
}

}  // namespace excent

using namespace excent;

struct excent_egr { GraphFile f; };

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
    return g->f.fetch_offsets(v0, count, dst);
}
extern "C" int excent_egr_read_edges(excent_egr* g, unsigned long long e0, unsigned long long e1, int32_t* dst) {
    EX_CHECK_ARG(g && (dst || e0 == e1), "null argument");
    return g->f.fetch_entries(e0, e1, dst);
}
extern "C" int excent_egr_prefetch(excent_egr* g, const int32_t* vids, int k, unsigned long long* pages,
                                   unsigned long long* runs) {
    EX_CHECK_ARG(g && pages && runs && (vids || k == 0), "null argument");
    for (int i = 0; i < k; i++) EX_CHECK_ARG(vids[i] >= 0 && vids[i] < g->f.n, "vertex %d out of range", vids[i]);
    g->f.readahead_lists(vids, k, pages, runs);
    return EXCENT_OK;
}
extern "C" int excent_egr_drop_cache(excent_egr* g, unsigned long long e0, unsigned long long e1,
                                     unsigned long long v0, unsigned long long v1) {
    EX_CHECK_ARG(g && e0 <= e1 && e1 <= g->f.m && v0 <= v1 && v1 <= (ull)g->f.n, "bad range");
    g->f.evict(e0, e1, v0, v1);
    return EXCENT_OK;
}
