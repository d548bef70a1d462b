// graph_tools.cpp -- the EGR file tools around the engine:
//   excent_convert in.mtx out.egr [--sort] [--dedup] [--no-self-loops] [--symmetric]
//       MatrixMarket coordinate file -> wide EGR (tools/efficient_converter.py:5-113)
//   excent_info g.egr
//       header, max degree, sampled reverse-edge and self-loop check (tools/egr_info.cpp:10-30)
//   excent_evict [--report] file...
//       drop files from the page cache for cold-cache runs (tools/evict_file.c:18-65)
//
// The converter reads the text through a read-only mapping in two passes:
// degrees first (a team of threads over newline-aligned slices, counting with
// atomic adds), then the entries into a pre-sized output file mapped for
// writing, each list at its own cursor. Without --sort the entries of a list
// keep the file's order, as the reference converter writes them; --sort
// orders every list, --dedup also drops repeated entries (and compacts the
// file), --no-self-loops drops u == v, --symmetric adds v -> u for every
// u -> v entry (MatrixMarket "symmetric" files list one triangle).
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "common.h"
#include "egr.h"

namespace excent {

namespace {

// A read-only view of a whole file.
struct TextMap {
    int fd = -1;
    const char* p = nullptr;
    size_t n = 0;
    ~TextMap() {
        if (p && n) munmap((void*)p, n);
        if (fd >= 0) ::close(fd);
    }
    int open(const char* path) {
        fd = ::open(path, O_RDONLY);
        if (fd < 0) EX_FAIL(EXCENT_ERR_IO, "%s: %s", path, strerror(errno));
        struct stat st;
        if (fstat(fd, &st) != 0) EX_FAIL(EXCENT_ERR_IO, "%s: %s", path, strerror(errno));
        n = (size_t)st.st_size;
        if (n) {
            void* m = mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m == MAP_FAILED) { p = nullptr; EX_FAIL(EXCENT_ERR_IO, "mmap %s: %s", path, strerror(errno)); }
            p = static_cast<const char*>(m);
            madvise(m, n, MADV_SEQUENTIAL);
        }
        return EXCENT_OK;
    }
};

// Up to three leading unsigned integers of the line starting at *pos; moves
// *pos past the line. Returns the number of integers read (a token that is
// not an unsigned integer ends the scan; -1 for a comment line).
int scan_line(const char* s, size_t end, size_t* pos, long long out[3]) {
    size_t i = *pos;
    size_t eol = i;
    while (eol < end && s[eol] != '\n') eol++;
    *pos = eol < end ? eol + 1 : end;
    while (i < eol && (s[i] == ' ' || s[i] == '\t' || s[i] == '\r')) i++;
    if (i < eol && s[i] == '%') return -1;
    int got = 0;
    while (got < 3 && i < eol) {
        if (s[i] < '0' || s[i] > '9') break;
        long long v = 0;
        while (i < eol && s[i] >= '0' && s[i] <= '9') v = v * 10 + (s[i++] - '0');
        if (i < eol && !(s[i] == ' ' || s[i] == '\t' || s[i] == '\r')) break;   // e.g. "1.5": not an id
        out[got++] = v;
        while (i < eol && (s[i] == ' ' || s[i] == '\t' || s[i] == '\r')) i++;
    }
    return got;
}

// Newline-aligned slice boundaries of [b, e) for t threads.
std::vector<size_t> slices(const char* s, size_t b, size_t e, int t) {
    std::vector<size_t> cut(t + 1, e);
    cut[0] = b;
    for (int i = 1; i < t; i++) {
        size_t c = std::max(cut[i - 1], b + (e - b) * i / t);
        while (c < e && c > b && s[c - 1] != '\n') c++;
        cut[i] = c;
    }
    return cut;
}

struct ConvertStats {
    ull n = 0, entries_read = 0, skipped = 0, self_loops = 0, m = 0;
};

}  // namespace

enum { CONV_SORT = 1, CONV_DEDUP = 2, CONV_NO_SELF = 4, CONV_SYMMETRIC = 8 };

static int convert_mtx(const char* in, const char* out, int flags, ConvertStats& cs) {
    TextMap t;
    EX_TRY(t.open(in));
    const char* s = t.p;
    // size line: the first line that is not a comment
    size_t pos = 0;
    long long hdr[3] = {0, 0, 0};
    int got = 0;
    while (pos < t.n && (got = scan_line(s, t.n, &pos, hdr)) == -1) {}
    if (got < 2) EX_FAIL(EXCENT_ERR_IO, "%s: no MatrixMarket size line", in);
    const long long nn = std::max(hdr[0], hdr[1]);
    if (nn < 1 || nn > 0x7fffffffLL) EX_FAIL(EXCENT_ERR_IO, "%s: bad size line (%lld x %lld)", in, hdr[0], hdr[1]);
    const int n = (int)nn;
    cs.n = (ull)n;
    const bool sym = flags & CONV_SYMMETRIC, no_self = flags & CONV_NO_SELF;
    const int team = std::max(1, std::min(omp_get_max_threads(), (int)(t.n / (1 << 20)) + 1));
    const std::vector<size_t> cut = slices(s, pos, t.n, team);

    // pass 1: degrees (entries of sources past n are skipped, as the reference converter does)
    std::vector<ull> deg((size_t)n + 1, 0);
    std::atomic<long long> bad_line{-1};
    std::atomic<ull> read{0}, skipped{0}, selfs{0};
#pragma omp parallel num_threads(team)
    {
        const int me = omp_get_thread_num();
        ull r = 0, sk = 0, sl = 0;
        long long v3[3];
        for (size_t p = cut[me]; p < cut[me + 1];) {
            const size_t at = p;
            const int k = scan_line(s, cut[me + 1], &p, v3);
            if (k < 2) continue;
            r++;
            if (v3[0] < 1) { bad_line = (long long)at; continue; }
            if (v3[0] > n) { sk++; continue; }
            if (v3[1] < 1 || v3[1] > n) { bad_line = (long long)at; continue; }
            if (v3[0] == v3[1]) { sl++; if (no_self) continue; }
            __atomic_fetch_add(&deg[v3[0] - 1], 1ull, __ATOMIC_RELAXED);
            if (sym && v3[0] != v3[1]) __atomic_fetch_add(&deg[v3[1] - 1], 1ull, __ATOMIC_RELAXED);
        }
        read += r; skipped += sk; selfs += sl;
    }
    if (bad_line >= 0) {
        const long long at = bad_line;
        const char* l = s + at;
        const char* e = (const char*)memchr(l, '\n', t.n - at);
        EX_FAIL(EXCENT_ERR_IO, "%s: entry \"%.*s\" is not a pair of 1-based vertex ids within n = %d", in,
                (int)std::min<long>(60, (e ? e : s + t.n) - l), l, n);
    }
    cs.entries_read = read;
    cs.skipped = skipped;
    cs.self_loops = selfs;
    std::vector<ull> off((size_t)n + 1, 0);
    for (int v = 0; v < n; v++) off[v + 1] = off[v] + deg[v];
    const ull m = off[n];

    // the output, pre-sized and mapped for writing
    const size_t head = 16, offsets_bytes = ((size_t)n + 1) * sizeof(ull);
    const size_t bytes = head + offsets_bytes + m * sizeof(int32_t);
    const int fd = ::open(out, O_RDWR | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) EX_FAIL(EXCENT_ERR_IO, "%s: %s", out, strerror(errno));
    if (ftruncate(fd, (off_t)bytes) != 0) { ::close(fd); EX_FAIL(EXCENT_ERR_IO, "%s: %s", out, strerror(errno)); }
    void* map = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
    if (map == MAP_FAILED) { ::close(fd); EX_FAIL(EXCENT_ERR_IO, "mmap %s: %s", out, strerror(errno)); }
    int32_t* lists = reinterpret_cast<int32_t*>(static_cast<char*>(map) + head + offsets_bytes);

    // pass 2: entries to their lists; file order per list unless the lists get sorted anyway
    std::vector<ull> cursor(off.begin(), off.end() - 1);
    const bool ordered = !(flags & (CONV_SORT | CONV_DEDUP));
    auto place = [&](int u, int v) {
        const ull at = ordered ? cursor[u]++ : __atomic_fetch_add(&cursor[u], 1ull, __ATOMIC_RELAXED);
        lists[at] = v;
    };
    auto scan_slice = [&](size_t b, size_t e) {
        long long v3[3];
        for (size_t p = b; p < e;) {
            if (scan_line(s, e, &p, v3) < 2 || v3[0] > n) continue;
            const int u = (int)v3[0] - 1, v = (int)v3[1] - 1;
            if (u == v && no_self) continue;
            place(u, v);
            if (sym && u != v) place(v, u);
        }
    };
    if (ordered) {
        scan_slice(cut[0], cut[team]);
    } else {
#pragma omp parallel num_threads(team)
        scan_slice(cut[omp_get_thread_num()], cut[omp_get_thread_num() + 1]);
    }

    // sort / dedup per list, then pack the lists forward over the dropped entries
    ull kept = m;
    if (!ordered) {
        std::vector<ull> len(n);
#pragma omp parallel for schedule(dynamic, 1024)
        for (int v = 0; v < n; v++) {
            int32_t* b = lists + off[v];
            int32_t* e = lists + off[v + 1];
            std::sort(b, e);
            len[v] = (flags & CONV_DEDUP) ? (ull)(std::unique(b, e) - b) : (ull)(e - b);
        }
        ull w = 0;
        for (int v = 0; v < n; v++) {
            if (w != off[v]) memmove(lists + w, lists + off[v], len[v] * sizeof(int32_t));
            off[v] = w;
            w += len[v];
        }
        off[n] = w;
        kept = w;
    }
    int32_t hdr32[2] = {n, -1};
    const int64_t m64 = (int64_t)kept;
    memcpy(map, hdr32, sizeof hdr32);
    memcpy(static_cast<char*>(map) + 8, &m64, sizeof m64);
    memcpy(static_cast<char*>(map) + head, off.data(), offsets_bytes);
    // the packed lists sit right after the offsets, so only the tail goes
    const size_t final_bytes = head + offsets_bytes + kept * sizeof(int32_t);
    const bool synced = msync(map, bytes, MS_SYNC) == 0;
    munmap(map, bytes);
    const bool cut_ok = ftruncate(fd, (off_t)final_bytes) == 0;
    ::close(fd);
    if (!synced || !cut_ok) EX_FAIL(EXCENT_ERR_IO, "%s: write failed", out);
    cs.m = kept;
    return EXCENT_OK;
}

// ---------------------------------------------------------------- info

static int egr_report(const char* path, std::string& line) {
    GraphFile g;
    EX_TRY(g.open(path, 16, true, true));
    const ull* off = g.offsets();
    const int n = g.n;
    const ull m = g.m;
    ull maxd = 0;
    for (int v = 0; v < n; v++) maxd = std::max(maxd, off[v + 1] - off[v]);
    // 20000 entries drawn with mt19937_64 seeded 7: is the reverse entry there, is it a self-loop
    const int samples = m ? 20000 : 0;
    int missing = 0, loops = 0;
    std::mt19937_64 rng(7);
    const int32_t* all = g.list(0);
    for (int i = 0; i < samples; i++) {
        const ull e = rng() % m;
        const int src = (int)(std::upper_bound(off, off + n, e) - off) - 1;   // the list holding entry e
        const int dst = all[e];
        if (src == dst) loops++;
        if (dst < 0 || dst >= n) { missing++; continue; }
        const int32_t* b = g.list(dst);
        const int32_t* en = b + g.degree(dst);
        const bool found = std::is_sorted(b, en) ? std::binary_search(b, en, src) : std::find(b, en, src) != en;
        if (!found) missing++;
    }
    char buf[512];
    snprintf(buf, sizeof buf,
             "n=%d m=%llu (%.2f GB edges) maxdeg=%llu  reverse-edge missing %d/%d (%.1f%%) self-loops %d  m>2^32-1: %s\n",
             n, m, m * 4.0 / 1e9, maxd, missing, samples, samples ? 100.0 * missing / samples : 0.0, loops,
             m > 4294967295ull ? "YES" : "no");
    line = buf;
    return EXCENT_OK;
}

// ---------------------------------------------------------------- evict

// Share of the file's pages resident in the page cache (mincore), -1 on error.
static double resident_share(int fd, size_t bytes) {
    if (bytes == 0) return 0.0;
    void* p = mmap(nullptr, bytes, PROT_READ, MAP_SHARED, fd, 0);
    if (p == MAP_FAILED) return -1.0;
    const size_t page = (size_t)sysconf(_SC_PAGESIZE), pages = (bytes + page - 1) / page;
    std::vector<unsigned char> in(pages);
    double share = -1.0;
    if (mincore(p, bytes, in.data()) == 0) {
        size_t r = 0;
        for (unsigned char c : in) r += c & 1;
        share = (double)r / (double)pages;
    }
    munmap(p, bytes);
    return share;
}

}  // namespace excent

using namespace excent;

extern "C" int excent_mtx_to_egr(const char* in, const char* out, int flags, unsigned long long* stats) {
    EX_CHECK_ARG(in && out, "null argument");
    EX_CHECK_ARG((flags & ~15) == 0, "unknown flags 0x%x", flags);
    ConvertStats cs;
    EX_TRY(convert_mtx(in, out, flags, cs));
    if (stats) {
        stats[0] = cs.n; stats[1] = cs.entries_read; stats[2] = cs.skipped; stats[3] = cs.self_loops; stats[4] = cs.m;
    }
    return EXCENT_OK;
}

extern "C" int excent_egr_report(const char* path, char* out, int cap) {
    EX_CHECK_ARG(path && out && cap > 0, "null argument");
    std::string line;
    EX_TRY(egr_report(path, line));
    EX_CHECK_ARG((int)line.size() < cap, "report needs %zu bytes", line.size() + 1);
    memcpy(out, line.c_str(), line.size() + 1);
    return EXCENT_OK;
}

extern "C" int excent_convert_main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <input.mtx> <output.egr> [--sort] [--dedup] [--no-self-loops] [--symmetric]\n",
                argv[0]);
        return 1;
    }
    int flags = 0;
    for (int i = 3; i < argc; i++) {
        const std::string a = argv[i];
        if (a == "--sort") flags |= CONV_SORT;
        else if (a == "--dedup") flags |= CONV_DEDUP | CONV_SORT;
        else if (a == "--no-self-loops") flags |= CONV_NO_SELF;
        else if (a == "--symmetric") flags |= CONV_SYMMETRIC;
        else { fprintf(stderr, "unknown option %s\n", a.c_str()); return 1; }
    }
    ull st[5];
    if (excent_mtx_to_egr(argv[1], argv[2], flags, st) != EXCENT_OK) {
        fprintf(stderr, "%s\n", excent_last_error());
        return 1;
    }
    printf("%s: n=%llu, %llu entries read (%llu past n skipped, %llu self-loops), %llu written to %s\n", argv[1], st[0],
           st[1], st[2], st[3], st[4], argv[2]);
    return 0;
}

extern "C" int excent_info_main(int argc, char** argv) {
    if (argc != 2) { fprintf(stderr, "usage: %s <graph.egr>\n", argv[0]); return 1; }
    char line[512];
    if (excent_egr_report(argv[1], line, sizeof line) != EXCENT_OK) {
        fprintf(stderr, "%s\n", excent_last_error());
        return 1;
    }
    fputs(line, stdout);
    return 0;
}

extern "C" int excent_evict_main(int argc, char** argv) {
    if (argc < 2) { fprintf(stderr, "usage: %s [--report] <file> [...]\n", argv[0]); return 1; }
    const bool report = !strcmp(argv[1], "--report");
    int rc = 0;
    for (int i = report ? 2 : 1; i < argc; i++) {
        const int fd = ::open(argv[i], O_RDONLY);
        if (fd < 0) { perror(argv[i]); rc = 1; continue; }
        struct stat st;
        fstat(fd, &st);
        const size_t bytes = (size_t)st.st_size;
        if (report) {   // resident share only, nothing evicted
            printf("%.1f\n", 100 * resident_share(fd, bytes));
        } else {
            const double before = resident_share(fd, bytes);
            fdatasync(fd);
            const int e = posix_fadvise(fd, 0, 0, POSIX_FADV_DONTNEED);
            const double after = resident_share(fd, bytes);
            printf("%s: %.1f%% -> %.1f%% resident%s\n", argv[i], 100 * before, 100 * after,
                   e ? " (fadvise failed)" : "");
            if (e || after > 0.01) rc = 1;
        }
        ::close(fd);
    }
    return rc;
}
