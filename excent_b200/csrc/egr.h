// egr.h -- the EGR graph file as the host runtime sees it.
//
// An EGR file (README.md:136-146 of SPADE-IITJ/ExCent) is a CSR graph:
//   int32 n, then either int32 m with uint32 offsets[n+1] ("narrow"), or
//   int32 -1, int64 m with uint64 offsets[n+1] ("wide"), then int32
//   adjacency entries[m].
// GraphFile maps the whole file read-only and serves three kinds of access:
//   * offsets: converted into RAM (narrow files always, wide ones on request)
//     or read in place from the mapping;
//   * bulk entry ranges (streamed chunks): positional reads split into fixed
//     8 MiB pieces that a team of threads claims from a shared cursor;
//   * single lists (gathered vertices): pointers into the mapping, with a
//     readahead step that requests each run of touched pages once.
// Chunk boundaries and the page/run counts of a readahead equal those of the
// reference reader (include/StaticGraph.h); errors are status codes.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace excent {

typedef unsigned long long ull;

class GraphFile {
public:
    int n = 0;
    ull m = 0;
    bool wide = false;

    GraphFile() = default;
    GraphFile(const GraphFile&) = delete;
    GraphFile& operator=(const GraphFile&) = delete;
    ~GraphFile();

    // Open, check the header against the file size, map it. offsets_in_ram:
    // keep a RAM copy of wide offsets (narrow offsets are always widened into
    // RAM). check_offsets: verify offsets[0] == 0, offsets[n] == m and that
    // they never decrease.
    int open(const char* path, int io_threads, bool offsets_in_ram, bool check_offsets);

    const ull* offsets() const { return off_; }
    ull degree(int v) const { return off_[v + 1] - off_[v]; }
    const int32_t* list(int v) const { return entries_ + off_[v]; }
    int io_threads() const { return team_; }

    int fetch_offsets(size_t v0, size_t count, ull* dst) const;
    int fetch_entries(ull e0, ull e1, int32_t* dst) const;
    // Ask the kernel to read ahead the pages of the k lists of vids (in the
    // order given). The ids are cut into parts = clamp(k / 1024, 1,
    // io_threads) contiguous parts; inside a part, the page spans of
    // consecutive lists merge into one run while each starts no later than
    // the run's end. Returns the pages and runs requested.
    void readahead_lists(const int32_t* vids, int k, ull* pages, ull* runs) const;
    // Drop the entries [e0, e1) and the offsets of vertices [v0, v1] from this
    // process's mapping and from the page cache (cold-cache measurements).
    void evict(ull e0, ull e1, size_t v0, size_t v1) const;

private:
    struct Mapping {
        void* base = nullptr;
        size_t bytes = 0;
    };
    int fd_ = -1;
    int team_ = 16;            // reader threads
    size_t offsets_at_ = 0;    // byte position of offsets[0]
    size_t entries_at_ = 0;    // byte position of entries[0]
    Mapping map_;
    std::vector<ull> ram_offsets_;
    const ull* off_ = nullptr;
    const int32_t* entries_ = nullptr;

    int pread_all(void* dst, size_t bytes, size_t at) const;
    int pread_team(void* dst, size_t bytes, size_t at) const;
    void drop_bytes(size_t b0, size_t b1) const;
};

}  // namespace excent
