// egr.h -- storage-resident EGR graph file: header parse (narrow int32 or
// wide int64 offsets), mmap of the whole file, offsets in RAM or mapped,
// parallel pread of edge ranges, page-deduplicated readahead of gathered
// adjacency lists, and page-cache eviction of a chunk.
//
// Same file format and the same observable behaviour (chunk boundaries,
// page/run counts of a gather) as the reference reader
// (include/StaticGraph.h:23-171); errors are returned as status codes.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace excent {

typedef unsigned long long ull;

class EgrFile {
public:
    int n = 0;
    ull m = 0;
    bool wide = false;

    ~EgrFile();
    // Open and validate the header and file size. offsets_in_ram: copy wide
    // offsets to RAM (narrow offsets are always converted into RAM).
    int open(const char* path, int io_threads, bool offsets_in_ram, bool validate);

    ull offset(size_t v) const { return off_[v]; }
    ull degree(int v) const { return off_[v + 1] - off_[v]; }
    const int32_t* edges(int v) const { return nlist_ + off_[v]; }
    const ull* offsets() const { return off_; }
    size_t nlist_offset() const { return nlist_off_; }
    int io_threads() const { return io_threads_; }

    int read_offsets(size_t v0, size_t cnt, ull* dst) const;
    int read_edges(ull e0, ull e1, int32_t* dst) const;
    // MADV_WILLNEED over the merged page runs of the k lists (vids ascending
    // or not); parts = clamp(k / 1024, 1, io_threads) independent run merges.
    void prefetch_lists(const int32_t* vids, int k, ull* pages, ull* runs) const;
    void drop_cache(ull e0, ull e1, size_t v0, size_t v1) const;

private:
    int fd_ = -1;
    int io_threads_ = 16;
    size_t idx_off_ = 0, nlist_off_ = 0;
    std::vector<ull> ram_off_;
    const ull* off_ = nullptr;
    void* map_ = nullptr;
    size_t map_size_ = 0;
    const int32_t* nlist_ = nullptr;

    int read_exact(void* dst, size_t bytes, size_t off) const;
    int read_parallel(void* dst, size_t bytes, size_t off) const;
};

}  // namespace excent
