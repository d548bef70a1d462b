// planner.h -- host-side planning of a run: chunk cap and chunk table, GPU
// cache sizing (whole chunks, or high-degree lists), the per-pass fetch plan
// and the gathered-list build, and the stream/gather crossover tau.
//
// Every decision here is integer (or an FP64 comparison) and reproduces the
// reference's host code bit for bit on the same inputs; each function names
// the reference lines it follows (src/excent.cu, include/StaticGraph.h).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace excent {

typedef unsigned long long ull;

struct Chunk {
    int v0, v1;
    ull e0, e1;
    ull edges() const { return e1 - e0; }
};

// --chunk-medges / --target-chunks / --min-chunk-medges (src/excent.cu:321-326)
ull chunk_cap(ull m, double chunk_medges, double target_chunks, double min_chunk_medges);
// greedy contiguous chunks of <= cap edges, >= 1 vertex (include/StaticGraph.h:128-139)
std::vector<Chunk> plan_chunks(int n, const ull* off, ull cap);

// Number of leading chunks that fit in free - reserve bytes (src/excent.cu:410-421).
int cache_chunks(const std::vector<Chunk>& ch, ull free_bytes, ull reserve);

// Degree cache selection (src/excent.cu:428-491). score: optional uint16[n]
// ranking (--hot-rank); otherwise by degree threshold T with a quota.
struct HotSet {
    std::vector<int32_t> ids;   // ascending
    std::vector<ull> off;       // nh + 1
    std::vector<uint32_t> bits; // ceil(n/32) words
    ull T = 0;                  // degree threshold (0 with a score ranking)
    ull edges() const { return off.empty() ? 0 : off.back(); }
};
HotSet hot_select(int n, const ull* off, ull budget, const uint16_t* score, int threads);

// Per-chunk mode 0 skip, 1 resident, 2 stream, 3 gather (src/excent.cu:666-678).
struct FetchPlan {
    std::vector<uint8_t> mode;
    ull pend_v = 0, demand = 0;
    bool need_bitmap = false;
};
void fetch_plan(const std::vector<Chunk>& ch, const ull* cnt, const std::vector<uint8_t>& resident,
                const std::vector<uint8_t>& loaded, double stream_ratio, bool hot_mode, int pass,
                const std::vector<int>& hlo, const std::vector<int>& hhi, FetchPlan& out);

// Ascending pending ids of [v0, v1) from the bitmap and the prefix sums of
// their degrees (src/excent.cu:711-723). Returns k; off holds k + 1 entries.
int gather_list(int v0, int v1, const uint32_t* bitmap, const ull* idx, int32_t* vids, ull* off);

// Crossover from one stream and three gather timings (src/excent.cu:566-572).
double tau_from_timings(double t_stream, const double* t_g, const double* f);

}  // namespace excent
