// planner.h -- host-side planning of a run: the chunk cap and chunk table,
// the GPU cache sizing (a resident prefix of whole chunks, or a set of
// high-degree lists), the per-pass fetch decision of each chunk, the gathered
// list of a chunk's pending vertices, and the stream/gather crossover tau.
//
// Every decision is integer (or one FP64 comparison) and gives the same
// result as the reference's host code on the same inputs; each function
// names the reference lines whose behaviour it reproduces (src/excent.cu,
// include/StaticGraph.h of SPADE-IITJ/ExCent).
#pragma once
#include <cstdint>
#include <vector>

namespace excent {

typedef unsigned long long ull;

// A contiguous vertex range [v0, v1) and its entries [e0, e1).
struct Chunk {
    int v0, v1;
    ull e0, e1;
    ull edges() const { return e1 - e0; }
};

// Entries per chunk: --chunk-medges when given, else ceil(m / target_chunks)
// held to [min_chunk_medges * 1e6, 64e6] (src/excent.cu:321-326).
ull chunk_cap(ull m, double chunk_medges, double target_chunks, double min_chunk_medges);

// Cut the vertex range into chunks: each chunk runs from its first vertex to
// the last offset boundary within cap entries of its start, and holds at
// least one vertex (include/StaticGraph.h:128-139).
std::vector<Chunk> split_chunks(int n, const ull* off, ull cap);

// How many leading chunks fit, whole, in free - reserve bytes of device
// memory (src/excent.cu:410-421).
int resident_prefix(const std::vector<Chunk>& ch, ull free_bytes, ull reserve);

// The degree cache: which lists to hold on the device within `budget` bytes,
// a list of degree d costing 4 d + 16 bytes (src/excent.cu:428-491).
//  * By degree: lists are admitted from the highest degree down. Every
//    degree value of 2^20 or more is admitted whole or not at all; below
//    that, a degree value that does not fit whole is admitted partly, the
//    first vertices in id order. Admission stops at the first value that
//    does not fit whole; threshold reports that value (or the lowest degree
//    present when everything fits, 2^20 - 1 when none is below 2^20).
//  * By score (--hot-rank, uint16 per vertex, 0 = never): whole score levels
//    from the highest down while they fit; of the first level that does not,
//    the vertices in id order that still fit in what is left.
struct HotLists {
    std::vector<int32_t> ids;    // ascending
    std::vector<ull> off;        // ids.size() + 1
    std::vector<uint32_t> bits;  // ceil(n / 32) words
    ull threshold = 0;           // 0 with a score ranking
    ull edges() const { return off.empty() ? 0 : off.back(); }
};
HotLists select_hot_lists(int n, const ull* off, ull budget, const uint16_t* score, int threads);

// Fetch decision of one chunk for one pass (src/excent.cu:666-677):
// nothing pending -> SKIP; resident and already loaded -> CACHED; resident
// but not loaded yet, or pending degree sum >= tau * chunk entries -> STREAM;
// the pass-0 fill of a chunk holding degree-cache lists -> STREAM; otherwise
// GATHER the pending lists.
enum FetchMode : uint8_t { FETCH_SKIP = 0, FETCH_CACHED = 1, FETCH_STREAM = 2, FETCH_GATHER = 3 };
struct ChunkDemand {
    ull pending;     // vertices
    ull degree_sum;  // entries of the pending vertices
};
FetchMode fetch_mode(const ChunkDemand& d, ull chunk_entries, bool resident, bool loaded, double tau,
                     bool pass0_hot_fill);

// The pass's plan over every chunk: modes, totals and whether any chunk
// gathers (so the bitmap must come back to the host).
struct PassPlan {
    std::vector<uint8_t> mode;
    ull pending = 0, demand = 0;
    bool need_bitmap = false;
};
void plan_pass(const std::vector<Chunk>& ch, const ull* cnt, const std::vector<uint8_t>& resident,
               const std::vector<uint8_t>& loaded, double tau, bool hot_mode, int pass, const std::vector<int>& hlo,
               const std::vector<int>& hhi, PassPlan& out);

// Pending vertices of [v0, v1) from the bitmap, ascending, and the prefix
// sums of their degrees (src/excent.cu:711-723). Returns k; off holds k + 1.
int pending_lists(int v0, int v1, const uint32_t* bitmap, const ull* idx, int32_t* vids, ull* off);

// The crossover tau from one streamed read and three gathers at demand
// fractions f[0..2] (src/excent.cu:566-572): the fraction at which a gather
// takes as long as the stream, on the piecewise-linear curve through the
// three gathers (proportional through the origin outside them), held to
// [0.005, 1].
double crossover_tau(double t_stream, const double* t_gather, const double* f);

}  // namespace excent
