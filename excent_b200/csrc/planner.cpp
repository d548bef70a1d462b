// planner.cpp -- planner.h and its C entry points.
#include "planner.h"

#include <omp.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>

#include "common.h"

namespace excent {

ull chunk_cap(ull m, double chunk_medges, double target_chunks, double min_chunk_medges) {
    if (chunk_medges > 0) return (ull)(chunk_medges * 1e6);
    const ull floor_cap = (ull)(min_chunk_medges * 1e6), ceil_cap = 64000000ull;
    const ull even = (ull)std::ceil((double)m / target_chunks);
    return even < floor_cap ? floor_cap : (even > ceil_cap ? ceil_cap : even);
}

// The chunk starting at v ends at the last offset boundary b in [v, n] with
// off[b] <= limit, found by galloping from v (chunks are usually far shorter
// than the graph), but holds at least one vertex.
static int chunk_end(int n, const ull* off, int v, ull limit) {
    long long b = v, step = 1;         // off[v] <= limit always
    while (b + step <= n && off[b + step] <= limit) { b += step; step <<= 1; }
    long long hi = std::min<long long>(b + step, (long long)n + 1);   // off[hi] > limit, or hi == n + 1
    while (hi - b > 1) {
        const long long mid = b + (hi - b) / 2;
        if (off[mid] <= limit) b = mid; else hi = mid;
    }
    return (int)std::max<long long>(b, (long long)v + 1);
}

std::vector<Chunk> split_chunks(int n, const ull* off, ull cap) {
    std::vector<Chunk> out;
    for (int v = 0; v < n;) {
        const int end = chunk_end(n, off, v, off[v] + cap);
        out.push_back({v, end, off[v], off[end]});
        v = end;
    }
    return out;
}

int resident_prefix(const std::vector<Chunk>& ch, ull free_bytes, ull reserve) {
    const ull room = free_bytes > reserve ? free_bytes - reserve : 0;
    ull used = 0;
    int fit = 0;
    for (const Chunk& c : ch) {
        const ull bytes = c.edges() * sizeof(int32_t);
        if (bytes > room - used) break;
        used += bytes;
        fit++;
    }
    return fit;
}

// ------------------------------------------------------------ degree cache

static inline ull list_cost(ull d) { return 4 * d + 16; }   // entries, id, offset
static constexpr ull kWholeFrom = 1ull << 20;                // degree values admitted whole or not at all

// bit-length class of a degree (d >= 1): class k holds [2^(k-1), 2^k)
static inline int degree_class(ull d) { return 64 - __builtin_clzll(d); }

// (threshold, quota): every list of degree > threshold is admitted, and the
// first `quota` lists of degree == threshold in id order.
struct Admission { ull threshold; ull quota; };

static Admission admit_by_degree(int n, const ull* off, ull budget, int threads) {
    // pass 1: count and cost per bit-length class, lowest degree present
    ull cnt[65] = {0}, cost[65] = {0}, lowest = ULLONG_MAX;
#pragma omp parallel num_threads(threads)
    {
        ull c[65] = {0}, s[65] = {0}, lo = ULLONG_MAX;
#pragma omp for schedule(static) nowait
        for (int v = 0; v < n; v++) {
            const ull d = off[v + 1] - off[v];
            if (!d) continue;
            const int k = degree_class(d);
            c[k]++;
            s[k] += list_cost(d);
            lo = std::min(lo, d);
        }
#pragma omp critical
        {
            for (int k = 0; k < 65; k++) { cnt[k] += c[k]; cost[k] += s[k]; }
            lowest = std::min(lowest, lo);
        }
    }
    // whole classes from the top while they fit
    ull used = 0;
    int k = 64;
    for (; k >= 1; k--) {
        if (!cnt[k]) continue;
        if (cost[k] > budget - used) break;
        used += cost[k];
    }
    if (k < 1) {   // everything fits
        if (lowest == ULLONG_MAX || lowest >= kWholeFrom) return {kWholeFrom - 1, 0};
        return {lowest, ULLONG_MAX};
    }
    // pass 2: the degree values of the crossing class, highest first
    const ull lo = 1ull << (k - 1), hi = k >= 64 ? ULLONG_MAX : (1ull << k);   // [lo, hi)
    std::vector<std::pair<ull, ull>> values;   // (degree, lists)
    if (lo >= kWholeFrom) {   // few lists this long: collect and sort them
        std::vector<ull> ds;
#pragma omp parallel num_threads(threads)
        {
            std::vector<ull> mine;
#pragma omp for schedule(static) nowait
            for (int v = 0; v < n; v++) {
                const ull d = off[v + 1] - off[v];
                if (d >= lo && d < hi) mine.push_back(d);
            }
#pragma omp critical
            ds.insert(ds.end(), mine.begin(), mine.end());
        }
        std::sort(ds.begin(), ds.end(), std::greater<ull>());
        for (ull d : ds) {
            if (values.empty() || values.back().first != d) values.push_back({d, 0});
            values.back().second++;
        }
    } else {
        std::vector<ull> hist(hi - lo, 0);
#pragma omp parallel num_threads(threads)
        {
            std::vector<ull> h(hi - lo, 0);
#pragma omp for schedule(static) nowait
            for (int v = 0; v < n; v++) {
                const ull d = off[v + 1] - off[v];
                if (d >= lo && d < hi) h[d - lo]++;
            }
#pragma omp critical
            for (size_t i = 0; i < h.size(); i++) hist[i] += h[i];
        }
        for (ull i = hi - lo; i-- > 0;) if (hist[i]) values.push_back({lo + i, hist[i]});
    }
    for (const auto& [d, lists] : values) {
        const ull fit = (budget - used) / list_cost(d);
        if (fit >= lists) { used += lists * list_cost(d); continue; }
        return {d, d >= kWholeFrom ? 0 : fit};
    }
    return {values.back().first, ULLONG_MAX};   // not reached: the class did not fit whole
}

// Score levels: (S, room left for level S) -- every level above S admitted.
static std::pair<int, ull> admit_by_score(int n, const ull* off, const uint16_t* score, ull budget, int threads) {
    std::vector<ull> level(65536, 0);
#pragma omp parallel num_threads(threads)
    {
        std::vector<ull> l(65536, 0);
#pragma omp for schedule(static) nowait
        for (int v = 0; v < n; v++) {
            const ull d = off[v + 1] - off[v];
            if (d && score[v]) l[score[v]] += list_cost(d);
        }
#pragma omp critical
        for (int s = 0; s < 65536; s++) level[s] += l[s];
    }
    // at_or_above[s]: cost of every level >= s; the boundary level is the
    // highest one that takes the total past the budget
    std::vector<ull> at_or_above(65537, 0);
    for (int s = 65535; s >= 1; s--) at_or_above[s] = at_or_above[s + 1] + level[s];
    int S = 0;
    for (int lo = 1, hi = 65535; lo <= hi;) {   // largest s with at_or_above[s] > budget
        const int mid = (lo + hi) / 2;
        if (at_or_above[mid] > budget) { S = mid; lo = mid + 1; } else hi = mid - 1;
    }
    return {S, S ? budget - at_or_above[S + 1] : 0};
}

HotLists select_hot_lists(int n, const ull* off, ull budget, const uint16_t* score, int threads) {
    threads = std::max(1, threads);
    HotLists H;
    H.bits.assign(((size_t)n + 31) / 32, 0);
    std::vector<uint8_t> take(n, 0);
    if (score) {
        const std::pair<int, ull> level = admit_by_score(n, off, score, budget, threads);
        const int S = level.first;
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int v = 0; v < n; v++)
            take[v] = off[v + 1] > off[v] && score[v] && score[v] > S;
        // the boundary level, greedily in id order
        ull left = level.second;
        for (int v = 0; S && v < n; v++) {
            const ull d = off[v + 1] - off[v];
            if (d && score[v] == S && list_cost(d) <= left) { take[v] = 1; left -= list_cost(d); }
        }
        H.threshold = 0;
    } else {
        const Admission a = admit_by_degree(n, off, budget, threads);
#pragma omp parallel for num_threads(threads) schedule(static)
        for (int v = 0; v < n; v++) take[v] = off[v + 1] - off[v] > a.threshold;
        ull quota = a.quota;
        for (int v = 0; quota && v < n; v++)
            if (off[v + 1] - off[v] == a.threshold) { take[v] = 1; quota--; }
        H.threshold = a.threshold;
    }
    H.off.push_back(0);
    for (int v = 0; v < n; v++) {
        if (!take[v]) continue;
        H.ids.push_back(v);
        H.off.push_back(H.off.back() + (off[v + 1] - off[v]));
        H.bits[v >> 5] |= 1u << (v & 31);
    }
    return H;
}

// ------------------------------------------------------------ per pass

FetchMode fetch_mode(const ChunkDemand& d, ull chunk_entries, bool resident, bool loaded, double tau,
                     bool pass0_hot_fill) {
    if (d.pending == 0) return FETCH_SKIP;
    if (resident) return loaded ? FETCH_CACHED : FETCH_STREAM;   // first touch fills the cache
    if ((double)d.degree_sum >= tau * chunk_entries || pass0_hot_fill) return FETCH_STREAM;
    return FETCH_GATHER;
}

void plan_pass(const std::vector<Chunk>& ch, const ull* cnt, const std::vector<uint8_t>& resident,
               const std::vector<uint8_t>& loaded, double tau, bool hot_mode, int pass, const std::vector<int>& hlo,
               const std::vector<int>& hhi, PassPlan& out) {
    const int nc = (int)ch.size();
    out.mode.resize(nc);
    out.pending = out.demand = 0;
    out.need_bitmap = false;
    for (int c = 0; c < nc; c++) {
        const ChunkDemand d{cnt[2 * c], cnt[2 * c + 1]};
        out.pending += d.pending;
        out.demand += d.degree_sum;
        const FetchMode fm = fetch_mode(d, ch[c].edges(), resident[c] != 0, loaded[c] != 0, tau,
                                        hot_mode && pass == 0 && hhi[c] > hlo[c]);
        out.mode[c] = fm;
        out.need_bitmap |= fm == FETCH_GATHER;
    }
}

int pending_lists(int v0, int v1, const uint32_t* bitmap, const ull* idx, int32_t* vids, ull* off) {
    int k = 0;
    if (v0 < v1) {
        const int w0 = v0 >> 5, w1 = (v1 - 1) >> 5;
        for (int w = w0; w <= w1; w++) {
            uint32_t bits = bitmap[w];
            if (w == w0) bits &= ~0u << (v0 & 31);                          // below v0
            if (w == w1 && ((v1 & 31) != 0)) bits &= (1u << (v1 & 31)) - 1u; // from v1 on
            for (; bits; bits &= bits - 1) vids[k++] = (w << 5) + __builtin_ctz(bits);
        }
    }
    off[0] = 0;
    for (int i = 0; i < k; i++) off[i + 1] = off[i] + (idx[vids[i] + 1] - idx[vids[i]]);
    return k;
}

double crossover_tau(double t_stream, const double* t_gather, const double* f) {
    double tau;
    if (t_gather[0] >= t_stream) {            // even the smallest gather is slower: scale down
        tau = f[0] * t_stream / t_gather[0];
    } else if (t_gather[2] < t_stream) {      // even the largest gather is faster: scale up
        tau = f[2] * t_stream / t_gather[2];
    } else {                                  // the segment whose right end reaches t_stream
        const int j = t_gather[1] >= t_stream ? 1 : 2;
        const double slope = (f[j] - f[j - 1]) * (t_stream - t_gather[j - 1]);
        tau = f[j - 1] + slope / (t_gather[j] - t_gather[j - 1]);
    }
    return std::min(1.0, std::max(0.005, tau));
}

}  // namespace excent

using namespace excent;

extern "C" unsigned long long excent_chunk_cap(unsigned long long m, double chunk_medges, double target_chunks,
                                               double min_chunk_medges) {
    return chunk_cap(m, chunk_medges, target_chunks, min_chunk_medges);
}

extern "C" int excent_plan_chunks(int n, const unsigned long long* off, unsigned long long cap, int* nc,
                                  unsigned long long* out, int out_cap) {
    EX_CHECK_ARG(n >= 1 && off && nc && cap >= 1, "bad argument");
    const std::vector<Chunk> ch = split_chunks(n, off, cap);
    *nc = (int)ch.size();
    if (out) {
        EX_CHECK_ARG(out_cap >= (int)ch.size(), "output holds %d chunks, need %zu", out_cap, ch.size());
        for (size_t c = 0; c < ch.size(); c++) {
            out[4 * c] = (ull)ch[c].v0; out[4 * c + 1] = (ull)ch[c].v1;
            out[4 * c + 2] = ch[c].e0; out[4 * c + 3] = ch[c].e1;
        }
    }
    return EXCENT_OK;
}

extern "C" int excent_cache_chunks(int nc, const unsigned long long* chunk_edges, unsigned long long free_bytes,
                                   unsigned long long reserve, int* resident) {
    EX_CHECK_ARG(nc >= 0 && (chunk_edges || nc == 0) && resident, "bad argument");
    std::vector<Chunk> ch(nc);
    for (int c = 0; c < nc; c++) ch[c] = {c, c + 1, 0, chunk_edges[c]};
    *resident = resident_prefix(ch, free_bytes, reserve);
    return EXCENT_OK;
}

extern "C" int excent_hot_select(int n, const unsigned long long* off, unsigned long long budget, const uint16_t* score,
                                 int* nh, int32_t* ids, unsigned long long* hoff, uint32_t* bits,
                                 unsigned long long* threshold) {
    EX_CHECK_ARG(n >= 1 && off && nh, "bad argument");
    const HotLists H = select_hot_lists(n, off, budget, score, omp_get_max_threads());
    *nh = (int)H.ids.size();
    if (ids) std::copy(H.ids.begin(), H.ids.end(), ids);
    if (hoff) std::copy(H.off.begin(), H.off.end(), hoff);
    if (bits) std::copy(H.bits.begin(), H.bits.end(), bits);
    if (threshold) *threshold = H.threshold;
    return EXCENT_OK;
}

extern "C" int excent_fetch_plan(int nc, const unsigned long long* chunk_edges, const unsigned long long* cnt,
                                 const uint8_t* resident, const uint8_t* loaded, double stream_ratio, int hot_mode,
                                 int pass, const int* hlo, const int* hhi, uint8_t* mode,
                                 unsigned long long* pend_v, unsigned long long* demand, int* need_bitmap) {
    EX_CHECK_ARG(nc >= 1 && chunk_edges && cnt && resident && loaded && hlo && hhi && mode, "bad argument");
    std::vector<Chunk> ch(nc);
    for (int c = 0; c < nc; c++) ch[c] = {c, c + 1, 0, chunk_edges[c]};
    PassPlan P;
    plan_pass(ch, cnt, std::vector<uint8_t>(resident, resident + nc), std::vector<uint8_t>(loaded, loaded + nc),
              stream_ratio, hot_mode != 0, pass, std::vector<int>(hlo, hlo + nc), std::vector<int>(hhi, hhi + nc), P);
    std::copy(P.mode.begin(), P.mode.end(), mode);
    if (pend_v) *pend_v = P.pending;
    if (demand) *demand = P.demand;
    if (need_bitmap) *need_bitmap = P.need_bitmap;
    return EXCENT_OK;
}

extern "C" int excent_gather_list(int v0, int v1, const uint32_t* bitmap, const unsigned long long* idx, int32_t* vids,
                                  unsigned long long* off, int* k) {
    EX_CHECK_ARG(v0 >= 0 && v0 <= v1 && bitmap && idx && vids && off && k, "bad argument");
    *k = pending_lists(v0, v1, bitmap, idx, vids, off);
    return EXCENT_OK;
}

extern "C" double excent_tau(double t_stream, const double* t_g, const double* f) {
    return crossover_tau(t_stream, t_g, f);
}
