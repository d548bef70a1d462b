// planner.cpp -- planner.h and its C entry points.
#include "planner.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.h"

namespace excent {

ull chunk_cap(ull m, double chunk_medges, double target_chunks, double min_chunk_medges) {
    if (chunk_medges > 0) return (ull)(chunk_medges * 1e6);
    const ull lo = (ull)(min_chunk_medges * 1e6), hi = 64000000ull;
    return std::min(hi, std::max(lo, (ull)std::ceil((double)m / target_chunks)));
}

std::vector<Chunk> plan_chunks(int n, const ull* off, ull cap) {
    std::vector<Chunk> out;
    int v = 0;
    while (v < n) {
        const ull limit = off[v] + cap;
        int v1 = (int)(std::upper_bound(off + v + 1, off + n + 1, limit) - off) - 1;
        if (v1 <= v) v1 = v + 1;
        out.push_back({v, v1, off[v], off[v1]});
        v = v1;
    }
    return out;
}

int cache_chunks(const std::vector<Chunk>& ch, ull free_bytes, ull reserve) {
    ull avail = free_bytes > reserve ? free_bytes - reserve : 0;
    int c = 0;
    for (; c < (int)ch.size(); c++) {
        const ull need = ch[c].edges() * sizeof(int32_t);
        if (need > avail) break;
        avail -= need;
    }
    return c;
}

static inline ull hot_cost(ull d) { return d * sizeof(int32_t) + 2 * sizeof(int32_t) + sizeof(ull); }

HotSet hot_select(int n, const ull* off, ull budget, const uint16_t* score, int threads) {
    const ull CAP = 1ull << 20;
    std::vector<ull> hist(CAP, 0), big;
    // degree histogram (< 2^20) and the list of larger degrees
#pragma omp parallel num_threads(std::max(1, threads))
    {
        std::vector<ull> lh(CAP, 0), lb;
#pragma omp for schedule(static) nowait
        for (int v = 0; v < n; v++) {
            const ull d = off[v + 1] - off[v];
            if (d >= CAP) lb.push_back(d); else lh[d]++;
        }
#pragma omp critical
        {
            for (ull d = 0; d < CAP; d++) hist[d] += lh[d];
            big.insert(big.end(), lb.begin(), lb.end());
        }
    }
    std::sort(big.rbegin(), big.rend());
    ull used = 0, T = 0, quota = 0;
    bool done = false;
    for (ull d : big) {
        if (used + hot_cost(d) > budget) { T = d; quota = 0; done = true; break; }
        used += hot_cost(d);
        T = d;
        quota++;
    }
    if (!done) { quota = 0; T = CAP - 1; }
    for (ull d = CAP - 1; !done && d >= 1; d--) {
        if (!hist[d]) continue;
        const ull take = std::min<ull>(hist[d], (budget - used) / hot_cost(d));
        used += take * hot_cost(d);
        T = d;
        quota = take;
        if (take < hist[d]) done = true;
    }
    // --hot-rank: highest scores first, the boundary score partly (src/excent.cu:459-473)
    int S = 0;
    ull s_left = 0;
    if (score) {
        std::vector<double> cs(65536, 0.0);
        for (int v = 0; v < n; v++) {
            const ull d = off[v + 1] - off[v];
            if (d && score[v]) cs[score[v]] += (double)hot_cost(d);
        }
        double u = 0;
        for (int s = 65535; s >= 1; s--) {
            if (u + cs[s] <= (double)budget) { u += cs[s]; continue; }
            S = s;
            s_left = budget - (ull)u;
            break;
        }
    }
    HotSet H;
    H.off.push_back(0);
    H.bits.assign(((size_t)n + 31) / 32, 0);
    for (int v = 0; v < n; v++) {
        const ull d = off[v + 1] - off[v];
        if (d == 0) continue;
        if (score) {
            if (score[v] == 0 || score[v] < S) continue;
            if (score[v] == S) {
                if (hot_cost(d) > s_left) continue;
                s_left -= hot_cost(d);
            }
        } else {
            const bool take = d > T || (d == T && quota > 0);
            if (!take) continue;
            if (d == T) quota--;
        }
        H.ids.push_back(v);
        H.off.push_back(H.off.back() + d);
        H.bits[v >> 5] |= 1u << (v & 31);
    }
    H.T = score ? 0 : T;
    return H;
}

void fetch_plan(const std::vector<Chunk>& ch, const ull* cnt, const std::vector<uint8_t>& resident,
                const std::vector<uint8_t>& loaded, double stream_ratio, bool hot_mode, int pass,
                const std::vector<int>& hlo, const std::vector<int>& hhi, FetchPlan& out) {
    const int nc = (int)ch.size();
    out.mode.assign(nc, 0);
    out.pend_v = out.demand = 0;
    out.need_bitmap = false;
    for (int c = 0; c < nc; c++) {
        const ull cv = cnt[2 * c], ce = cnt[2 * c + 1];
        out.pend_v += cv;
        out.demand += ce;
        if (cv == 0) continue;
        if (resident[c] && loaded[c]) out.mode[c] = 1;
        else if (resident[c] || (double)ce >= stream_ratio * ch[c].edges()) out.mode[c] = 2;
        else if (hot_mode && pass == 0 && hhi[c] > hlo[c]) out.mode[c] = 2;
        else { out.mode[c] = 3; out.need_bitmap = true; }
    }
}

int gather_list(int v0, int v1, const uint32_t* bitmap, const ull* idx, int32_t* vids, ull* off) {
    int k = 0;
    for (int v = v0; v < v1;) {
        const uint32_t w = bitmap[v >> 5] >> (v & 31);
        if (!w) { v = (v | 31) + 1; continue; }
        v += __builtin_ctz(w);
        if (v >= v1) break;
        vids[k++] = v;
        v++;
    }
    off[0] = 0;
    for (int i = 0; i < k; i++) off[i + 1] = off[i] + (idx[vids[i] + 1] - idx[vids[i]]);
    return k;
}

double tau_from_timings(double t_stream, const double* t_g, const double* f) {
    double tau;
    if (t_g[0] >= t_stream) tau = f[0] * t_stream / t_g[0];
    else if (t_g[2] < t_stream) tau = f[2] * t_stream / t_g[2];
    else {
        const int j = t_g[1] >= t_stream ? 1 : 2;
        tau = f[j - 1] + (f[j] - f[j - 1]) * (t_stream - t_g[j - 1]) / (t_g[j] - t_g[j - 1]);
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
    std::vector<Chunk> ch = plan_chunks(n, off, cap);
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
    *resident = cache_chunks(ch, free_bytes, reserve);
    return EXCENT_OK;
}

extern "C" int excent_hot_select(int n, const unsigned long long* off, unsigned long long budget, const uint16_t* score,
                                 int* nh, int32_t* ids, unsigned long long* hoff, uint32_t* bits,
                                 unsigned long long* threshold) {
    EX_CHECK_ARG(n >= 1 && off && nh, "bad argument");
    HotSet H = hot_select(n, off, budget, score, omp_get_max_threads());
    *nh = (int)H.ids.size();
    if (ids) memcpy(ids, H.ids.data(), H.ids.size() * sizeof(int32_t));
    if (hoff) memcpy(hoff, H.off.data(), H.off.size() * sizeof(ull));
    if (bits) memcpy(bits, H.bits.data(), H.bits.size() * sizeof(uint32_t));
    if (threshold) *threshold = H.T;
    return EXCENT_OK;
}

extern "C" int excent_fetch_plan(int nc, const unsigned long long* chunk_edges, const unsigned long long* cnt,
                                 const uint8_t* resident, const uint8_t* loaded, double stream_ratio, int hot_mode,
                                 int pass, const int* hlo, const int* hhi, uint8_t* mode,
                                 unsigned long long* pend_v, unsigned long long* demand, int* need_bitmap) {
    EX_CHECK_ARG(nc >= 1 && chunk_edges && cnt && resident && loaded && hlo && hhi && mode, "bad argument");
    std::vector<Chunk> ch(nc);
    for (int c = 0; c < nc; c++) ch[c] = {c, c + 1, 0, chunk_edges[c]};
    FetchPlan P;
    fetch_plan(ch, cnt, std::vector<uint8_t>(resident, resident + nc), std::vector<uint8_t>(loaded, loaded + nc),
               stream_ratio, hot_mode != 0, pass, std::vector<int>(hlo, hlo + nc), std::vector<int>(hhi, hhi + nc), P);
    memcpy(mode, P.mode.data(), nc);
    if (pend_v) *pend_v = P.pend_v;
    if (demand) *demand = P.demand;
    if (need_bitmap) *need_bitmap = P.need_bitmap;
    return EXCENT_OK;
}

extern "C" int excent_gather_list(int v0, int v1, const uint32_t* bitmap, const unsigned long long* idx, int32_t* vids,
                                  unsigned long long* off, int* k) {
    EX_CHECK_ARG(v0 >= 0 && v0 <= v1 && bitmap && idx && vids && off && k, "bad argument");
    *k = gather_list(v0, v1, bitmap, idx, vids, off);
    return EXCENT_OK;
}

extern "C" double excent_tau(double t_stream, const double* t_g, const double* f) {
    return tau_from_timings(t_stream, t_g, f);
}
