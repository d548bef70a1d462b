// runtime.cpp -- the excent command line: the reference's option surface and
// stdout lines (src/excent.cu:242-806) over the B200 engine. One host control
// thread plans each pass (fetch plan per chunk: skip, HBM-cached, streamed,
// gathered), stages streamed chunks and gathered lists through two pinned
// slots with deduplicated page readahead, and drives the device engine
// through its C entry points (include/excent_b200.h).
#include <omp.h>
#include <sys/resource.h>
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.h"
#include "egr.h"
#include "planner.h"

namespace excent {

typedef std::chrono::steady_clock Clock;
static double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

struct Options {
    std::string graph;
    double chunk_medges = 0, stream_ratio = 2.0, reserve_mb = 256, target_chunks = 16, min_chunk_medges = 4;
    double list_frac = 0.5;
    bool use_cache = true;
    std::string cache_mode = "auto", hot_when = "end", hot_order = "sweep", trace_file, hot_rank;
    bool stream_auto = true, recalibrate = false, dedup = true, count_pushes = false;
    int group_opt = 0;
    std::string zero_copy = "auto";
    int max_passes = 100000;
    std::string dump, measure;
    double alpha = -1, beta = 1.0, lambda = -1, eps_pr = 0.01, eps_katz = -1, eps_ev = -1;
    // B200 additions
    int device = 0;
    double budget_gb = 0;      // cap on the free device memory used for sizing (0: none)
    bool device_loop = false;  // fully cached graphs: load at setup, run the on-device pass loop
    bool ev_init_fp64 = false; // eigenvector initial residual from the FP64 lambda1
    int hub_targets = -1;      // shared-memory aggregation of the top-degree targets (-1: auto)
    int hub_order = 1;         // device loop: the high-degree lists 0 in table order, 1 first, 2 last
    std::string host_cache = "off";   // pinned: entries past the HBM cache read in place from pinned host memory
};

static const char* USAGE =
    "usage: %s graph.egr --measure pr|katz|ev|all [--alpha A] [--beta 1] [--lambda L] "
    "[--eps-pr 0.01] [--eps-katz E] [--eps-ev E] [--chunk-medges auto] [--target-chunks 16] "
    "[--min-chunk-medges 4] [--list-frac 0.5] [--stream-ratio auto|R] "
    "[--reserve-mb 256] [--cache chunks|hot|none] [--max-passes N] [--dump PREFIX]\n";

// Option parse of src/excent.cu:251-316: same flags, defaults and messages.
// Returns 0 on success, 1 (with the message printed to stderr) otherwise.
static int parse_options(int argc, char** argv, Options& o) {
    if (argc < 2) { fprintf(stderr, USAGE, argv[0]); return 1; }
    o.graph = argv[1];
    for (int i = 2; i < argc; i++) {
        const std::string a = argv[i];
        auto next = [&](const char*& v) {
            if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); return false; }
            v = argv[++i];
            return true;
        };
        const char* v = nullptr;
        bool ok = true;
        if (a == "--chunk-medges") { if ((ok = next(v))) o.chunk_medges = atof(v); }
        else if (a == "--target-chunks") { if ((ok = next(v))) o.target_chunks = atof(v); }
        else if (a == "--min-chunk-medges") { if ((ok = next(v))) o.min_chunk_medges = atof(v); }
        else if (a == "--list-frac") { if ((ok = next(v))) o.list_frac = atof(v); }
        else if (a == "--stream-ratio") {
            if ((ok = next(v))) { o.stream_auto = !strcmp(v, "auto"); if (!o.stream_auto) o.stream_ratio = atof(v); }
        } else if (a == "--dedup") {
            if ((ok = next(v))) {
                if (strcmp(v, "on") && strcmp(v, "off")) { fprintf(stderr, "--dedup must be on or off\n"); return 1; }
                o.dedup = !strcmp(v, "on");
            }
        } else if (a == "--hot-rank") { if ((ok = next(v))) o.hot_rank = v; }
        else if (a == "--recalibrate") o.recalibrate = true;
        else if (a == "--reserve-mb") { if ((ok = next(v))) o.reserve_mb = atof(v); }
        else if (a == "--no-cache") o.use_cache = false;
        else if (a == "--cache") { if ((ok = next(v))) o.cache_mode = v; }
        else if (a == "--hot-when") { if ((ok = next(v))) o.hot_when = v; }
        else if (a == "--hot-order") { if ((ok = next(v))) o.hot_order = v; }
        else if (a == "--trace-pending") { if ((ok = next(v))) o.trace_file = v; }
        else if (a == "--group") { if ((ok = next(v))) o.group_opt = atoi(v); }
        else if (a == "--count-pushes") o.count_pushes = true;
        else if (a == "--zero-copy") { if ((ok = next(v))) o.zero_copy = v; }
        else if (a == "--max-passes") { if ((ok = next(v))) o.max_passes = atoi(v); }
        else if (a == "--dump") { if ((ok = next(v))) o.dump = v; }
        else if (a == "--measure") { if ((ok = next(v))) o.measure = v; }
        else if (a == "--alpha") { if ((ok = next(v))) o.alpha = atof(v); }
        else if (a == "--beta") { if ((ok = next(v))) o.beta = atof(v); }
        else if (a == "--lambda") { if ((ok = next(v))) o.lambda = atof(v); }
        else if (a == "--eps-pr") { if ((ok = next(v))) o.eps_pr = atof(v); }
        else if (a == "--eps-katz") { if ((ok = next(v))) o.eps_katz = atof(v); }
        else if (a == "--eps-ev") { if ((ok = next(v))) o.eps_ev = atof(v); }
        else if (a == "--device") { if ((ok = next(v))) o.device = atoi(v); }
        else if (a == "--gpu-budget-gb") { if ((ok = next(v))) o.budget_gb = atof(v); }
        else if (a == "--device-loop") o.device_loop = true;
        else if (a == "--hub-targets") {
            if ((ok = next(v))) {
                if (!strcmp(v, "auto")) o.hub_targets = -1;
                else if (!strcmp(v, "off")) o.hub_targets = 0;
                else o.hub_targets = atoi(v);
                if (o.hub_targets < -1) { fprintf(stderr, "--hub-targets must be auto, off or a count\n"); return 1; }
            }
        }
        else if (a == "--host-cache") {
            if ((ok = next(v))) {
                if (strcmp(v, "pinned") && strcmp(v, "off")) { fprintf(stderr, "--host-cache must be pinned or off\n"); return 1; }
                o.host_cache = v;
            }
        }
        else if (a == "--hub-order") {
            if ((ok = next(v))) {
                if (!strcmp(v, "table")) o.hub_order = 0;
                else if (!strcmp(v, "first")) o.hub_order = 1;
                else if (!strcmp(v, "last")) o.hub_order = 2;
                else { fprintf(stderr, "--hub-order must be first, last or table\n"); return 1; }
            }
        }
        else { fprintf(stderr, "unknown option %s\n", a.c_str()); return 1; }
        if (!ok) return 1;
    }
    if (!o.use_cache) o.cache_mode = "none";
    if (o.cache_mode != "chunks" && o.cache_mode != "hot" && o.cache_mode != "none" && o.cache_mode != "auto") {
        fprintf(stderr, "--cache must be auto, chunks, hot or none\n");
        return 1;
    }
    return 0;
}

static std::pair<long, long> faults() {
    struct rusage ru;
    getrusage(RUSAGE_SELF, &ru);
    return {(long)ru.ru_majflt, (long)ru.ru_minflt};
}

#define RT_CK(x) do { const int rc_ = (x); if (rc_ != EXCENT_OK) { \
    fprintf(stderr, "excent: %s\n", excent_last_error()); return 1; } } while (0)

static const char* MNAME[3] = {"pr", "katz", "ev"};

static int run(const Options& o) {
    const auto T0 = Clock::now();
    excent_measures M;
    if (excent_measures_make(&M, o.measure.c_str(), o.alpha, o.beta, o.lambda, o.eps_pr, o.eps_katz, o.eps_ev) !=
        EXCENT_OK) {
        fprintf(stderr, "%s\n", excent_last_error());
        return 1;
    }
    if (o.ev_init_fp64) M.flags |= EXCENT_EV_INIT_FP64;
    EgrFile g;
    if (g.open(o.graph.c_str(), 16, /*offsets_in_ram=*/false, true) != EXCENT_OK) {
        fprintf(stderr, "%s\n", excent_last_error());
        return 1;
    }
    const int n = g.n;
    const ull m = g.m;
    const ull cap = chunk_cap(m, o.chunk_medges, o.target_chunks, o.min_chunk_medges);
    const std::vector<Chunk> chunks = plan_chunks(n, g.offsets(), cap);
    const int nc = (int)chunks.size();
    ull max_chunk_edges = 0;
    int max_chunk_verts = 0;
    for (const Chunk& c : chunks) {
        max_chunk_edges = std::max(max_chunk_edges, c.edges());
        max_chunk_verts = std::max(max_chunk_verts, c.v1 - c.v0);
    }
    const auto T_open = Clock::now();
    printf("graph: n=%d m=%llu chunks=%d (cap %llu, max %llu edges, %d vertices)  open %.2fs\n", n, m, nc, cap,
           max_chunk_edges, max_chunk_verts, secs(T0, T_open));
    fflush(stdout);

    std::vector<int> cv0(nc);
    std::vector<ull> ce(nc + 1);
    for (int c = 0; c < nc; c++) { cv0[c] = chunks[c].v0; ce[c] = chunks[c].e0; }
    ce[nc] = m;
    excent_engine* e = nullptr;
    RT_CK(excent_engine_create(o.device, n, m, &M, nc, cv0.data(), ce.data(), &e));
    struct Guard { excent_engine* e; ~Guard() { excent_engine_destroy(e); } } guard{e};
    {   // offsets in 16M-entry pieces (src/excent.cu:360-369)
        const size_t B = (size_t)1 << 24;
        std::vector<ull> stage(std::min(B, (size_t)n + 1));
        for (size_t v0 = 0; v0 < (size_t)n + 1; v0 += B) {
            const size_t cnt = std::min(B, (size_t)n + 1 - v0);
            RT_CK(g.read_offsets(v0, cnt, stage.data()));
            RT_CK(excent_engine_upload_offsets(e, stage.data(), v0, cnt));
        }
    }
    if (!o.trace_file.empty()) RT_CK(excent_engine_trace(e, 1));
    RT_CK(excent_engine_init(e));

    excent_device_info_t di;
    RT_CK(excent_device_info(o.device, &di));
    const bool zc = o.zero_copy == "on" || (o.zero_copy == "auto" && di.integrated);
    RT_CK(excent_engine_slots_create(e, max_chunk_edges, max_chunk_verts, zc ? 1 : 0));
    int32_t *s_edges[2], *s_vids[2];
    ull* s_off[2];
    for (int s = 0; s < 2; s++) RT_CK(excent_engine_slot_buffers(e, s, &s_edges[s], &s_vids[s], &s_off[s]));

    auto free_mem = [&]() -> int {
        if (excent_device_info(o.device, &di) != EXCENT_OK) {
            fprintf(stderr, "excent: %s\n", excent_last_error());
            return 1;
        }
        return 0;
    };
    const ull reserve = (ull)(o.reserve_mb * (1 << 20));
    std::string cache_mode = o.cache_mode;
    auto avail_free = [&]() -> ull {
        ull f = di.free_bytes;
        if (o.budget_gb > 0) f = std::min<ull>(f, (ull)(o.budget_gb * (1ull << 30)));
        return f;
    };
    if (free_mem()) return 1;
    if (o.host_cache == "pinned") cache_mode = "chunks";   // an HBM chunk prefix, the rest in host memory
    if (cache_mode == "auto") {   // src/excent.cu:402-409
        const ull freeB = avail_free();
        const bool fits = freeB > reserve && m * sizeof(int) <= freeB - reserve;
        cache_mode = fits ? "chunks" : "hot";
        printf("cache: auto -> %s\n", fits ? "chunks (the whole graph fits)" : "high-degree lists");
    }
    const bool hot_mode_req = cache_mode == "hot";
    std::vector<uint8_t> resident(nc, 0), loaded(nc, 0);
    int n_resident = 0;
    ull resident_edges = 0;
    if (cache_mode == "chunks") {   // whole chunks in file order (src/excent.cu:410-421), one arena
        if (free_mem()) return 1;
        n_resident = cache_chunks(chunks, avail_free(), reserve);
        while (n_resident > 0) {
            if (excent_engine_reserve_cache(e, chunks[n_resident - 1].e1) == EXCENT_OK) break;
            n_resident--;   // the allocation failed: keep fewer chunks
        }
        for (int c = 0; c < n_resident; c++) { resident[c] = 1; resident_edges += chunks[c].edges(); }
        if (n_resident > 0) {   // shared-memory sums for the top-degree targets of cached pushes
            const int k = o.hub_targets < 0 ? std::min(M.nm == 1 ? 16384 : 4096, n) : o.hub_targets;
            if (k > 0 && excent_engine_set_hub_targets(e, k) != EXCENT_OK)   // an optimisation: go on without it
                fprintf(stderr, "excent: hub targets off (%s)\n", excent_last_error());
        }
    }
    RT_CK(excent_engine_set_hub_order(e, o.hub_order));
    int nh = 0;
    ull hot_edges = 0, hot_deg_min = 0;
    bool hot_mode = hot_mode_req;
    std::vector<int> hlo(nc, 0), hhi(nc, 0);
    if (hot_mode) {   // src/excent.cu:428-513
        if (free_mem()) return 1;
        const ull bits = (((ull)n + 31) / 32) * sizeof(uint32_t);
        const ull freeB = avail_free();
        const ull budget = freeB > reserve + bits ? freeB - reserve - bits : 0;
        std::vector<uint16_t> score;
        if (!o.hot_rank.empty()) {
            score.resize(n);
            FILE* f = fopen(o.hot_rank.c_str(), "rb");
            if (!f || fread(score.data(), sizeof(uint16_t), n, f) != (size_t)n) {
                fprintf(stderr, "--hot-rank: cannot read %d entries from %s\n", n, o.hot_rank.c_str());
                if (f) fclose(f);
                return 1;
            }
            fclose(f);
        }
        HotSet H = hot_select(n, g.offsets(), budget, score.empty() ? nullptr : score.data(), 16);
        nh = (int)H.ids.size();
        hot_edges = H.edges();
        hot_deg_min = H.T;
        bool ok = nh > 0;
        if (ok && excent_engine_hot_setup(e, nh, H.ids.data(), H.off.data(), H.bits.data()) != EXCENT_OK) ok = false;
        if (!ok) {
            fprintf(stderr, "degree cache: could not allocate %d lists (%.2f GB); running without a cache\n", nh,
                    hot_edges * 4.0 / 1e9);
            nh = 0;
            hot_edges = 0;
        } else {
            for (int c = 0; c < nc; c++) {
                hlo[c] = (int)(std::lower_bound(H.ids.begin(), H.ids.end(), chunks[c].v0) - H.ids.begin());
                hhi[c] = (int)(std::lower_bound(H.ids.begin(), H.ids.end(), chunks[c].v1) - H.ids.begin());
            }
        }
    }

    // tau: cached per graph and machine, else measured on the middle chunk (src/excent.cu:515-579)
    double stream_ratio = o.stream_ratio, t_calib = 0;
    bool stream_auto = o.stream_auto;
    std::string tau_file;
    if (stream_auto) {
        const char* home = getenv("HOME");
        std::string base = o.graph.substr(o.graph.find_last_of('/') + 1);
        std::string dir = std::string(home ? home : ".") + "/.cache";
        mkdir(dir.c_str(), 0755);
        dir += "/excent";
        mkdir(dir.c_str(), 0755);
        tau_file = dir + "/" + base + "." + std::to_string(n) + "." + std::to_string(m) + ".tau";
        FILE* f = o.recalibrate ? nullptr : fopen(tau_file.c_str(), "r");
        if (f) {
            if (fscanf(f, "%lf %lf", &stream_ratio, &t_calib) == 2) {
                printf("fetch rule: tau = %.3f (measured earlier on this machine in %.2fs, %s)\n", stream_ratio,
                       t_calib, tau_file.c_str());
                stream_auto = false;
            }
            fclose(f);
        }
    }
    if (stream_auto) {
        const auto c0 = Clock::now();
        const Chunk& ch = chunks[nc / 2];
        g.drop_cache(ch.e0, ch.e1, ch.v0, ch.v1);
        auto a = Clock::now();
        RT_CK(g.read_edges(ch.e0, ch.e1, s_edges[0]));
        const double t_stream = secs(a, Clock::now());
        const double fr[3] = {0.05, 0.15, 0.4};
        double f_got[3], t_g[3];
        std::vector<std::pair<ull, int>> byd;
        for (int v = ch.v0; v < ch.v1; v++) byd.push_back({g.degree(v), v});
        std::sort(byd.begin(), byd.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        for (int j = 0; j < 3; j++) {
            std::vector<int> pick;
            for (ull acc = 0; acc < fr[j] * ch.edges() && pick.size() < byd.size();) {
                acc += byd[pick.size()].first;
                pick.push_back(byd[pick.size()].second);
            }
            std::sort(pick.begin(), pick.end());
            g.drop_cache(ch.e0, ch.e1, ch.v0, ch.v1);
            a = Clock::now();
            const int k = (int)pick.size();
            for (int i = 0; i < k; i++) s_vids[0][i] = pick[i];
            s_off[0][0] = 0;
            for (int i = 0; i < k; i++) s_off[0][i + 1] = s_off[0][i] + g.degree(s_vids[0][i]);
            ull pg, rn;
            if (o.dedup) g.prefetch_lists(s_vids[0], k, &pg, &rn);
#pragma omp parallel for schedule(dynamic, 256) num_threads(16)
            for (int i = 0; i < k; i++)
                memcpy(s_edges[0] + s_off[0][i], g.edges(s_vids[0][i]), g.degree(s_vids[0][i]) * sizeof(int32_t));
            t_g[j] = secs(a, Clock::now());
            f_got[j] = ch.edges() ? (double)s_off[0][k] / ch.edges() : 0.0;
        }
        stream_ratio = tau_from_timings(t_stream, t_g, f_got);
        t_calib = secs(c0, Clock::now());
        printf("fetch rule: tau = %.3f (stream %.3fs; gather %.3fs / %.3fs / %.3fs at demand %.3f / %.3f / %.3f)  "
               "calibrate %.2fs\n", stream_ratio, t_stream, t_g[0], t_g[1], t_g[2], f_got[0], f_got[1], f_got[2],
               t_calib);
        if (FILE* f = fopen(tau_file.c_str(), "w")) { fprintf(f, "%.6f %.4f\n", stream_ratio, t_calib); fclose(f); }
    } else if (tau_file.empty()) {
        printf("fetch rule: tau = %.3f (given)\n", stream_ratio);
    }

    // --device-loop on a fully cached graph: load every chunk now and run the on-device pass loop
    // --host-cache pinned: the chunks past the HBM prefix are read once into pinned host memory and
    // the on-device pass loop pushes from there in place
    const bool host_loop = o.host_cache == "pinned" && !hot_mode;
    const bool dev_loop = (o.device_loop && cache_mode == "chunks" && n_resident == nc && !hot_mode) || host_loop;
    ull host_gb_edges = 0;
    if (dev_loop) {
        for (int c = 0; c < n_resident; c++) {
            RT_CK(g.read_edges(chunks[c].e0, chunks[c].e1, s_edges[0]));
            RT_CK(excent_engine_load_cache(e, chunks[c].e0, chunks[c].e1, s_edges[0]));
            loaded[c] = 1;
        }
        if (host_loop) {
            int32_t* h = nullptr;
            ull first = 0;
            RT_CK(excent_engine_host_cache(e, &h, &first));
            if (h) RT_CK(g.read_edges(first, m, h));
            host_gb_edges = m - first;
            printf("host cache: pinned, %.2f GB (%d chunks past the GPU cache), lists read in place over the host link\n",
                   host_gb_edges * 4.0 / 1e9, nc - n_resident);
        }
    }
    RT_CK(excent_engine_sync(e));
    const auto T_setup = Clock::now();
    printf("staging: %s\n", zc ? "zero copy (pinned, GPU-mapped buffers read in place)"
                               : "pinned host buffers copied to the GPU");
    if (hot_mode && !o.hot_rank.empty())
        printf("GPU cache ranked by passes pending (%s): %d vertices (%.1f%% of edges, %.2f GB)  setup %.2fs\n",
               o.hot_rank.c_str(), nh, 100.0 * hot_edges / m, hot_edges * 4.0 / 1e9, secs(T_open, T_setup));
    else if (hot_mode)
        printf("GPU degree cache: %d vertices with degree >= %llu (%.1f%% of edges, %.2f GB)  setup %.2fs\n", nh,
               hot_deg_min, 100.0 * hot_edges / m, hot_edges * 4.0 / 1e9, secs(T_open, T_setup));
    else
        printf("GPU edge cache: %d/%d chunks resident (%.1f%% of edges)  setup %.2fs\n", n_resident, nc,
               100.0 * resident_edges / m, secs(T_open, T_setup));
    fflush(stdout);

    // ---- passes
    double t_io = 0, t_wait = 0, t_snap = 0;
    ull bytes_stream = 0, bytes_gather = 0;
    long tot_maj = 0, tot_min = 0;
    ull tot_pages = 0, tot_runs = 0;
    int pass = 0;
    std::vector<std::pair<int, int>> hot_ranges;
    if (o.hot_order == "ranges") { for (int c = 0; c < nc; c++) if (hhi[c] > hlo[c]) hot_ranges.push_back({hlo[c], hhi[c]}); }
    else if (nh) hot_ranges.push_back({0, nh});
    std::vector<ull> cnt(2 * (size_t)nc);
    std::vector<uint32_t> bitmap(((size_t)n + 31) / 32);
    FetchPlan plan;
    int cur = 0;
    bool busy[2] = {false, false};
    const auto acquire = [&](int s) -> int {
        if (busy[s]) {
            const auto a = Clock::now();
            const int rc = excent_engine_slot_wait(e, s);
            t_wait += secs(a, Clock::now());
            busy[s] = false;
            return rc;
        }
        return EXCENT_OK;
    };
    auto launch_hot = [&](int after_slots) -> int {
        for (auto [lo, hi] : hot_ranges) EX_TRY(excent_engine_push_hot(e, lo, hi, after_slots));
        return EXCENT_OK;
    };
    if (dev_loop) {
        const auto a = Clock::now();
        RT_CK(excent_engine_solve(e, o.list_frac, o.max_passes, 1));
        excent_stats st;
        std::vector<excent_pass_log> log(std::min(o.max_passes, 1 << 17) + 1);
        RT_CK(excent_engine_stats(e, &st, log.data(), (int)log.size()));
        pass = st.passes;
        if (host_loop) {   // the lists read in place are this mode's gathered bytes
            ull hp = 0;
            RT_CK(excent_engine_host_pushed(e, &hp));
            bytes_gather += hp * 4;
        }
        for (int p = 0; p < pass && p < (int)log.size(); p++)
            printf("pass %3d: pending %llu v, demand ratio %.4f | resident %d stream %d gather %d | cached high-degree "
                   "pending %llu | faults major %ld minor %ld | gather pages %llu runs %llu\n",
                   p, log[p].pending, (double)log[p].demand / m, log[p].n_list + log[p].n_range, 0, 0, 0ull, 0L, 0L,
                   0ull, 0ull);
        t_wait += secs(a, Clock::now());
    }
    for (; !dev_loop && pass < o.max_passes; pass++) {
        const auto a = Clock::now();
        const auto f0 = faults();
        ull pass_pages = 0, pass_runs = 0;
        const bool hot_skip = hot_mode && nh > 0 && pass > 0;
        ull hotpend = 0;
        RT_CK(excent_engine_snapshot(e, hot_skip ? 1 : 0, cnt.data(), &hotpend, nullptr));
        fetch_plan(chunks, cnt.data(), resident, loaded, stream_ratio, hot_mode, pass, hlo, hhi, plan);
        if (plan.need_bitmap) RT_CK(excent_engine_bitmap(e, bitmap.data()));
        t_snap += secs(a, Clock::now());
        if (plan.pend_v == 0 && hotpend == 0) break;
        int nres = 0, nstream = 0, ngather = 0;
        if (hot_skip && hotpend && o.hot_when != "end") RT_CK(launch_hot(0));
        for (int c = 0; c < nc; c++) nres += plan.mode[c] == 1;
        if (nres) RT_CK(excent_engine_push_cached(e, plan.mode.data(), cnt.data(), o.list_frac));
        for (int c = 0; c < nc; c++) {
            if (plan.mode[c] < 2) continue;
            const Chunk& ch = chunks[c];
            const int s = cur;
            cur ^= 1;
            RT_CK(acquire(s));
            const auto io0 = Clock::now();
            if (plan.mode[c] == 2) {
                nstream++;
                RT_CK(g.read_edges(ch.e0, ch.e1, s_edges[s]));
                bytes_stream += ch.edges() * sizeof(int32_t);
                t_io += secs(io0, Clock::now());
                const bool fill_hot = hot_mode && pass == 0 && hhi[c] > hlo[c] && nh > 0;
                RT_CK(excent_engine_push_stream(e, s, c, cnt.data(), o.list_frac, resident[c] ? 1 : 0,
                                                fill_hot ? hlo[c] : 0, fill_hot ? hhi[c] : 0));
                if (resident[c]) loaded[c] = 1;
            } else {
                ngather++;
                const int k = gather_list(ch.v0, ch.v1, bitmap.data(), g.offsets(), s_vids[s], s_off[s]);
                const ull ne = s_off[s][k];
                if (o.dedup) {
                    ull pg, rn;
                    g.prefetch_lists(s_vids[s], k, &pg, &rn);
                    pass_pages += pg;
                    pass_runs += rn;
                }
                int32_t* dst = s_edges[s];
                const ull* so = s_off[s];
                const int32_t* sv = s_vids[s];
#pragma omp parallel for schedule(dynamic, 256) num_threads(16)
                for (int i = 0; i < k; i++) memcpy(dst + so[i], g.edges(sv[i]), g.degree(sv[i]) * sizeof(int32_t));
                bytes_gather += ne * sizeof(int32_t) + (size_t)k * (sizeof(int32_t) + sizeof(ull));
                t_io += secs(io0, Clock::now());
                RT_CK(excent_engine_push_gather(e, s, k, ne));
            }
            busy[s] = true;
        }
        if (hot_skip && o.hot_when != "start") RT_CK(launch_hot(1));
        const auto w0 = Clock::now();
        RT_CK(excent_engine_sync(e));
        busy[0] = busy[1] = false;
        t_wait += secs(w0, Clock::now());
        const auto f1 = faults();
        tot_maj += f1.first - f0.first;
        tot_min += f1.second - f0.second;
        tot_pages += pass_pages;
        tot_runs += pass_runs;
        printf("pass %3d: pending %llu v, demand ratio %.4f | resident %d stream %d gather %d | cached high-degree "
               "pending %llu | faults major %ld minor %ld | gather pages %llu runs %llu\n",
               pass, plan.pend_v, (double)plan.demand / m, nres, nstream, ngather, hotpend, f1.first - f0.first,
               f1.second - f0.second, pass_pages, pass_runs);
    }
    const auto T_iter = Clock::now();

    std::vector<double> sum(M.nm, 0.0);
    {
        std::vector<float> vals(n);
        for (int i = 0; i < M.nm; i++) {
            RT_CK(excent_engine_read(e, i, 0, vals.data(), 0, n));
            for (int v = 0; v < n; v++) sum[i] += vals[v];
            if (!o.dump.empty()) {
                const std::string p = o.dump + "." + MNAME[M.kind[i]] + ".bin";
                FILE* df = fopen(p.c_str(), "wb");
                if (!df || fwrite(vals.data(), sizeof(float), n, df) != (size_t)n) {
                    fprintf(stderr, "cannot write %s\n", p.c_str());
                    if (df) fclose(df);
                    return 1;
                }
                fclose(df);
            }
        }
    }
    if (!o.trace_file.empty()) {
        std::vector<uint16_t> tr(n);
        RT_CK(excent_engine_read_trace(e, tr.data()));
        FILE* tf = fopen(o.trace_file.c_str(), "wb");
        if (!tf || fwrite(tr.data(), sizeof(uint16_t), n, tf) != (size_t)n) {
            fprintf(stderr, "cannot write %s\n", o.trace_file.c_str());
            if (tf) fclose(tf);
            return 1;
        }
        fclose(tf);
    }
    const auto T_end = Clock::now();
    excent_stats st;
    RT_CK(excent_engine_stats(e, &st, nullptr, 0));
    printf("passes %d  measure %s (n=%d):", pass, o.measure.c_str(), n);
    for (int i = 0; i < M.nm; i++) printf("  %s sum %.6e", MNAME[M.kind[i]], sum[i]);
    printf("\n");
    if (o.count_pushes) printf("edges pushed: %.2f x |E|\n", m ? (double)st.pushed / m : 0.0);
    printf("launches from GPU memory: %llu pending-only, %llu whole-range\n", st.n_list, st.n_range);
    printf("bytes shipped: stream %.2f GB, gather %.2f GB (graph edges %.2f GB)\n", bytes_stream / 1e9,
           bytes_gather / 1e9, m * 4.0 / 1e9);
    printf("page faults in passes: major %ld, minor %ld | gather dedup %s: %llu pages in %llu runs\n", tot_maj, tot_min,
           o.dedup ? "on" : "off", tot_pages, tot_runs);
    printf("time: open %.2fs setup %.2fs passes %.2fs [cpu io %.2fs, gpu wait %.2fs, snapshot %.2fs] result %.2fs | "
           "internal total %.2fs\n", secs(T0, T_open), secs(T_open, T_setup), secs(T_setup, T_iter), t_io, t_wait, t_snap,
           secs(T_iter, T_end), secs(T0, T_end));
    const double tp = secs(T_setup, T_iter);
    printf("throughput: %.3f GTEPS (%llu adjacency entries pushed in %.3fs of passes); residual sum (FP64):", tp > 0 ? st.pushed / tp / 1e9 : 0.0,
           st.pushed, tp);
    for (int i = 0; i < M.nm; i++) printf(" %s %.6e", MNAME[M.kind[i]], st.rsum[i]);
    printf("\n");
    return 0;
}

}  // namespace excent

extern "C" int excent_cli_main(int argc, char** argv) {
    excent::Options o;
    if (excent::parse_options(argc, argv, o)) return 1;
    return excent::run(o);
}
