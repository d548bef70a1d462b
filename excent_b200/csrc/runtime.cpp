// runtime.cpp -- the excent command line over the B200 engine.
//
// The option surface, messages and stdout lines are the reference's
// (src/excent.cu:242-806): that is the drop-in contract. Behind it a Run
// object opens the graph file, creates the device engine, sizes the GPU
// caches, settles the stream/gather rule tau (cache file or a cold-cache
// probe), then drives the passes: on the device alone (--device-loop,
// --host-cache pinned), or host-planned, where each pass's chunks are
// skipped, pushed from HBM, streamed, or gathered list by list through the
// engine's two pinned staging slots (Staging) with page readahead and a
// byte-balanced parallel copy of the lists.
#include <omp.h>
#include <sys/resource.h>
#include <sys/stat.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
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
    int hub_order = -1;        // the high-degree lists 0 in table order, 1 first, 2 last, -1 by the chunk count
    std::string host_cache = "off";   // pinned: entries past the HBM cache read in place from pinned host memory
    int chunk_sweep = -1;      // cached pushes one chunk per launch (1), in one launch (0), -1 by the chunk count
    double sweep_demand = 0.5; // ... in the passes whose pending entries reach this fraction of m
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
        else if (a == "--ev-init") {
            if ((ok = next(v))) {
                if (strcmp(v, "fp64") && strcmp(v, "reference")) {
                    fprintf(stderr, "--ev-init must be fp64 or reference\n");
                    return 1;
                }
                o.ev_init_fp64 = !strcmp(v, "fp64");
            }
        }
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
        else if (a == "--chunk-sweep") {
            if ((ok = next(v))) {
                if (strcmp(v, "on") && strcmp(v, "off") && strcmp(v, "auto")) {
                    fprintf(stderr, "--chunk-sweep must be on, off or auto\n");
                    return 1;
                }
                o.chunk_sweep = !strcmp(v, "auto") ? -1 : !strcmp(v, "on");
            }
        }
        else if (a == "--sweep-demand") {
            if ((ok = next(v))) {
                o.sweep_demand = atof(v);
                if (!(o.sweep_demand >= 0.0)) { fprintf(stderr, "--sweep-demand must be a fraction >= 0\n"); return 1; }
            }
        }
        else if (a == "--hub-order") {
            if ((ok = next(v))) {
                if (!strcmp(v, "table")) o.hub_order = 0;
                else if (!strcmp(v, "first")) o.hub_order = 1;
                else if (!strcmp(v, "last")) o.hub_order = 2;
                else if (!strcmp(v, "launch-first")) o.hub_order = 3;
                else if (!strcmp(v, "auto")) o.hub_order = -1;
                else { fprintf(stderr, "--hub-order must be first, last, launch-first, table or auto\n"); return 1; }
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

// ------------------------------------------------------------------ helpers

static std::pair<long, long> fault_counts() {
    struct rusage ru;
    getrusage(RUSAGE_SELF, &ru);
    return {(long)ru.ru_majflt, (long)ru.ru_minflt};
}

#define RT_CK(x) do { const int rc_ = (x); if (rc_ != EXCENT_OK) { \
    fprintf(stderr, "excent: %s\n", excent_last_error()); return 1; } } while (0)

static const char* MNAME[3] = {"pr", "katz", "ev"};

// What a run spends and ships, in the terms of the reference's summary lines.
struct Tally {
    double io = 0, wait = 0, snap = 0;   // host reads/gathers, waits on the GPU, snapshots + plans
    ull stream_bytes = 0, gather_bytes = 0;
    long major = 0, minor = 0;
    ull pages = 0, runs = 0;
};

// Copy the k pending lists (vids, prefix offsets off[k+1]) out of the mapped
// file into dst. The output is cut into equal shares of entries, one per
// reader thread, so a share may start or end inside a list and one long list
// is copied by several threads.
static void copy_lists(const GraphFile& g, const int32_t* vids, const ull* off, int k, int32_t* dst, int threads) {
    const ull total = off[k];
    if (total == 0) return;
    const int team = (int)std::max<ull>(1, std::min<ull>((ull)threads, total / 4096 + 1));
#pragma omp parallel num_threads(team)
    {
        const int t = omp_get_thread_num();
        const ull b0 = total * t / team, b1 = total * (t + 1) / team;
        // first list holding entry b0
        int i = (int)(std::upper_bound(off, off + k + 1, b0) - off) - 1;
        for (ull b = b0; b < b1 && i < k; i++) {
            const ull lo = std::max(b, off[i]), hi = std::min(b1, off[i + 1]);
            if (hi > lo) memcpy(dst + lo, g.list(vids[i]) + (lo - off[i]), (hi - lo) * sizeof(int32_t));
            b = hi;
        }
    }
}

// The engine's two staging slots seen from the host: which one is next, its
// buffers, and the work that fills one (a streamed chunk, or the gathered
// lists of a chunk's pending vertices).
class Staging {
public:
    Staging(excent_engine* e, const GraphFile& g, Tally& tally, bool dedup) : e_(e), g_(g), t_(tally), dedup_(dedup) {}

    int create(ull max_entries, int max_vertices, bool zero_copy) {
        EX_TRY(excent_engine_slots_create(e_, max_entries, max_vertices, zero_copy ? 1 : 0));
        for (int s = 0; s < 2; s++) EX_TRY(excent_engine_slot_buffers(e_, s, &entries_[s], &vids_[s], &off_[s]));
        return EXCENT_OK;
    }
    int32_t* entries(int s) const { return entries_[s]; }
    int32_t* vids(int s) const { return vids_[s]; }
    ull* offsets(int s) const { return off_[s]; }

    // The next slot in rotation, once its previous work is done.
    int claim(int* slot) {
        const int s = next_;
        next_ ^= 1;
        if (in_flight_[s]) {
            const auto w = Clock::now();
            const int rc = excent_engine_slot_wait(e_, s);
            t_.wait += secs(w, Clock::now());
            in_flight_[s] = false;
            EX_TRY(rc);
        }
        *slot = s;
        return EXCENT_OK;
    }
    void all_idle() { in_flight_[0] = in_flight_[1] = false; }

    // A whole chunk read from storage and pushed (src/excent.cu:696-707).
    int stream(int c, const Chunk& ch, const ull* cnt, double list_frac, bool cache_fill, int hlo, int hhi) {
        int s;
        EX_TRY(claim(&s));
        const auto a = Clock::now();
        EX_TRY(g_.fetch_entries(ch.e0, ch.e1, entries_[s]));
        t_.stream_bytes += ch.edges() * sizeof(int32_t);
        t_.io += secs(a, Clock::now());
        EX_TRY(excent_engine_push_stream(e_, s, c, cnt, list_frac, cache_fill ? 1 : 0, hlo, hhi));
        in_flight_[s] = true;
        return EXCENT_OK;
    }

    // The pending lists of [v0, v1) per the bitmap into slot s; returns (k, entries).
    int fill_lists(int s, const int32_t* ids, int k, ull* pages, ull* runs) {
        ull* o = off_[s];
        if (ids != vids_[s]) std::copy(ids, ids + k, vids_[s]);
        o[0] = 0;
        for (int i = 0; i < k; i++) o[i + 1] = o[i] + g_.degree(vids_[s][i]);
        *pages = *runs = 0;
        if (dedup_) g_.readahead_lists(vids_[s], k, pages, runs);
        copy_lists(g_, vids_[s], o, k, entries_[s], g_.io_threads());
        return EXCENT_OK;
    }

    // The pending vertices of a chunk gathered and pushed (src/excent.cu:711-739).
    int gather(const Chunk& ch, const uint32_t* bitmap, ull* pages, ull* runs) {
        int s;
        EX_TRY(claim(&s));
        const auto a = Clock::now();
        const int k = pending_lists(ch.v0, ch.v1, bitmap, g_.offsets(), vids_[s], off_[s]);
        EX_TRY(fill_lists(s, vids_[s], k, pages, runs));
        const ull ne = off_[s][k];
        t_.gather_bytes += ne * sizeof(int32_t) + (ull)k * (sizeof(int32_t) + sizeof(ull));
        t_.io += secs(a, Clock::now());
        EX_TRY(excent_engine_push_gather(e_, s, k, ne));
        in_flight_[s] = true;
        return EXCENT_OK;
    }

private:
    excent_engine* e_;
    const GraphFile& g_;
    Tally& t_;
    bool dedup_;
    int next_ = 0;
    bool in_flight_[2] = {false, false};
    int32_t* entries_[2] = {nullptr, nullptr};
    int32_t* vids_[2] = {nullptr, nullptr};
    ull* off_[2] = {nullptr, nullptr};
};

// ------------------------------------------------------------------ tau

// The crossover is kept per graph and machine in
// $HOME/.cache/excent/<file name>.<n>.<m>.tau as "%.6f %.4f\n" (tau, seconds
// the calibration took), the reference's cache file (src/excent.cu:517-533, 576).
static std::string tau_file_for(const std::string& graph, int n, ull m) {
    const char* home = getenv("HOME");
    const size_t slash = graph.find_last_of('/');
    const std::string name = slash == std::string::npos ? graph : graph.substr(slash + 1);
    std::string dir = std::string(home ? home : ".") + "/.cache";
    mkdir(dir.c_str(), 0755);
    dir += "/excent";
    mkdir(dir.c_str(), 0755);
    return dir + "/" + name + "." + std::to_string(n) + "." + std::to_string(m) + ".tau";
}

// Measure tau on one chunk from a cold page cache: the time to stream it,
// against gathers of its highest-degree lists (ties by id) that cover 5 %,
// 15 % and 40 % of its entries; crossover_tau interpolates between them.
struct TauProbe {
    double t_stream = 0, t_gather[3] = {0, 0, 0}, frac[3] = {0, 0, 0};
};
static int probe_tau(const GraphFile& g, const Chunk& ch, Staging& st, TauProbe& pr) {
    static const double kTargets[3] = {0.05, 0.15, 0.4};
    g.evict(ch.e0, ch.e1, ch.v0, ch.v1);
    auto a = Clock::now();
    EX_TRY(g.fetch_entries(ch.e0, ch.e1, st.entries(0)));
    pr.t_stream = secs(a, Clock::now());
    const int nv = ch.v1 - ch.v0;
    std::vector<int32_t> by_degree(nv);
    std::iota(by_degree.begin(), by_degree.end(), ch.v0);
    std::stable_sort(by_degree.begin(), by_degree.end(),
                     [&](int32_t x, int32_t y) { return g.degree(x) > g.degree(y); });
    std::vector<ull> covered(nv + 1, 0);   // entries of the first i lists in that order
    for (int i = 0; i < nv; i++) covered[i + 1] = covered[i] + g.degree(by_degree[i]);
    for (int j = 0; j < 3; j++) {
        const double want = kTargets[j] * (double)ch.edges();
        int k = 0;   // fewest lists whose entries reach the target
        while (k < nv && (double)covered[k] < want) k++;
        std::vector<int32_t> pick(by_degree.begin(), by_degree.begin() + k);
        std::sort(pick.begin(), pick.end());
        g.evict(ch.e0, ch.e1, ch.v0, ch.v1);
        a = Clock::now();
        ull pages, runs;
        EX_TRY(st.fill_lists(0, pick.data(), k, &pages, &runs));
        pr.t_gather[j] = secs(a, Clock::now());
        pr.frac[j] = ch.edges() ? (double)st.offsets(0)[k] / (double)ch.edges() : 0.0;
    }
    return EXCENT_OK;
}

// ------------------------------------------------------------------ the run

class Run {
public:
    explicit Run(const Options& o) : o_(o) {}
    ~Run() { if (e_) excent_engine_destroy(e_); }

    int main() {
        T0_ = Clock::now();
        if (excent_measures_make(&M_, o_.measure.c_str(), o_.alpha, o_.beta, o_.lambda, o_.eps_pr, o_.eps_katz,
                                 o_.eps_ev) != EXCENT_OK) {
            fprintf(stderr, "%s\n", excent_last_error());
            return 1;
        }
        if (o_.ev_init_fp64) M_.flags |= EXCENT_EV_INIT_FP64;
        if (g_.open(o_.graph.c_str(), 16, /*offsets_in_ram=*/false, true) != EXCENT_OK) {
            fprintf(stderr, "%s\n", excent_last_error());
            return 1;
        }
        if (int rc = open_engine()) return rc;
        if (int rc = size_caches()) return rc;
        if (int rc = fetch_rule()) return rc;
        if (int rc = load_for_device_loop()) return rc;
        RT_CK(excent_engine_sync(e_));
        T_setup_ = Clock::now();
        print_setup();
        const int rc = dev_loop_ ? device_passes() : host_passes();
        if (rc) return rc;
        T_iter_ = Clock::now();
        if (int r = results()) return r;
        return 0;
    }

private:
    const Options& o_;
    excent_measures M_{};
    GraphFile g_;
    std::vector<Chunk> ch_;
    int nc_ = 0;
    ull max_entries_ = 0;
    int max_vertices_ = 0;
    excent_engine* e_ = nullptr;
    excent_device_info_t di_{};
    bool zc_ = false;
    Tally tally_;
    std::unique_ptr<Staging> staging_;
    // caches
    std::string cache_mode_;
    std::vector<uint8_t> resident_, loaded_;
    int n_resident_ = 0;
    ull resident_entries_ = 0;
    bool hot_mode_ = false;
    int nh_ = 0;
    ull hot_entries_ = 0, hot_threshold_ = 0;
    std::vector<int> hlo_, hhi_;
    double tau_ = 2.0;
    bool dev_loop_ = false, host_loop_ = false;
    int passes_ = 0;
    Clock::time_point T0_, T_open_, T_setup_, T_iter_;

    ull usable_free() const {
        ull f = di_.free_bytes;
        if (o_.budget_gb > 0) f = std::min<ull>(f, (ull)(o_.budget_gb * (1ull << 30)));
        return f;
    }
    int refresh_free() {
        if (excent_device_info(o_.device, &di_) != EXCENT_OK) {
            fprintf(stderr, "excent: %s\n", excent_last_error());
            return 1;
        }
        return 0;
    }

    int open_engine() {
        const int n = g_.n;
        const ull m = g_.m;
        const ull cap = chunk_cap(m, o_.chunk_medges, o_.target_chunks, o_.min_chunk_medges);
        ch_ = split_chunks(n, g_.offsets(), cap);
        nc_ = (int)ch_.size();
        for (const Chunk& c : ch_) {
            max_entries_ = std::max(max_entries_, c.edges());
            max_vertices_ = std::max(max_vertices_, c.v1 - c.v0);
        }
        T_open_ = Clock::now();
        printf("graph: n=%d m=%llu chunks=%d (cap %llu, max %llu edges, %d vertices)  open %.2fs\n", n, m, nc_, cap,
               max_entries_, max_vertices_, secs(T0_, T_open_));
        fflush(stdout);
        std::vector<int> cv0(nc_);
        std::vector<ull> ce(nc_ + 1);
        for (int c = 0; c < nc_; c++) { cv0[c] = ch_[c].v0; ce[c] = ch_[c].e0; }
        ce[nc_] = m;
        RT_CK(excent_engine_create(o_.device, n, m, &M_, nc_, cv0.data(), ce.data(), &e_));
        // offsets go up in pieces of 16M entries through one staging vector
        const size_t piece = size_t(1) << 24, total = (size_t)n + 1;
        std::vector<ull> stage(std::min(piece, total));
        for (size_t v0 = 0; v0 < total; v0 += piece) {
            const size_t cnt = std::min(piece, total - v0);
            RT_CK(g_.fetch_offsets(v0, cnt, stage.data()));
            RT_CK(excent_engine_upload_offsets(e_, stage.data(), v0, cnt));
        }
        if (!o_.trace_file.empty()) RT_CK(excent_engine_trace(e_, 1));
        RT_CK(excent_engine_init(e_));
        RT_CK(excent_device_info(o_.device, &di_));
        zc_ = o_.zero_copy == "on" || (o_.zero_copy == "auto" && di_.integrated);
        staging_.reset(new Staging(e_, g_, tally_, o_.dedup));
        RT_CK(staging_->create(max_entries_, max_vertices_, zc_));
        return 0;
    }

    // Chunk prefix in HBM, or the degree cache (src/excent.cu:400-513).
    int size_caches() {
        const ull reserve = (ull)(o_.reserve_mb * (1 << 20));
        const ull m = g_.m;
        cache_mode_ = o_.cache_mode;
        resident_.assign(nc_, 0);
        loaded_.assign(nc_, 0);
        hlo_.assign(nc_, 0);
        hhi_.assign(nc_, 0);
        if (refresh_free()) return 1;
        if (o_.host_cache == "pinned") cache_mode_ = "chunks";   // an HBM chunk prefix, the rest in host memory
        if (cache_mode_ == "auto") {
            const ull room = usable_free();
            const bool whole = room > reserve && m * sizeof(int32_t) <= room - reserve;
            cache_mode_ = whole ? "chunks" : "hot";
            printf("cache: auto -> %s\n", whole ? "chunks (the whole graph fits)" : "high-degree lists");
        }
        if (cache_mode_ == "chunks") {
            if (refresh_free()) return 1;
            n_resident_ = resident_prefix(ch_, usable_free(), reserve);
            // one arena for the prefix; if it does not fit after all, keep fewer chunks
            while (n_resident_ > 0 && excent_engine_reserve_cache(e_, ch_[n_resident_ - 1].e1) != EXCENT_OK)
                n_resident_--;
            for (int c = 0; c < n_resident_; c++) { resident_[c] = 1; resident_entries_ += ch_[c].edges(); }
            if (n_resident_ > 0) {   // shared-memory sums for the top-degree targets of cached pushes
                // fewer slots when each launch covers one chunk: a slot pays only with many adds per flush
                const bool sweeping = o_.chunk_sweep == 1 || (o_.chunk_sweep < 0 && ch_.size() > 1);
                const int k_auto = M_.nm == 1 ? (sweeping ? 2048 : 16384) : 4096;
                const int k = o_.hub_targets < 0 ? std::min(k_auto, g_.n) : o_.hub_targets;
                if (k > 0 && excent_engine_set_hub_targets(e_, k) != EXCENT_OK)   // an optimisation: go on without it
                    fprintf(stderr, "excent: hub targets off (%s)\n", excent_last_error());
            }
        }
        RT_CK(excent_engine_set_hub_order(e_, o_.hub_order));
        RT_CK(excent_engine_set_chunk_sweep(e_, o_.chunk_sweep));
        RT_CK(excent_engine_set_sweep_demand(e_, o_.sweep_demand));
        hot_mode_ = cache_mode_ == "hot";
        if (hot_mode_) return setup_degree_cache(reserve);
        return 0;
    }

    int setup_degree_cache(ull reserve) {
        const int n = g_.n;
        if (refresh_free()) return 1;
        const ull bitmap_bytes = (((ull)n + 31) / 32) * sizeof(uint32_t);
        const ull room = usable_free();
        const ull budget = room > reserve + bitmap_bytes ? room - reserve - bitmap_bytes : 0;
        std::vector<uint16_t> score;
        if (!o_.hot_rank.empty()) {
            score.resize(n);
            FILE* f = fopen(o_.hot_rank.c_str(), "rb");
            const bool ok = f && fread(score.data(), sizeof(uint16_t), n, f) == (size_t)n;
            if (f) fclose(f);
            if (!ok) {
                fprintf(stderr, "--hot-rank: cannot read %d entries from %s\n", n, o_.hot_rank.c_str());
                return 1;
            }
        }
        const HotLists H = select_hot_lists(n, g_.offsets(), budget, score.empty() ? nullptr : score.data(), 16);
        nh_ = (int)H.ids.size();
        hot_entries_ = H.edges();
        hot_threshold_ = H.threshold;
        if (nh_ == 0 || excent_engine_hot_setup(e_, nh_, H.ids.data(), H.off.data(), H.bits.data()) != EXCENT_OK) {
            fprintf(stderr, "degree cache: could not allocate %d lists (%.2f GB); running without a cache\n", nh_,
                    hot_entries_ * 4.0 / 1e9);
            nh_ = 0;
            hot_entries_ = 0;
            return 0;
        }
        for (int c = 0; c < nc_; c++) {   // each chunk's slice of the (ascending) hot ids
            hlo_[c] = (int)(std::lower_bound(H.ids.begin(), H.ids.end(), ch_[c].v0) - H.ids.begin());
            hhi_[c] = (int)(std::lower_bound(H.ids.begin(), H.ids.end(), ch_[c].v1) - H.ids.begin());
        }
        return 0;
    }

    int fetch_rule() {
        tau_ = o_.stream_ratio;
        if (!o_.stream_auto) {
            printf("fetch rule: tau = %.3f (given)\n", tau_);
            return 0;
        }
        const std::string file = tau_file_for(o_.graph, g_.n, g_.m);
        if (!o_.recalibrate) {
            double t = 0, t_calib = 0;
            FILE* f = fopen(file.c_str(), "r");
            const bool got = f && fscanf(f, "%lf %lf", &t, &t_calib) == 2;
            if (f) fclose(f);
            if (got) {
                tau_ = t;
                printf("fetch rule: tau = %.3f (measured earlier on this machine in %.2fs, %s)\n", tau_, t_calib,
                       file.c_str());
                return 0;
            }
        }
        const auto c0 = Clock::now();
        TauProbe pr;
        RT_CK(probe_tau(g_, ch_[nc_ / 2], *staging_, pr));
        tau_ = crossover_tau(pr.t_stream, pr.t_gather, pr.frac);
        const double t_calib = secs(c0, Clock::now());
        printf("fetch rule: tau = %.3f (stream %.3fs; gather %.3fs / %.3fs / %.3fs at demand %.3f / %.3f / %.3f)  "
               "calibrate %.2fs\n", tau_, pr.t_stream, pr.t_gather[0], pr.t_gather[1], pr.t_gather[2], pr.frac[0],
               pr.frac[1], pr.frac[2], t_calib);
        if (FILE* f = fopen(file.c_str(), "w")) { fprintf(f, "%.6f %.4f\n", tau_, t_calib); fclose(f); }
        return 0;
    }

    // --device-loop on a fully cached graph: load every chunk now and run the
    // on-device pass loop. --host-cache pinned: the chunks past the HBM prefix
    // go once into pinned host memory, which the device loop reads in place.
    int load_for_device_loop() {
        host_loop_ = o_.host_cache == "pinned" && !hot_mode_;
        dev_loop_ = (o_.device_loop && cache_mode_ == "chunks" && n_resident_ == nc_ && !hot_mode_) || host_loop_;
        if (!dev_loop_) return 0;
        const auto t0 = Clock::now();
        for (int c = 0; c < n_resident_; c++) {
            RT_CK(g_.fetch_entries(ch_[c].e0, ch_[c].e1, staging_->entries(0)));
            RT_CK(excent_engine_load_cache(e_, ch_[c].e0, ch_[c].e1, staging_->entries(0)));
            loaded_[c] = 1;
        }
        if (host_loop_) {
            const auto t1 = Clock::now();
            ull first = 0;
            double t_read = 0;
            RT_CK(fill_host_cache(&first, &t_read));
            printf("host cache: pinned, %.2f GB (%d chunks past the GPU cache), lists read in place over the host link "
                   "(GPU cache load %.2fs, read %.2fs, pinning %.2fs past the read)\n",
                   (g_.m - first) * 4.0 / 1e9, nc_ - n_resident_, secs(t0, t1), t_read,
                   secs(t1, Clock::now()) - t_read);
        }
        return 0;
    }

    // The entries past the GPU cache into host memory, read in 1 GiB pieces by
    // the reader team; a second thread pins each piece once it is read while
    // the next one is read (or the whole range after the read, on a device that
    // cannot address pinned memory by its host address).
    int fill_host_cache(ull* first, double* t_read) {
        int32_t* h = nullptr;
        int pieces_ok = 0;
        RT_CK(excent_engine_host_cache_begin(e_, &h, first, &pieces_ok));
        const ull cnt = g_.m - *first;
        if (!h || cnt == 0) return 0;
        const ull piece = 1ull << 28;
        std::atomic<ull> filled{0};
        std::atomic<int> stop{0};
        std::string pin_error;
        std::thread pinner;
        if (pieces_ok)
            pinner = std::thread([&] {
                ull done = 0;
                while (done < cnt && !stop.load()) {
                    const ull f = filled.load();
                    if (f == done) { std::this_thread::sleep_for(std::chrono::milliseconds(2)); continue; }
                    if (excent_engine_host_cache_pin(e_, f) != EXCENT_OK) { pin_error = excent_last_error(); break; }
                    done = f;
                }
            });
        const auto r0 = Clock::now();
        int rc = EXCENT_OK;
        for (ull at = 0; at < cnt && rc == EXCENT_OK && pin_error.empty(); at += piece) {
            const ull to = std::min(cnt, at + piece);
            rc = g_.fetch_entries(*first + at, *first + to, h + at);
            if (rc == EXCENT_OK) filled.store(to);
        }
        *t_read = secs(r0, Clock::now());
        if (rc != EXCENT_OK) stop.store(1);
        if (pinner.joinable()) pinner.join();
        RT_CK(rc);
        if (!pin_error.empty()) { fprintf(stderr, "excent: %s\n", pin_error.c_str()); return 1; }
        if (!pieces_ok) RT_CK(excent_engine_host_cache_pin(e_, cnt));
        return 0;
    }

    void print_setup() {
        const ull m = g_.m;
        printf("staging: %s\n", zc_ ? "zero copy (pinned, GPU-mapped buffers read in place)"
                                    : "pinned host buffers copied to the GPU");
        if (hot_mode_ && !o_.hot_rank.empty())
            printf("GPU cache ranked by passes pending (%s): %d vertices (%.1f%% of edges, %.2f GB)  setup %.2fs\n",
                   o_.hot_rank.c_str(), nh_, 100.0 * hot_entries_ / m, hot_entries_ * 4.0 / 1e9, secs(T_open_, T_setup_));
        else if (hot_mode_)
            printf("GPU degree cache: %d vertices with degree >= %llu (%.1f%% of edges, %.2f GB)  setup %.2fs\n", nh_,
                   hot_threshold_, 100.0 * hot_entries_ / m, hot_entries_ * 4.0 / 1e9, secs(T_open_, T_setup_));
        else
            printf("GPU edge cache: %d/%d chunks resident (%.1f%% of edges)  setup %.2fs\n", n_resident_, nc_,
                   100.0 * resident_entries_ / m, secs(T_open_, T_setup_));
        fflush(stdout);
    }

    static void pass_line(int pass, ull pending, double demand_ratio, int nres, int nstream, int ngather, ull hotpend,
                          long maj, long min, ull pages, ull runs) {
        printf("pass %3d: pending %llu v, demand ratio %.4f | resident %d stream %d gather %d | cached high-degree "
               "pending %llu | faults major %ld minor %ld | gather pages %llu runs %llu\n",
               pass, pending, demand_ratio, nres, nstream, ngather, hotpend, maj, min, pages, runs);
    }

    int device_passes() {
        const auto a = Clock::now();
        RT_CK(excent_engine_solve(e_, o_.list_frac, o_.max_passes, 1));
        excent_stats st;
        std::vector<excent_pass_log> log(std::min(o_.max_passes, 1 << 17) + 1);
        RT_CK(excent_engine_stats(e_, &st, log.data(), (int)log.size()));
        passes_ = st.passes;
        if (host_loop_) {   // the lists read in place are this mode's gathered bytes
            ull over_link = 0;
            RT_CK(excent_engine_host_pushed(e_, &over_link));
            tally_.gather_bytes += over_link * 4;
        }
        for (int p = 0; p < passes_ && p < (int)log.size(); p++)
            pass_line(p, log[p].pending, (double)log[p].demand / g_.m, log[p].n_list + log[p].n_range, 0, 0, 0, 0, 0,
                      0, 0);
        tally_.wait += secs(a, Clock::now());
        return 0;
    }

    // The degree cache's pending lists, per range of hot ids: either one range
    // over all of them (--hot-order sweep) or one per chunk (ranges).
    int push_hot(bool after_slots) {
        if (o_.hot_order == "ranges") {
            for (int c = 0; c < nc_; c++)
                if (hhi_[c] > hlo_[c]) EX_TRY(excent_engine_push_hot(e_, hlo_[c], hhi_[c], after_slots ? 1 : 0));
        } else if (nh_) {
            EX_TRY(excent_engine_push_hot(e_, 0, nh_, after_slots ? 1 : 0));
        }
        return EXCENT_OK;
    }

    // The reference's pass (src/excent.cu:656-760): snapshot and plan; the
    // degree cache before (--hot-when start|both); every cached chunk in one
    // launch; the streamed and gathered chunks through the slots; the degree
    // cache after the slots (end|both); then wait for the GPU.
    int host_passes() {
        std::vector<ull> cnt(2 * (size_t)nc_);
        std::vector<uint32_t> bitmap(((size_t)g_.n + 31) / 32);
        PassPlan plan;
        for (passes_ = 0; passes_ < o_.max_passes; passes_++) {
            const int pass = passes_;
            const auto t0 = Clock::now();
            const auto f0 = fault_counts();
            const bool hot_skip = hot_mode_ && nh_ > 0 && pass > 0;
            ull hotpend = 0;
            RT_CK(excent_engine_snapshot(e_, hot_skip ? 1 : 0, cnt.data(), &hotpend, nullptr));
            plan_pass(ch_, cnt.data(), resident_, loaded_, tau_, hot_mode_, pass, hlo_, hhi_, plan);
            if (plan.need_bitmap) RT_CK(excent_engine_bitmap(e_, bitmap.data()));
            tally_.snap += secs(t0, Clock::now());
            if (plan.pending == 0 && hotpend == 0) break;

            int counts[4] = {0, 0, 0, 0};
            for (uint8_t md : plan.mode) counts[md]++;
            if (hot_skip && hotpend && o_.hot_when != "end") RT_CK(push_hot(false));
            if (counts[FETCH_CACHED]) RT_CK(excent_engine_push_cached(e_, plan.mode.data(), cnt.data(), o_.list_frac));
            ull pages = 0, runs = 0;
            for (int c = 0; c < nc_; c++) {
                if (plan.mode[c] == FETCH_STREAM) {
                    const bool fill_hot = hot_mode_ && pass == 0 && hhi_[c] > hlo_[c] && nh_ > 0;
                    RT_CK(staging_->stream(c, ch_[c], cnt.data(), o_.list_frac, resident_[c] != 0,
                                           fill_hot ? hlo_[c] : 0, fill_hot ? hhi_[c] : 0));
                    if (resident_[c]) loaded_[c] = 1;
                } else if (plan.mode[c] == FETCH_GATHER) {
                    ull pg = 0, rn = 0;
                    RT_CK(staging_->gather(ch_[c], bitmap.data(), &pg, &rn));
                    pages += pg;
                    runs += rn;
                }
            }
            if (hot_skip && o_.hot_when != "start") RT_CK(push_hot(true));
            const auto w0 = Clock::now();
            RT_CK(excent_engine_sync(e_));
            staging_->all_idle();
            tally_.wait += secs(w0, Clock::now());
            const auto f1 = fault_counts();
            tally_.major += f1.first - f0.first;
            tally_.minor += f1.second - f0.second;
            tally_.pages += pages;
            tally_.runs += runs;
            pass_line(pass, plan.pending, (double)plan.demand / g_.m, counts[FETCH_CACHED], counts[FETCH_STREAM],
                      counts[FETCH_GATHER], hotpend, f1.first - f0.first, f1.second - f0.second, pages, runs);
        }
        return 0;
    }

    int write_floats(const std::string& path, const void* data, size_t bytes) {
        FILE* f = fopen(path.c_str(), "wb");
        const bool ok = f && fwrite(data, 1, bytes, f) == bytes;
        if (f) fclose(f);
        if (!ok) fprintf(stderr, "cannot write %s\n", path.c_str());
        return ok ? 0 : 1;
    }

    int results() {
        const int n = g_.n;
        const ull m = g_.m;
        std::vector<double> sum(M_.nm, 0.0);
        std::vector<float> vals(n);
        for (int i = 0; i < M_.nm; i++) {
            RT_CK(excent_engine_read(e_, i, 0, vals.data(), 0, n));
            sum[i] = std::accumulate(vals.begin(), vals.end(), 0.0);
            if (!o_.dump.empty() &&
                write_floats(o_.dump + "." + MNAME[M_.kind[i]] + ".bin", vals.data(), (size_t)n * sizeof(float)))
                return 1;
        }
        if (!o_.trace_file.empty()) {
            std::vector<uint16_t> tr(n);
            RT_CK(excent_engine_read_trace(e_, tr.data()));
            if (write_floats(o_.trace_file, tr.data(), (size_t)n * sizeof(uint16_t))) return 1;
        }
        const auto T_end = Clock::now();
        excent_stats st;
        RT_CK(excent_engine_stats(e_, &st, nullptr, 0));
        printf("passes %d  measure %s (n=%d):", passes_, o_.measure.c_str(), n);
        for (int i = 0; i < M_.nm; i++) printf("  %s sum %.6e", MNAME[M_.kind[i]], sum[i]);
        printf("\n");
        if (o_.count_pushes) printf("edges pushed: %.2f x |E|\n", m ? (double)st.pushed / m : 0.0);
        printf("launches from GPU memory: %llu pending-only, %llu whole-range\n", st.n_list, st.n_range);
        printf("bytes shipped: stream %.2f GB, gather %.2f GB (graph edges %.2f GB)\n", tally_.stream_bytes / 1e9,
               tally_.gather_bytes / 1e9, m * 4.0 / 1e9);
        printf("page faults in passes: major %ld, minor %ld | gather dedup %s: %llu pages in %llu runs\n",
               tally_.major, tally_.minor, o_.dedup ? "on" : "off", tally_.pages, tally_.runs);
        printf("time: open %.2fs setup %.2fs passes %.2fs [cpu io %.2fs, gpu wait %.2fs, snapshot %.2fs] result %.2fs | "
               "internal total %.2fs\n", secs(T0_, T_open_), secs(T_open_, T_setup_), secs(T_setup_, T_iter_),
               tally_.io, tally_.wait, tally_.snap, secs(T_iter_, T_end), secs(T0_, T_end));
        const double tp = secs(T_setup_, T_iter_);
        printf("throughput: %.3f GTEPS (%llu adjacency entries pushed in %.3fs of passes); residual sum (FP64):",
               tp > 0 ? st.pushed / tp / 1e9 : 0.0, st.pushed, tp);
        for (int i = 0; i < M_.nm; i++) printf(" %s %.6e", MNAME[M_.kind[i]], st.rsum[i]);
        printf("\n");
        return 0;
    }
};

}  // namespace excent

extern "C" int excent_cli_main(int argc, char** argv) {
    excent::Options o;
    if (excent::parse_options(argc, argv, o)) return 1;
    excent::Run r(o);
    return r.main();
}
