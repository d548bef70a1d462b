/*
 * excent_b200.h -- C ABI of libexcent_b200.so, the B200 (sm_100a) engine for
 * ExCent's asynchronous delta-push centrality path (PageRank, Katz,
 * eigenvector, and the single-stream `all` pass).
 *
 * Plain C types only: pointers, sizes, status codes. Every call returns an
 * EXCENT_* status; on failure excent_last_error() holds a message (thread
 * local). Nothing here exits the process.
 *
 * The reference (SPADE-IITJ/ExCent) is a monolithic CLI whose kernels are
 * launched directly from main(); its internal seam is the Measures table
 * passed by value to every kernel (src/excent.cu:29-37) and the launches at
 * src/excent.cu:663 (snapshot), :642-649 (compact + push of a chunk in GPU
 * memory), :738 (push of a gathered list), :618-624 (hot cache) and :705 (hot
 * fill). Each entry point below names the reference code it replaces.
 * Reference paths are relative to the reference project.
 */
#ifndef EXCENT_B200_H
#define EXCENT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define EXCENT_OK 0
#define EXCENT_ERR_ARG 1     /* bad argument (message says which) */
#define EXCENT_ERR_CUDA 2    /* a CUDA runtime call failed */
#define EXCENT_ERR_IO 3      /* open / read / short read / bad file */
#define EXCENT_ERR_NOMEM 4   /* a device or pinned allocation failed */
#define EXCENT_ERR_STATE 5   /* call out of order (e.g. no graph uploaded) */
#define EXCENT_ERR_TIMEOUT 6 /* a bounded device wait gave up */

/* measure kinds, as src/excent.cu:22 numbers them */
#define EXCENT_PR 0
#define EXCENT_KATZ 1
#define EXCENT_EV 2

/* Message of the last failed call on this thread ("" if none). */
const char* excent_last_error(void);
/* Library ABI version (major * 100 + minor). */
int excent_version(void);

/* ------------------------------------------------------------ measures */

/* The per-run measure table: replaces struct Measures (src/excent.cu:29-37)
 * together with the init constants of k_init (:41-47). Vectors are per
 * measure, in run order. */
typedef struct excent_measures {
    int nm;            /* number of measures, 1..3 */
    int kind[3];       /* EXCENT_PR / EXCENT_KATZ / EXCENT_EV */
    float eps[3];      /* pending iff |r| > eps */
    float scale[3];    /* push weight numerator: d, alpha, or 1/lambda */
    int divdeg[3];     /* 1: weight = scale / deg(v) (PageRank) */
    double beta;       /* Katz initial residual */
    double lambda;     /* eigenvector initial residual deg/lambda - 1 */
    int flags;         /* EXCENT_EV_INIT_FP64 */
} excent_measures;

/* excent_measures.flags: compute the eigenvector's initial residual
 * deg/lambda1 - 1 with the FP64 lambda1. The reference rounds lambda1 to
 * float first (src/excent.cu:41, 372); that rounding leaves a component along
 * the principal eigenvector in the initial residual which the push (whose
 * operator has eigenvalue ~1 there) never removes, so on graphs with a large
 * (v1 . 1) the hub residuals can stay above a small eps for good. */
#define EXCENT_EV_INIT_FP64 1

/* Build the table for --measure pr|katz|ev|all with the reference's
 * validation and float rounding (src/excent.cu:307-316, 344-351). Negative
 * alpha / lambda / eps mean "not given". */
int excent_measures_make(excent_measures* out, const char* measure, double alpha, double beta, double lambda,
                         double eps_pr, double eps_katz, double eps_ev);

/* ------------------------------------------------------------ device engine */

typedef struct excent_engine excent_engine;

/* Create an engine on `device` for a graph of n vertices and m edges split
 * into nc chunks whose first vertices are chunk_v0[0..nc) and edge bounds
 * chunk_e[0..nc] (host arrays). Allocates the per-vertex state (values,
 * residuals, offsets, bitmap, pending lists, demand table). Replaces the
 * allocations of src/excent.cu:335-369. */
int excent_engine_create(int device, int n, unsigned long long m, const excent_measures* measures, int nc,
                         const int* chunk_v0, const unsigned long long* chunk_e, excent_engine** out);
int excent_engine_destroy(excent_engine* e);

/* Copy offsets idx[v0 .. v0+count) from host memory (pageable or pinned);
 * replaces the upload loop of src/excent.cu:360-369. */
int excent_engine_upload_offsets(excent_engine* e, const unsigned long long* idx, unsigned long long v0,
                                 unsigned long long count);

/* Copy a whole graph that is already in device memory (idx[n+1], adj[m]
 * device pointers, e.g. from excent_rmat_generate) into the engine: offsets
 * and a full edge cache, every chunk marked loaded. */
int excent_engine_upload_device(excent_engine* e, const unsigned long long* d_idx, const int32_t* d_adj);

/* Reserve the HBM edge cache for the first `edges` edges of the graph (the
 * resident chunk prefix); replaces the per-chunk cudaMalloc loop of
 * src/excent.cu:410-421. Returns EXCENT_ERR_NOMEM (and leaves no cache) if the
 * allocation fails. */
int excent_engine_reserve_cache(excent_engine* e, unsigned long long edges);
/* Copy edges [e0, e1) from host memory into the edge cache and mark the
 * chunks fully inside it as loaded. */
int excent_engine_load_cache(excent_engine* e, unsigned long long e0, unsigned long long e1, const int32_t* edges);
/* Mark chunk c as loaded (its edges were copied by a streamed push with
 * cache fill); src/excent.cu:707. */
int excent_engine_set_loaded(excent_engine* e, int c, int loaded);

/* k_init for every measure (src/excent.cu:370-372) and reset of the pass state. */
int excent_engine_init(excent_engine* e);

/* One demand snapshot (src/excent.cu:660-665): zero the demand table, launch
 * the snapshot kernel and copy back cnt[2*nc] (interleaved pending count and
 * pending degree sum per chunk), the hot pending count and the FP64 sum of
 * |r| per measure. use_hot: skip cached high-degree vertices (pass > 0 in hot
 * mode, src/excent.cu:662). Any output pointer may be NULL. */
int excent_engine_snapshot(excent_engine* e, int use_hot, unsigned long long* cnt, unsigned long long* hotpend,
                           double* rsum);
/* Copy the pending bitmap (ceil(n/32) words) to the host (src/excent.cu:678). */
int excent_engine_bitmap(excent_engine* e, uint32_t* words);
/* Copy the snapshot's pending list of chunk c (unordered) and its length. */
int excent_engine_chunk_list(excent_engine* e, int c, int32_t* ids, unsigned int* k);

/* Push every chunk whose mode[c] == 1 from the HBM edge cache in one launch,
 * each as its pending list when cnt < list_frac * chunk vertices, else as
 * its whole vertex range with the push-time re-check. Replaces the resident
 * loop and launch_chunk (src/excent.cu:629-652, 684-688). mode and cnt are
 * host arrays (cnt as returned by the last snapshot). */
int excent_engine_push_cached(excent_engine* e, const unsigned char* mode, const unsigned long long* cnt,
                              double list_frac);

/* Pinned double-buffered staging (src/excent.cu:224-233, 374-390). Two slots,
 * each with host buffers for edges (max_chunk_edges), vertex ids and offsets
 * (max_chunk_verts), device mirrors, a stream and an event. zero_copy maps
 * the host buffers into the device address space instead (:376-379). */
int excent_engine_slots_create(excent_engine* e, unsigned long long max_chunk_edges, int max_chunk_verts,
                               int zero_copy);
/* Host pointers of slot s (0 or 1) for the planner to fill. */
int excent_engine_slot_buffers(excent_engine* e, int s, int32_t** edges, int32_t** vids, unsigned long long** off);
/* Wait until slot s's previous work finished (src/excent.cu:599-601). */
int excent_engine_slot_wait(excent_engine* e, int s);
/* Streamed chunk c staged in slot s: copy its edges to the device (into the
 * edge cache when cache_fill and the chunk is resident), optionally fill the
 * hot cache lists of hot ids [hlo, hhi) from it (k_fill_hot, :704-705), then
 * push it as list or range (launch_chunk). Asynchronous on the slot stream.
 * src/excent.cu:696-707. */
int excent_engine_push_stream(excent_engine* e, int s, int c, const unsigned long long* cnt, double list_frac,
                              int cache_fill, int hlo, int hhi);
/* Gathered lists in slot s: k vertex ids, k+1 offsets, ne edges; copy and
 * push (src/excent.cu:732-739). Asynchronous on the slot stream. */
int excent_engine_push_gather(excent_engine* e, int s, int k, unsigned long long ne);

/* Degree (hot) cache of nh high-degree vertices: ids ascending, list offsets
 * off[nh+1], and the hot bitmap (ceil(n/32) words). Returns EXCENT_ERR_NOMEM
 * and leaves no cache when it does not fit (src/excent.cu:492-503). */
int excent_engine_hot_setup(excent_engine* e, int nh, const int32_t* ids, const unsigned long long* off,
                            const uint32_t* hot_bitmap);
/* Push the pending hot vertices among hot ids [lo, hi) from the hot cache,
 * after the slots' outstanding work (src/excent.cu:615-628, 745-748). The
 * pending count stays on the device: no host synchronisation per range. */
int excent_engine_push_hot(excent_engine* e, int lo, int hi, int after_slots);

/* The pending hot vertices among hot ids [lo, hi) on the current residuals,
 * as indices into the hot id list (unordered), and their count: the
 * compaction step of excent_engine_push_hot alone, synchronous
 * (src/excent.cu:178-182, 617-618). */
int excent_engine_hot_pending(excent_engine* e, int lo, int hi, int32_t* out, unsigned int* k);
/* Copy the hot cache's edge lists (off[nh] entries) to the host, after the
 * pass-0 fills of excent_engine_push_stream (src/excent.cu:211-220, 704-705). */
int excent_engine_hot_edges(excent_engine* e, int32_t* out);

/* Wait for all engine streams. */
int excent_engine_sync(excent_engine* e);

/* Device solve of a fully cached graph (every chunk resident and loaded):
 * init, then passes of snapshot -> on-device fetch plan -> push until no
 * vertex is pending or max_passes, with no host round trip per pass. With
 * use_graph the pass is one CUDA graph with a conditional while node.
 * Per-pass log and totals are kept for excent_engine_stats. */
int excent_engine_solve(excent_engine* e, double list_frac, int max_passes, int use_graph);

/* Same as excent_engine_solve but from the current values and residuals
 * (no k_init): for seeded or restarted solves. */
int excent_engine_resume(excent_engine* e, double list_frac, int max_passes, int use_graph);
/* Single-measure engines: zero values and residuals, then add vals[i] to the
 * residual of vids[i] (a personalized start, e.g. (1-d)/|S| on a seed set S
 * for personalized PageRank). Follow with excent_engine_resume. */
int excent_engine_seed(excent_engine* e, int k, const int32_t* vids, const float* vals);

typedef struct excent_pass_log {
    unsigned long long pending;   /* pending vertices at the snapshot */
    unsigned long long demand;    /* their total degree */
    unsigned long long hot_pending;
    unsigned long long pushed;    /* adjacency entries pushed in the pass */
    double rsum[3];               /* FP64 sum of |r| per measure at the snapshot */
    int n_list, n_range;          /* chunks pushed as lists / whole ranges */
    unsigned long long lanes;     /* entries pushed x measures with a nonzero weight (== pushed for one measure) */
    unsigned long long taken;     /* measures taken over the pushed vertices (== pushed vertices for one measure) */
} excent_pass_log;

typedef struct excent_stats {
    int passes;                   /* passes that pushed (the reference's "passes") */
    unsigned long long pushed;    /* adjacency entries pushed in total */
    unsigned long long n_list, n_range;
    double rsum[3];               /* final FP64 sum of |r| per measure */
} excent_stats;

/* Totals of the last solve, and up to cap pass records. */
int excent_engine_stats(excent_engine* e, excent_stats* st, excent_pass_log* log, int cap);

/* Copy values x (or residuals r) of measure i (run order) for vertices
 * [v0, v0+count) to the host as float32 (src/excent.cu:763-777). */
int excent_engine_read(excent_engine* e, int i, int residual, float* out, unsigned long long v0,
                       unsigned long long count);
/* Overwrite values and residuals of measure i from host float32 arrays of n
 * entries (either may be NULL to keep it). Test hook. */
int excent_engine_write(excent_engine* e, int i, const float* x, const float* r);

/* --trace-pending: a uint16 counter per vertex of the passes in which it was
 * pending (src/excent.cu:76, 606-607, 779-789). enable before init. */
int excent_engine_trace(excent_engine* e, int enable);
int excent_engine_read_trace(excent_engine* e, uint16_t* out);

/* Hub-target aggregation: re-encode the entries of the k highest-degree
 * vertices in the HBM edge cache as slots, so push kernels sum the
 * contributions to those targets in shared memory and add them to the
 * residuals once per block instead of once per entry (the hubs of a power-law
 * graph receive a large share of all entries, and same-address reductions
 * serialise in L2). k <= 32768 (one measure) or 8192 (float4 layout); 0 turns
 * it off and restores plain ids. Call after the cache is reserved: chunks
 * loaded so far are rewritten now, later loads (load_cache, upload_device,
 * cache-filling streamed pushes) as they land; reserving the cache again
 * turns it off. No reference counterpart. */
int excent_engine_set_hub_targets(excent_engine* e, int k);

/* Order of the high-degree lists (more than 256 entries) in each pass of the
 * device solve, of a host-driven cached push and inside each streamed or
 * gathered chunk: 1 first, so the large share
 * of a pass's residual they carry reaches the other vertices before those are
 * taken; 2 last, after every other pending vertex; 0 in table order with the
 * rest; 3 first inside each push launch (each chunk's own long lists before
 * its other lists, no graph-wide list); -1 (the default) 3 when the chunks are
 * swept one by one, else 1. */
int excent_engine_set_hub_order(excent_engine* e, int order);
/* Cached pushes chunk by chunk (1: one launch per chunk, each after the
 * previous one, as the reference launches its resident chunks on one stream,
 * src/excent.cu:684-688), every chunk in one launch (0), or -1 (the default):
 * chunk by chunk when the graph has more than one chunk. */
int excent_engine_set_chunk_sweep(excent_engine* e, int on);
/* A sweeping engine (excent_engine_set_chunk_sweep) pushes a pass chunk by
 * chunk only while the pass's pending entries (the sum of the pending
 * vertices' degrees) reach frac * m; a pass below that is pushed in one
 * launch, whose per-chunk launches would cost more than the ordering saves.
 * 0 sweeps every pass. Applies to the device solve and to cached pushes. */
int excent_engine_set_sweep_demand(excent_engine* e, double frac);
/* Tiles of 32 items a push warp claims at a time (1..1024), or 0 (the
 * default): up to 32, at least four claims per warp. Fewer tiles per claim
 * keep the items in flight closer together in table order. */
int excent_engine_set_claim_tiles(excent_engine* e, int tiles);
/* The scatter's ceiling on this graph: one reduction per edge-cache entry (in
 * cache order, to its target, into a scratch array shaped like the residuals),
 * best of three timed passes, as entries per second. Needs the whole graph in
 * the edge cache. No counterpart in the reference. */
int excent_engine_scatter_peak(excent_engine* e, double* entries_per_second);
/* Settings of the device solve tried by excent_engine_autotune. */
typedef struct excent_tune {
    int hub_targets;   /* shared-memory slots for the highest-degree targets */
    int hub_order;     /* 0 table order, 1 high-degree lists first, 2 last */
    int chunk_sweep;   /* 1: one launch per chunk, in chunk order */
    double ms;         /* one solve (graph launch) with these settings */
    double sweep_demand; /* with chunk_sweep: sweep passes whose pending entries reach this * m */
} excent_tune;
/* Time one device solve for each candidate and keep the fastest: chunk by
 * chunk, each launch's long lists first (sweep demand 0.25, 0.5 or 1.0 of m;
 * 2048 or the one-launch count of hub-target slots) or in table order, or the
 * graph's high-degree lists first in one launch (0 or two sizes of slots). tried (cap entries, may
 * be NULL) receives every candidate's time. Needs the whole graph in the edge
 * cache. No counterpart in the reference. */
int excent_engine_autotune(excent_engine* e, double list_frac, int max_passes, excent_tune* best,
                           excent_tune* tried, int cap, int* ntried);

/* Host cache for graphs larger than device memory: pinned, device-mapped host
 * memory for the entries past the HBM edge cache (entries [*first_edge, m),
 * *first_edge = the reserved cache size). The caller fills it (e.g. with
 * excent_egr_read_edges) before the next excent_engine_solve, whose push
 * kernels then read those lists in place over the host link (zero copy):
 * only the lists of pending vertices cross it, with no host-side gather or
 * staging copy. Reserving the edge cache again frees it. */
int excent_engine_host_cache(excent_engine* e, int32_t** host_edges, unsigned long long* first_edge);
/* The same host cache, pinned in pieces as the caller fills it: _begin maps
 * it in pageable memory (nothing pinned, nothing zero-filled ahead of the
 * reads); _pin(upto) pins its entries [0, upto) past what is pinned already,
 * so a reader can pin each filled piece while it reads the next. The last
 * call (upto = m - *first_edge) makes it usable by the solve. *pieces_ok = 0:
 * the device cannot address registered memory by its host address, so the
 * whole range must be pinned in that one last call. */
int excent_engine_host_cache_begin(excent_engine* e, int32_t** host_edges, unsigned long long* first_edge,
                                   int* pieces_ok);
int excent_engine_host_cache_pin(excent_engine* e, unsigned long long upto);
/* Entries pushed from the host cache since the last init (4 bytes each crossed the link). */
int excent_engine_host_pushed(excent_engine* e, unsigned long long* entries);

/* FP64 eigenvector normalisation step: with the unit principal eigenvector
 * v1 (n floats, host or device pointer; NULL turns it off), every snapshot
 * removes from the eigenvector residual its v1 component, measured in FP64
 * by the previous snapshot. The push maps that component to itself
 * (eigenvalue lambda1 * float(1/lambda1) ~ 1), so FP32 rounding noise that
 * lands on it is never pushed away and can keep hub residuals above a small
 * eps; removing it changes the result only along v1, i.e. not the unit
 * eigenvector the measure is compared as. No reference counterpart. */
int excent_engine_ev_project(excent_engine* e, const float* d_v1);

/* The engine's main CUDA stream (cudaStream_t), for callers that time
 * its work with their own events. */
int excent_engine_stream(excent_engine* e, void** stream);
/* Per-kernel timing of the device solve run without a graph (use_graph=0):
 * events around the snapshot, plan, push and hub kernels of every pushing
 * pass. profile_read returns the summed milliseconds {snapshot, plan, push,
 * hub} and the pass count since profiling was enabled. */
int excent_engine_profile(excent_engine* e, int enable);
int excent_engine_profile_read(excent_engine* e, double* ms, unsigned long long* passes);

/* Number of device kernel launches this engine issued so far. */
int excent_engine_launches(excent_engine* e, unsigned long long* launches);

/* Free / total device memory, integrated flag, SM count and compute
 * capability of `device` (the reference queries these at src/excent.cu:370,
 * 375, 404). */
typedef struct excent_device_info_t {
    unsigned long long free_bytes, total_bytes;
    int integrated, sms, cc_major, cc_minor;
} excent_device_info_t;
int excent_device_info(int device, excent_device_info_t* out);

/* ------------------------------------------------------------ EGR files */

/* A storage-resident EGR graph (README.md:136-146): the header is parsed
 * (int32 offsets, or int64 when the edge count is -1), the file is mapped,
 * offsets are validated (monotone, spanning [0, m]) and kept mapped or in
 * RAM. A truncated file, a bad header or failed reads return
 * EXCENT_ERR_IO instead of exiting. Replaces StaticGraph
 * (include/StaticGraph.h:29-68). */
typedef struct excent_egr excent_egr;
int excent_egr_open(const char* path, int io_threads, int offsets_in_ram, excent_egr** out);
int excent_egr_close(excent_egr* g);
int excent_egr_info(excent_egr* g, int* n, unsigned long long* m, int* wide);
/* Offsets idx[v0 .. v0+count) as uint64 (include/StaticGraph.h:81-84). */
int excent_egr_read_offsets(excent_egr* g, unsigned long long v0, unsigned long long count, unsigned long long* dst);
/* Edges [e0, e1) by parallel pread in 8 MiB pieces (include/StaticGraph.h:86-88, 160-170). */
int excent_egr_read_edges(excent_egr* g, unsigned long long e0, unsigned long long e1, int32_t* dst);
/* Page-deduplicated readahead of k adjacency lists; returns the pages and
 * runs requested (include/StaticGraph.h:90-114). */
int excent_egr_prefetch(excent_egr* g, const int32_t* vids, int k, unsigned long long* pages, unsigned long long* runs);
/* Evict a chunk's edges and offsets from the page cache (include/StaticGraph.h:116-126). */
int excent_egr_drop_cache(excent_egr* g, unsigned long long e0, unsigned long long e1, unsigned long long v0,
                          unsigned long long v1);

/* ------------------------------------------------------------ host planner */

/* Chunk edge cap: chunk_medges * 1e6 if > 0, else clamp(ceil(m / target_chunks),
 * min_chunk_medges * 1e6, 64e6) (src/excent.cu:321-326). */
unsigned long long excent_chunk_cap(unsigned long long m, double chunk_medges, double target_chunks,
                                    double min_chunk_medges);
/* Greedy contiguous chunks of <= cap edges, >= 1 vertex each; out gets 4
 * entries {v0, v1, e0, e1} per chunk (NULL: count only)
 * (include/StaticGraph.h:128-139). */
int excent_plan_chunks(int n, const unsigned long long* off, unsigned long long cap, int* nc,
                       unsigned long long* out, int out_cap);
/* Leading chunks that fit in free - reserve bytes (src/excent.cu:410-421). */
int excent_cache_chunks(int nc, const unsigned long long* chunk_edges, unsigned long long free_bytes,
                        unsigned long long reserve, int* resident);
/* Degree cache selection under a byte budget, by degree threshold or by a
 * uint16 score per vertex (--hot-rank); ids ascending, offsets nh+1, bitmap
 * ceil(n/32) words (src/excent.cu:428-491). Output arrays may be NULL to
 * count only (size them with n, n+1 and ceil(n/32)). */
int excent_hot_select(int n, const unsigned long long* off, unsigned long long budget, const uint16_t* score, int* nh,
                      int32_t* ids, unsigned long long* hoff, uint32_t* bits, unsigned long long* threshold);
/* Per-chunk mode 0 skip, 1 resident, 2 stream, 3 gather, with the pending
 * and demand totals and whether the bitmap is needed (src/excent.cu:666-678). */
int excent_fetch_plan(int nc, const unsigned long long* chunk_edges, const unsigned long long* cnt,
                      const uint8_t* resident, const uint8_t* loaded, double stream_ratio, int hot_mode, int pass,
                      const int* hlo, const int* hhi, uint8_t* mode, unsigned long long* pend_v,
                      unsigned long long* demand, int* need_bitmap);
/* Ascending pending ids of [v0, v1) from the bitmap and the prefix sums of
 * their degrees (src/excent.cu:711-723). */
int excent_gather_list(int v0, int v1, const uint32_t* bitmap, const unsigned long long* idx, int32_t* vids,
                       unsigned long long* off, int* k);
/* Stream/gather crossover tau from one stream time and three gather times at
 * demand fractions f[3], clamped to [0.005, 1] (src/excent.cu:566-572). */
double excent_tau(double t_stream, const double* t_g, const double* f);

/* ------------------------------------------------------------ command line */

/* The excent command line (argv as bin/excent takes it: graph.egr then the
 * flags of src/excent.cu:269-298, plus --device N, --gpu-budget-gb X and
 * --device-loop). Prints the reference's stdout lines; returns the process
 * exit code (0, or 1 on a usage or run error). */
int excent_cli_main(int argc, char** argv);
/* bin/excent_params graph.egr out.env [--device N]: lambda1, the Katz and
 * eigenvector fixed-point means (FP64, on the GPU) and the .env file the CLI
 * reads (tools/excent_params.cu:73-172: same arguments, stdout lines, keys). */
int excent_params_main(int argc, char** argv);
/* bin/excent_reference: the FP64 oracle of a graph on the GPU (ref.bin of n
 * doubles) and --compare / --rank / --compare-dumps of float32 dumps against
 * it (tools/centrality_reference.cu:71-214: same modes, files and lines). */
int excent_reference_main(int argc, char** argv);

/* Measured ceiling of the scatter's operation: `ops` reductions
 * (red.global.add.f32, or .v4.f32 with vec4) to uniformly random vertices of
 * an n-vertex array, best of three timed launches; per_second = ops / time.
 * Allocates the array for the call. No counterpart in the reference. */
int excent_reduction_peak(int device, int n, int vec4, unsigned long long ops, double* per_second);

/* ------------------------------------------------------------ EGR file tools */

/* MatrixMarket coordinate file -> wide EGR (tools/efficient_converter.py:5-113).
 * n = max(rows, cols) of the size line; every later line with at least two
 * integer fields is an entry u v (1-based; further fields are ignored); entries
 * whose source is past n are skipped, as the reference converter does; a
 * source < 1 or a target outside [1, n] is EXCENT_ERR_IO. Lists keep the file's
 * order unless flags ask otherwise: 1 sort each list, 2 sort and drop repeated
 * entries, 4 drop self-loops, 8 add v -> u for every u -> v (u != v).
 * stats (may be NULL): {n, entries read, skipped, self-loops read, m written}. */
int excent_mtx_to_egr(const char* in, const char* out, int flags, unsigned long long* stats);
/* One line on an EGR file: n, m, max degree, and 20000 entries sampled with
 * mt19937_64 seeded 7 checked for a reverse entry and for self-loops; the same
 * line tools/egr_info.cpp:10-30 prints. */
int excent_egr_report(const char* path, char* out, int cap);
/* bin/excent_convert in.mtx out.egr [--sort] [--dedup] [--no-self-loops] [--symmetric] */
int excent_convert_main(int argc, char** argv);
/* bin/excent_info graph.egr (the report line above). */
int excent_info_main(int argc, char** argv);
/* bin/excent_evict [--report] file...: drop files from the page cache
 * (posix_fadvise DONTNEED after fdatasync) and print the resident share before
 * and after, or only the share with --report (tools/evict_file.c:18-65). */
int excent_evict_main(int argc, char** argv);

/* ------------------------------------------------------------ batched solves */

/* B personalized PageRank (kind EXCENT_PR: weight d / deg) or Katz (kind
 * EXCENT_KATZ: weight alpha) solves at once on a cached graph given by device
 * pointers (offsets n+1, lists m; symmetric for the PageRank reading).
 * Residuals and values are vertex-major float32 [n][B], B in {32, 64, 128,
 * 256}. No reference counterpart: the reference runs one solve per process. */
typedef struct excent_batch excent_batch;
int excent_batch_create(int device, int n, unsigned long long m, const unsigned long long* d_idx, const int32_t* d_adj,
                        int B, int kind, double d_or_alpha, excent_batch** out);
int excent_batch_destroy(excent_batch* b);
/* Reset all lanes to zero and seed lanes 0..nq-1: lane q adds vals[i] to the
 * residual of vids[i] for i in [lane_off[q], lane_off[q+1]); eps[q] is its
 * absolute threshold. Lanes >= nq stay idle. */
int excent_batch_seed(excent_batch* b, int nq, const int* lane_off, const int32_t* vids, const float* vals,
                      const float* eps);
/* Passes until no lane of any vertex is pending (or max_passes); with
 * use_graph all passes run as one CUDA graph with a conditional while node. */
int excent_batch_solve(excent_batch* b, int max_passes, int use_graph);
/* Passes, pushed vertices, pushed adjacency entries, 16-byte lane-group
 * reductions issued, touched rows examined and segments of lists longer than
 * 512 entries queued by the last solve (any output may be NULL). */
int excent_batch_stats(excent_batch* b, int* passes, unsigned long long* pushed_vertices,
                       unsigned long long* pushed_edges, unsigned long long* lane_updates,
                       unsigned long long* rows_checked, unsigned long long* hub_segments);
/* Values (or residuals) of lane q for all n vertices, to host float32. */
int excent_batch_read(excent_batch* b, int lane, int residual, float* out);
int excent_batch_stream(excent_batch* b, void** stream);
/* greedy (default 1): when a vertex has any pending lane, push every lane of
 * its row whose residual is nonzero, since the one read of its list serves
 * them all; 0: push only the pending lanes. Either way every lane ends with
 * |r| <= eps. */
int excent_batch_set_greedy(excent_batch* b, int greedy);
/* Segments of lists longer than 512 entries whose row has more than `groups`
 * active 16-byte lane groups scatter over the groups (each reduction covers a
 * contiguous stretch of the target row); sparser ones with the lanes over the
 * entries. Default 4 (measured: 4 and 8 best, 64 slowest, at B = 256). */
int excent_batch_set_dense(excent_batch* b, int groups);
/* Autotuner: time one batch of min(B, nq) of the given queries (seeded as
 * in excent_batch_seed) at each width B in {32, 64, 128, 256}, with the
 * greedy whole-row push off and on, and return the pair with the lowest time
 * per query (best_greedy may be NULL); per_query_ms[8] gets the times, entry
 * 2*i + greedy for width i. */
int excent_batch_autotune(int device, int n, unsigned long long m, const unsigned long long* d_idx, const int32_t* d_adj,
                          int kind, double d_or_alpha, int nq, const int* lane_off, const int32_t* vids,
                          const float* vals, const float* eps, int max_passes, int* best_B, int* best_greedy,
                          double* per_query_ms);
int excent_batch_launches(excent_batch* b, unsigned long long* launches);

/* ------------------------------------------------------------ adjoint (VJP) */

/* A weighted directed graph on the device: forward CSR (out-lists) and raw
 * float32 weights given as device pointers (kept by the caller), row-normalised
 * weights wn = w / rowsum, and a transposed CSR with the edge permutation.
 * Forward fixed points: PageRank x = (1 - d) t + d W^T x (t: a teleport
 * vector, NULL = all ones) and Katz x = beta + alpha W^T x, solved by a
 * weighted delta-push to an absolute eps. The VJP of a scalar loss with
 * dL/dx = c solves lambda = c + s W lambda by the same push on the transposed
 * lists and returns dL/dt (or dL/dbeta) and dL/dw for the raw weights through
 * the normalisation. All vectors are device pointers. No reference
 * counterpart: the reference has neither weights nor gradients. */
typedef struct excent_wgraph excent_wgraph;
int excent_wgraph_create(int device, int n, unsigned long long m, const unsigned long long* d_idx, const int32_t* d_adj,
                         const float* d_w, excent_wgraph** out);
int excent_wgraph_destroy(excent_wgraph* g);
/* New raw weights (device pointer, CSR order): renormalise. */
int excent_wgraph_set_weights(excent_wgraph* g, const float* d_w);
/* kind EXCENT_PR (s = d) or EXCENT_KATZ (s = alpha); d_t: teleport / beta
 * (n floats, NULL = ones); result copied to d_x_out when not NULL and kept
 * for the VJP. */
int excent_wgraph_forward(excent_wgraph* g, int kind, double s, const float* d_t, float eps, int max_passes,
                          float* d_x_out, int* passes, unsigned long long* pushed);
/* Adjoint solve for dL/dx = d_c after excent_wgraph_forward; writes dL/dt
 * (n) and dL/dw (m, CSR order of the forward graph) where not NULL. */
int excent_wgraph_vjp(excent_wgraph* g, const float* d_c, float eps, int max_passes, float* d_grad_t, float* d_grad_w,
                      int* passes, unsigned long long* pushed);
/* The adjoint vector lambda of the last VJP (n floats, device). */
int excent_wgraph_lambda(excent_wgraph* g, float* d_out);
/* FP64 Jacobi checks: loss c . x with raw weight `edge` shifted by delta
 * (edge < 0: none), and the FP64 gradient (dL/dt into grad_t[n], dL/dw into
 * grad_w[m], host arrays, either may be NULL). */
int excent_wgraph_loss_fp64(excent_wgraph* g, int kind, double s, const float* d_t, const float* d_c, long long edge,
                            double delta, double tol, double* loss);
int excent_wgraph_grad_fp64(excent_wgraph* g, int kind, double s, const float* d_t, const float* d_c, double tol,
                            double* grad_t, double* grad_w);
int excent_wgraph_stream(excent_wgraph* g, void** stream);
/* Out of core: move the transposed lists and their weights (4 + 4 + 8 bytes
 * per entry) to pinned, device-mapped host memory; the adjoint push then
 * reads them in place over the host link, the way excent_engine_host_cache
 * serves the plain engine. Irreversible for this graph. */
int excent_wgraph_host_transposed(excent_wgraph* g);

/* ------------------------------------------------------------ FP64 tools */

/* Given constants of a symmetric device-resident graph (offsets and lists
 * are device pointers): lambda1 by FP64 power iteration from the unit
 * all-ones vector (stop when the relative change of lambda1 < 1e-12 after 10
 * sweeps, <= 5000), the eigenvector fixed-point mean (v1 . 1)^2 / n, Katz
 * alpha = katz_numerator / lambda1 and the mean of x = 1 + alpha A x.
 * out = {lambda1, alpha, meanEV, meanKatz, sweeps}; d_v1 (device, n floats,
 * may be NULL) receives the unit principal eigenvector. tools/excent_params.cu:133-163. */
int excent_params_fp64(int device, int n, const unsigned long long* d_idx, const int32_t* d_adj,
                       double katz_numerator, double* out, float* d_v1);
/* Same results as excent_params_fp64, but the call allocates no device
 * memory: for hosts that keep every byte of device memory in their own pool
 * and forbid a library from calling cudaMalloc (or cannot afford the
 * device-wide synchronisation cudaMalloc/cudaFree may cause). Its two FP64
 * vectors and reduction slots live in a static device array of the library
 * (16 MiB + 512 bytes, held by every GPU that loads the library until exit),
 * so n must be <= EXCENT_NOALLOC_MAX_N; larger graphs get EXCENT_ERR_ARG.
 * Each call looks the array's address up (cudaGetSymbolAddress) on the
 * device it runs on, runs on the legacy default stream, reads sums back to
 * the host every sweep and ends with cudaDeviceSynchronize, so it must not
 * be called while any stream on the device is being captured. All calls
 * share the array: calls that overlap on the GPU race and must be serialised
 * by the caller. A graph with no edges gets EXCENT_ERR_ARG, as with
 * excent_params_fp64. No counterpart in the reference. */
#define EXCENT_NOALLOC_MAX_N (1 << 20)
int excent_params_fp64_noalloc(int device, int n, const unsigned long long* d_idx, const int32_t* d_adj,
                               double katz_numerator, double* out, float* d_v1);
/* FP64 reference solution on the device: kind 0 PageRank (x0 = 0.15,
 * x = 0.15 + 0.85 sum x_u / L(u)), 1 Katz (x = beta + alpha sum x_u),
 * 2 eigenvector (power iteration, unit L2 norm, sign fixed by the sum); Jacobi
 * until max|dx| / max|x| <= tol (eigenvector: max|dx| <= tol) or maxit.
 * x_out is a host array of n doubles. tools/centrality_reference.cu:31-59, 184-214. */
int excent_reference_fp64(int device, int n, const unsigned long long* d_idx, const int32_t* d_adj, int kind,
                          double alpha, double beta, double tol, int maxit, double* x_out, int* iterations);

/* FP64 personalized PageRank on the device: Jacobi on x = t + d sum x_u / L(u)
 * with t[v] = the sum of vals over the k seeds at v (the seeded solve's
 * initial residual), from x = t until max|dx| / max|x| <= tol or maxit. The
 * oracle of batched and seeded solves on graphs too large for the CPU one.
 * x_out: n doubles on the host. */
int excent_ppr_fp64(int device, int n, const unsigned long long* d_idx, const int32_t* d_adj, double d, int k,
                    const int32_t* vids, const float* vals, double tol, int maxit, double* x_out, int* iterations);

/* ------------------------------------------------------------ R-MAT graphs */

/* A graph held in device memory (CSR offsets, lists, optional weights). */
typedef struct excent_dgraph excent_dgraph;

/* Seeded R-MAT graph on `device`: n = 2^scale vertices, edge_factor * n / 2
 * pairs drawn (symmetric: both directions added) or edge_factor * n
 * (directed), quadrant probabilities a, b, c (d = 1 - a - b - c), self-loops
 * and duplicates dropped, lists sorted. weights: also float32 weights
 * uniform on [0.5, 1.5) per CSR edge. No reference counterpart: the
 * reference ingests .mtx files (tools/efficient_converter.py:5-113). */
int excent_rmat_generate(int device, int scale, int edge_factor, unsigned long long seed, double a, double b,
                         double c, int symmetric, int weights, excent_dgraph** out);
/* The symmetric graph of excent_rmat_generate (the same CSR, bit for bit),
 * generated in source-vertex partitions that fit device memory and written
 * as a wide EGR file: for out-of-core graphs larger than HBM holds at once.
 * max_part_keys = 0 sizes the partitions from free device memory. Writes the
 * entry count to *m_out and the number of partitions to *parts_out. No
 * reference counterpart (the reference converts .mtx files). */
int excent_rmat_write_egr(int device, int scale, int edge_factor, unsigned long long seed, double a, double b,
                          double c, unsigned long long max_part_keys, const char* path, unsigned long long* m_out,
                          int* parts_out);
int excent_dgraph_info(excent_dgraph* g, int* n, unsigned long long* m);
int excent_dgraph_device_ptrs(excent_dgraph* g, unsigned long long** idx, int32_t** adj, float** w);
/* Copy offsets (n+1), lists (m) and weights (m, if generated) to host memory; any may be NULL. */
int excent_dgraph_download(excent_dgraph* g, unsigned long long* idx, int32_t* adj, float* w);
int excent_dgraph_destroy(excent_dgraph* g);

#ifdef __cplusplus
}
#endif
#endif /* EXCENT_B200_H */
