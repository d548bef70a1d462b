// engine.cu -- the device engine of libexcent_b200: per-vertex state in HBM,
// the demand-snapshot kernel, the on-device fetch plan for cached chunks, the
// degree-dispatched push kernels, the hot (degree) cache kernels, staging
// slots, and the C entry points of include/excent_b200.h that drive them.
//
// Reference seams replaced (SPADE-IITJ/ExCent, paths relative to the project):
//   k_init                         src/excent.cu:41-47
//   k_snapshot (+ k_compact)       src/excent.cu:49-98, 150-164
//   push_vertex_g / k_push_*       src/excent.cu:100-148, 166-176, 199-209
//   k_compact_hot / k_fill_hot     src/excent.cu:178-182, 211-220
//   launch policy                  src/excent.cu:235-240, 629-652
#include <cuda_runtime.h>

#include <sys/mman.h>
#include <unistd.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "common.h"
#include "device.cuh"

namespace excent {

static constexpr int SNAP_GROUP = 16;     // bitmap words per warp step in the snapshot (512 vertices)
static constexpr unsigned HUB_MIN = 256;  // degree > 256: split into segments for whole warps
static constexpr unsigned HUB_SEG = 1024; // edges per hub segment
static constexpr int UNROLL = 4;          // independent index loads per lane in flight
static constexpr int STAGE_INTS = 1024;   // per warp: shared-memory stage of a tile's short lists (4 KiB)
static constexpr int BLOCK = 256;

enum { SRC_TABLE = 0, SRC_CHUNK = 1, SRC_GATHER = 2, SRC_HOT = 3, SRC_HUBS = 4 };
enum { WT_NONE = 0, WT_LIST = 1, WT_RANGE = 2 };
enum { LISTS_ALL = 0, LISTS_SHORT = 1, LISTS_LONG = 2 };

struct HubSeg {
    const int* nb;
    unsigned len;
    unsigned pad;
    float4 p;
};

// The work queue of one push launch: tiles are claimed in batches from
// `claim` (high 32 bits: batches claimed); long lists are queued as segments
// at `tail` and scattered by k_segments after the launch, one warp per
// segment. Nothing inside k_push waits on another warp, and no counter is
// contended by more than one atomic per warp and batch (claiming single
// segments inside the launch, one CAS on a shared head per segment, was
// measured ~100x slower on a 16.7M-vertex graph). Zeroed before every launch.
struct PushQueue {
    ull tail, claim, pad0, pad1;
};
static constexpr int TILE_BATCH = 32;           // at most this many tiles (of 32 items) per claim
static constexpr unsigned SPIN_LIMIT = 1u << 24; // bounded polls of an mbarrier

// Device control block: counters that live across kernels of one pass.
struct Ctrl {
    ull hotpend;
    ull pushed;        // adjacency entries pushed since init
    ull items;         // work items of the cached push in this pass
    int pass;          // passes that pushed so far
    int done;          // 1 once a snapshot found nothing pending (or max passes)
    int err;           // 1: a hub queue overflowed; 3: a bounded wait for a bulk copy gave up
    int sweep_pass;    // this pass is pushed chunk by chunk (set by k_plan)
    double rsum[MAXM]; // FP64 sum |r| of the last snapshot
    unsigned hcount;   // hot pending list length
    unsigned pad2;
    double ev_dot;     // FP64 (r_ev . v1) accumulated by the snapshot
    double ev_corr;    // component removed from r_ev by the next snapshot
    ull host_pushed;   // entries pushed from lists read in place in host memory
    ull chunk_runs;    // chunk launches a sweeping solve ran (chunks with items, summed over passes)
    ull lanes;         // sum over pushed lists of entries x measures carrying a nonzero weight
    ull taken;         // sum over pushed vertices of the measures taken
};

struct PassRec {
    ull pending, demand, hot_pending, pushed_before, lanes_before, taken_before;
    double rsum[MAXM];
    int n_list, n_range;
    int pad, pad1;
};

struct SnapArgs {
    int n, nc, words, groups_per_warp;
    void* r;
    const float* v1;   // unit principal eigenvector (EV normalisation step) or null
    int ev;            // measure index of the eigenvector
    double ev_skip;    // a pending v1 correction up to this size is carried, not written
    DevMeasures M;
    const ull* idx;
    const int* cv0;
    const uint32_t* hot;
    uint32_t* bitmap;
    ull* cnt;
    int* list;
    uint16_t* trace;
    Ctrl* ctrl;
};

struct PushArgs {
    void* x;
    void* r;
    DevMeasures M;
    const ull* idx;
    const uint32_t* hot;      // range items skip these (cached high-degree vertices)
    // SRC_TABLE: chunks from the HBM edge cache per the work table
    int nc;
    const int* cv0;
    const uint8_t* wt_type;
    const unsigned* wt_prefix; // nc + 1 item prefix
    const int* list;
    const int* cache;
    // SRC_CHUNK: one chunk, list or range, edges at ebase + (idx[v] - e0)
    int ctype, cv_0;
    unsigned ccount;
    const int* ebase;
    ull e0;
    // SRC_GATHER: k ids, offsets and edges staged together
    const int* vids;
    const ull* off;
    const int* gedges;
    unsigned gk;
    // SRC_HOT: compacted indices into the hot cache
    const int* hlist;
    const int* hids;
    const ull* hoff;
    const int* hedges;
    // outputs
    HubSeg* hubq;
    ull hub_cap;
    PushQueue* q;
    Ctrl* ctrl;
    // hub-target aggregation: encoded cache entries name slots of hub_id[hub_k]
    const int* hub_id;
    int hub_k;
    // high-degree-first order: SRC_HUBS pushes the lists longer than HUB_MIN
    // (hubv[*hubv_cnt]) first; SRC_TABLE then skips them
    const int* hubv;
    const ull* hubv_cnt;
    int lists;          // LISTS_ALL, or only the lists of at most HUB_MIN entries, or only the longer ones
    int chunk;          // SRC_TABLE: only chunk `chunk`'s items (-1: every chunk's)
    int stage;          // SRC_CHUNK / SRC_GATHER: bulk-copy each tile's short lists into shared memory
    int claim_tiles;    // tiles per claim; 0: up to TILE_BATCH, at least four claims per warp
    // lists past the device cache read in place from pinned host memory (zero copy)
    const int* hcache;   // entries [cache_edges, m), device-mapped
    ull cache_edges;
};

// Where list b (an edge offset) lives: the HBM cache prefix, or host memory past it.
__device__ __forceinline__ const int* list_at(const PushArgs& a, ull b) {
    return b < a.cache_edges ? a.cache + b : a.hcache + (b - a.cache_edges);
}

// Shared accumulators of the hub targets: zero at kernel start ...
template <typename T>
__device__ __forceinline__ T* hacc_init(int hub_k) {
    extern __shared__ float4 s_dyn[];
    T* h = reinterpret_cast<T*>(s_dyn);
    for (int i = threadIdx.x; i < hub_k; i += blockDim.x) h[i] = T{};
    __syncthreads();
    return hub_k ? h : nullptr;
}
// ... and one reduction per nonzero slot at kernel end (after every warp finished).
template <typename T>
__device__ __forceinline__ void hacc_flush(T* h, T* r, const int* hub_id, int hub_k) {
    __syncthreads();
    for (int i = threadIdx.x; i < hub_k; i += blockDim.x) {
        const T v = h[i];
        if (nonzero(v)) red_add(r, hub_id[i], v);
    }
}

// ------------------------------------------------------------------ kernels

template <int L>
__global__ void k_init(int n, const ull* idx, typename Lane<L>::T* x, typename Lane<L>::T* r, int nm, int k0, int k1,
                       int k2, float beta, double lambda) {
    const int kind[3] = {k0, k1, k2};
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n;
         v += (long long)gridDim.x * blockDim.x) {
        float xs[3], rs[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            xs[k] = 0.f; rs[k] = 0.f;
            if (k >= nm) continue;
            // src/excent.cu:43-45
            if (kind[k] == 0) { xs[k] = 0.f; rs[k] = 1.f - 0.85f; }
            else if (kind[k] == 1) { xs[k] = 0.f; rs[k] = beta; }
            else { xs[k] = 1.f; rs[k] = (float)((double)(idx[v + 1] - idx[v]) / lambda - 1.0); }  // lambda: see init_state
        }
        if constexpr (L == 1) { x[v] = xs[0]; r[v] = rs[0]; }
        else { x[v] = make_float4(xs[0], xs[1], xs[2], 0.f); r[v] = make_float4(rs[0], rs[1], rs[2], 0.f); }
    }
}

__device__ __forceinline__ int chunk_of(long long v, const int* cv0, int nc) {
    int lo = 0, hi = nc - 1;  // last chunk with cv0[c] <= v
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (cv0[mid] <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Demand snapshot. Each warp owns a contiguous run of 16-word groups; per
// group it ballots 512 vertices (one bitmap word per 32), writes the words
// coalesced, and adds the group's pending count and degree sum to its chunk
// with one atomic pair (per-lane atomics only where a group straddles a chunk
// boundary). The same atomic returns the offset at which the group's pending
// ids are appended to the chunk's list region list[cv0[c] ..]. Integer
// outputs equal src/excent.cu:69-98 exactly; list order is not defined.
template <int L>
__global__ void __launch_bounds__(BLOCK) k_snapshot(SnapArgs a) {
    typedef typename Lane<L>::T T;
    T* r = reinterpret_cast<T*>(a.r);
    const int lane = threadIdx.x & 31;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long ngroups = (a.words + SNAP_GROUP - 1) / SNAP_GROUP;
    long long g0 = gw * a.groups_per_warp, g1 = g0 + a.groups_per_warp;
    if (g1 > ngroups) g1 = ngroups;
    double rs0 = 0, rs1 = 0, rs2 = 0, evd = 0;
    // the v1 component measured by the previous snapshot is removed here only once it
    // matters (|c| max|v1| above a thousandth of eps); until then the residuals stay as
    // stored and the next dot product measures the component again, carried over
    const double evc_in = a.v1 ? a.ctrl->ev_corr : 0.0;
    const double evc = fabs(evc_in) > a.ev_skip ? evc_in : 0.0;
    unsigned hp = 0;
    for (long long g = g0; g < g1; g++) {
        const long long w0 = g * SNAP_GROUP;
        const int nw = (int)min((long long)SNAP_GROUP, (long long)a.words - w0);
        uint32_t myb = 0;
        ull mydeg = 0;
        for (int j4 = 0; j4 < nw; j4 += 4) {
            // four words' residuals (and v1 entries) in flight before they are examined
            T rq[4];
            float qq[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const long long v = (w0 + j4 + k) * 32 + lane;
                const bool in = j4 + k < nw && v < a.n;
                if (in) rq[k] = r[v];
                qq[k] = in && a.v1 ? a.v1[v] : 0.f;
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int j = j4 + k;
                if (j >= nw) break;
                const long long v = (w0 + j) * 32 + lane;
                bool pend = false;
                if (v < a.n) {
                    T rv = rq[k];
                    if (a.v1) {  // FP64 normalisation: drop the v1 component the push cannot remove
                        const float q = qq[k];
                        float* rp = reinterpret_cast<float*>(r + v) + (L == 1 ? 0 : a.ev);
                        float re;
                        if constexpr (L == 4) re = a.ev == 0 ? rv.x : a.ev == 1 ? rv.y : rv.z;
                        else re = rv;
                        if (evc != 0.0) {
                            re = (float)((double)re - evc * (double)q);
                            *rp = re;
                            if constexpr (L == 4) { if (a.ev == 0) rv.x = re; else if (a.ev == 1) rv.y = re; else rv.z = re; }
                            else rv = re;
                        }
                        evd += (double)re * (double)q;
                    }
                    if constexpr (L == 1) rs0 += fabs((double)rv);
                    else {
                        rs0 += fabs((double)rv.x);
                        rs1 += fabs((double)rv.y);
                        rs2 += fabs((double)rv.z);
                    }
                    pend = pending_of(rv, a.M);
                    if (a.trace && pend) a.trace[v]++;
                    if (a.hot && pend && bit_of(a.hot, v)) { hp++; pend = false; }
                    if (pend) mydeg += a.idx[v + 1] - a.idx[v];
                }
                const uint32_t b = __ballot_sync(FULL, pend);
                if (lane == j) myb = b;
            }
        }
        if (lane < nw) a.bitmap[w0 + lane] = myb;
        const unsigned cl = lane < nw ? (unsigned)__popc(myb) : 0u;
        const unsigned tot = __shfl_sync(FULL, warp_incl_scan(cl, lane), 31);
        if (tot == 0) continue;
        const long long vfirst = w0 * 32;
        long long vlast = (w0 + nw) * 32 - 1;
        if (vlast >= a.n) vlast = a.n - 1;
        const int c = chunk_of(vfirst, a.cv0, a.nc);
        const bool one = (c + 1 >= a.nc) || (vlast < a.cv0[c + 1]);
        if (one) {
            const ull dsum = warp_sum(mydeg);
            unsigned base = 0;
            if (lane == 0) {
                base = (unsigned)atomicAdd(&a.cnt[2 * c], (ull)tot);
                atomicAdd(&a.cnt[2 * c + 1], dsum);
            }
            base = __shfl_sync(FULL, base, 0);
            const unsigned excl = warp_incl_scan(cl, lane) - cl;
            int* out = a.list + a.cv0[c] + base;
            for (int j = 0; j < nw; j++) {
                const uint32_t b = __shfl_sync(FULL, myb, j);
                const unsigned e = __shfl_sync(FULL, excl, j);
                if ((b >> lane) & 1u) out[e + __popc(b & ((1u << lane) - 1u))] = (int)((w0 + j) * 32 + lane);
            }
        } else {
            // the group straddles chunk boundaries: group lanes by chunk, per word
            for (int j = 0; j < nw; j++) {
                const uint32_t b = __shfl_sync(FULL, myb, j);
                if (!b) continue;
                const long long v = (w0 + j) * 32 + lane;
                const bool pend = (b >> lane) & 1u;
                const int cc = pend ? chunk_of(v, a.cv0, a.nc) : -1;
                uint32_t rem = b;
                while (rem) {
                    const int leader = __ffs(rem) - 1;
                    const int cl2 = __shfl_sync(FULL, cc, leader);
                    const uint32_t mm = __ballot_sync(FULL, pend && cc == cl2);
                    const ull d = (pend && cc == cl2) ? a.idx[v + 1] - a.idx[v] : 0;
                    const ull ds = __shfl_sync(FULL, warp_sum(d), 0);
                    unsigned base = 0;
                    if (lane == leader) {
                        base = (unsigned)atomicAdd(&a.cnt[2 * cl2], (ull)__popc(mm));
                        atomicAdd(&a.cnt[2 * cl2 + 1], ds);
                    }
                    base = __shfl_sync(FULL, base, leader);
                    if ((mm >> lane) & 1u) a.list[a.cv0[cl2] + base + __popc(mm & ((1u << lane) - 1u))] = (int)v;
                    rem &= ~mm;
                }
            }
        }
    }
    // FP64 termination residual and hot pending count: block reduction, one atomic each
    __shared__ double s_rs[4][BLOCK / 32];
    __shared__ unsigned s_hp[BLOCK / 32];
    rs0 = warp_sum(rs0); rs1 = warp_sum(rs1); rs2 = warp_sum(rs2);
    evd = warp_sum(evd);
    hp = warp_sum(hp);
    const int wib = threadIdx.x >> 5;
    if (lane == 0) { s_rs[0][wib] = rs0; s_rs[1][wib] = rs1; s_rs[2][wib] = rs2; s_rs[3][wib] = evd; s_hp[wib] = hp; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
        unsigned th = 0;
        for (int i = 0; i < BLOCK / 32; i++) { t0 += s_rs[0][i]; t1 += s_rs[1][i]; t2 += s_rs[2][i]; t3 += s_rs[3][i]; th += s_hp[i]; }
        if (a.v1) atomicAdd(&a.ctrl->ev_dot, t3);
        atomicAdd(&a.ctrl->rsum[0], t0);
        if (a.M.nm > 1) atomicAdd(&a.ctrl->rsum[1], t1);
        if (a.M.nm > 2) atomicAdd(&a.ctrl->rsum[2], t2);
        if (th) atomicAdd(&a.ctrl->hotpend, (ull)th);
    }
}

// On-device fetch plan for a fully cached graph: per chunk with pending
// vertices choose its pending list (cnt < list_frac * vertices) or its whole
// range (src/excent.cu:639), build the item prefix, log the pass, decide
// termination (src/excent.cu:680, max passes :656), reset the counters the
// next snapshot accumulates into, and set the graph's loop condition.
__global__ void k_plan(int nc, const int* cv0, int n, ull* cnt, const uint8_t* cmode, double list_frac, int max_passes,
                       uint8_t* wt_type, unsigned* wt_prefix, Ctrl* ctrl, PushQueue* q0, PassRec* log, int log_cap,
                       cudaGraphConditionalHandle cond, int use_cond, const cudaGraphConditionalHandle* chunk_if,
                       int sweep, ull sweep_min) {
    __shared__ ull s_pend, s_dem;
    __shared__ unsigned s_carry;
    __shared__ int s_nl, s_nr, s_runs;
    __shared__ unsigned s_scan[1024];
    const int t = threadIdx.x;
    if (t == 0) { s_pend = 0; s_dem = 0; s_carry = 0; s_nl = 0; s_nr = 0; s_runs = 0; }
    __syncthreads();
    ull lp = 0, ld = 0;
    for (int c = t; c < nc; c += blockDim.x) { lp += cnt[2 * c]; ld += cnt[2 * c + 1]; }
    atomicAdd(&s_pend, lp);
    atomicAdd(&s_dem, ld);
    __syncthreads();
    const ull pend = s_pend, dem = s_dem, hp = ctrl->hotpend;
    const int p = ctrl->pass;
    const bool stop = ctrl->done || p >= max_passes || (pend == 0 && hp == 0);
    // a sweeping engine pushes a pass chunk by chunk while its demand is large, and in one
    // launch once the pending entries fall below sweep_min (the per-chunk launches would
    // then cost more than the in-pass ordering saves)
    const bool sweep_pass = sweep && !stop && dem >= sweep_min;
    // work table, scanned in tiles of blockDim.x chunks
    for (int base = 0; base < nc; base += blockDim.x) {
        const int c = base + t;
        unsigned items = 0;
        uint8_t ty = WT_NONE;
        if (!stop && c < nc && cmode[c] && cnt[2 * c] > 0) {
            const int v0 = cv0[c], v1 = c + 1 < nc ? cv0[c + 1] : n;
            // chunks read from host memory (mode 2) always push as ranges: a vertex that turns
            // pending during the pass is pushed in it, which saves whole passes over the link
            if (cmode[c] != 2 && (double)cnt[2 * c] < list_frac * (v1 - v0)) {
                ty = WT_LIST; items = (unsigned)cnt[2 * c]; atomicAdd(&s_nl, 1);
            }
            else { ty = WT_RANGE; items = (unsigned)(v1 - v0); atomicAdd(&s_nr, 1); }
        }
        s_scan[t] = items;
        __syncthreads();
        for (int o = 1; o < (int)blockDim.x; o <<= 1) {
            unsigned v = t >= o ? s_scan[t - o] : 0;
            __syncthreads();
            s_scan[t] += v;
            __syncthreads();
        }
        if (c < nc) {
            wt_type[c] = ty;
            wt_prefix[c + 1] = s_carry + s_scan[t];
            if (chunk_if) cudaGraphSetConditional(chunk_if[c], sweep_pass && items ? 1u : 0u);   // launch it?
            if (sweep_pass && items) atomicAdd(&s_runs, 1);
        }
        if (c == 0) wt_prefix[0] = 0;
        __syncthreads();
        if (t == blockDim.x - 1) s_carry += s_scan[t];
        __syncthreads();
    }
    __syncthreads();
    if (t == 0) {
        if (!stop && p < log_cap) {
            PassRec& R = log[p];
            R.pending = pend; R.demand = dem; R.hot_pending = hp; R.pushed_before = ctrl->pushed;
            R.lanes_before = ctrl->lanes; R.taken_before = ctrl->taken;
            for (int k = 0; k < MAXM; k++) R.rsum[k] = ctrl->rsum[k];
            R.n_list = s_nl; R.n_range = s_nr;
        }
        ctrl->items = stop ? 0 : s_carry;
        // pushes launched this pass: one per chunk with items, or the one whole-table push
        ctrl->chunk_runs += sweep_pass ? s_runs : (sweep && !stop && s_carry ? 1 : 0);
        ctrl->sweep_pass = sweep_pass ? 1 : 0;
        if (chunk_if) cudaGraphSetConditional(chunk_if[nc], sweep && !stop && !sweep_pass && s_carry ? 1u : 0u);
        if (stop) ctrl->done = 1; else ctrl->pass = p + 1;
        q0->tail = 0; q0->claim = 0;
        ctrl->hotpend = 0;
        ctrl->ev_corr = ctrl->ev_dot;
        ctrl->ev_dot = 0;
        if (!stop) for (int k = 0; k < MAXM; k++) ctrl->rsum[k] = 0;
        if (use_cond) cudaGraphSetConditional(cond, stop ? 0u : 1u);
    }
    // zero the demand table for the next snapshot (after everyone read it)
    __syncthreads();
    if (!stop) for (int c = t; c < 2 * nc; c += blockDim.x) cnt[c] = 0;
}

template <int SRC>
__device__ __forceinline__ bool get_item(const PushArgs& a, long long t, int& v, const int*& nb, ull& deg) {
    if constexpr (SRC == SRC_TABLE) {
        int lo = 0, hi = a.nc - 1;  // chunk c with prefix[c] <= t < prefix[c+1]
        if (a.chunk >= 0) {
            if (t >= (long long)a.wt_prefix[a.chunk + 1]) return false;
            lo = a.chunk;
        } else {
            if (t >= (long long)a.wt_prefix[a.nc]) return false;
            while (lo < hi) {
                int mid = (lo + hi + 1) >> 1;
                if ((long long)a.wt_prefix[mid] <= t) lo = mid; else hi = mid - 1;
            }
        }
        const unsigned i = (unsigned)(t - a.wt_prefix[lo]);
        if (a.wt_type[lo] == WT_LIST) v = a.list[a.cv0[lo] + i];
        else {
            v = a.cv0[lo] + (int)i;
            if (a.hot && bit_of(a.hot, v)) return false;
        }
        const ull b = a.idx[v];
        deg = a.idx[v + 1] - b;
        nb = list_at(a, b);
        return true;
    } else if constexpr (SRC == SRC_CHUNK) {
        if (t >= (long long)a.ccount) return false;
        if (a.ctype == WT_LIST) v = a.list[a.cv_0 + (int)t];
        else {
            v = a.cv_0 + (int)t;
            if (a.hot && bit_of(a.hot, v)) return false;
        }
        const ull b = a.idx[v];
        deg = a.idx[v + 1] - b;
        nb = a.ebase + (b - a.e0);
        return true;
    } else if constexpr (SRC == SRC_GATHER) {
        if (t >= (long long)a.gk) return false;
        v = a.vids[t];
        const ull b = a.off[t];
        deg = a.off[t + 1] - b;
        nb = a.gedges + b;
        return true;
    } else if constexpr (SRC == SRC_HUBS) {
        if (t >= (long long)*a.hubv_cnt) return false;
        v = a.hubv[t];
        const ull b = a.idx[v];
        deg = a.idx[v + 1] - b;
        nb = list_at(a, b);
        return true;
    } else {
        if (t >= (long long)a.ctrl->hcount) return false;
        const int j = a.hlist[t];
        v = a.hids[j];
        const ull b = a.hoff[j];
        deg = a.hoff[j + 1] - b;
        nb = a.hedges + b;
        return true;
    }
}

// Items [item_first, item_total) of one launch.
template <int SRC>
__device__ __forceinline__ long long item_first(const PushArgs& a) {
    if constexpr (SRC == SRC_TABLE) return a.chunk >= 0 ? a.wt_prefix[a.chunk] : 0;
    else return 0;
}
template <int SRC>
__device__ __forceinline__ long long item_total(const PushArgs& a) {
    if constexpr (SRC == SRC_TABLE) return a.wt_prefix[a.chunk >= 0 ? a.chunk + 1 : a.nc];
    else if constexpr (SRC == SRC_CHUNK) return a.ccount;
    else if constexpr (SRC == SRC_GATHER) return a.gk;
    else if constexpr (SRC == SRC_HUBS) return (long long)*a.hubv_cnt;
    else return a.ctrl->hcount;
}

// Scatter queued segment i (written by an earlier launch on the stream).
template <typename T>
__device__ __forceinline__ void scatter_segment(const PushArgs& a, T* r, T* hacc, int lane, ull i) {
    const HubSeg* hs = a.hubq + i;
    const int* nb = hs->nb;
    const unsigned len = hs->len;
    const float4 p4 = hs->p;
    T p;
    if constexpr (sizeof(T) == sizeof(float)) p = p4.x; else p = p4;
    warp_scatter(r, nb, len, p, lane, hacc);
}

// The segments a push launch queued: one warp per segment, right after it.
template <int L>
__global__ void __launch_bounds__(BLOCK) k_segments(void* rv, PushArgs a) {
    typedef typename Lane<L>::T T;
    T* r = reinterpret_cast<T*>(rv);
    const ull tail = min(a.q->tail, a.hub_cap);
    // a block none of whose warps has a segment leaves before it zeroes and flushes its slots
    if ((ull)blockIdx.x * (blockDim.x >> 5) >= tail) return;
    T* hacc = hacc_init<T>(a.hub_k);
    const int lane = threadIdx.x & 31;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (ull i = gw; i < tail; i += nwarps) scatter_segment(a, r, hacc, lane, i);
    hacc_flush(hacc, r, a.hub_id, a.hub_k);
}

// Push kernel (persistent grid, warp tiles of 32 items). Each lane takes one
// item's residual (the push-time re-check and exchange of
// src/excent.cu:109-112), then the warp dispatches by degree: lists of up to
// HUB_MIN entries are scattered edge-balanced across the warp (lane j handles
// the j-th entry of each 32-entry window of the tile's concatenated lists),
// longer lists are queued as HUB_SEG-entry segments for k_segments. Residuals
// are added with red.global (a float4 reduction per entry carries every
// measure of an `all` run), or in the block's shared hub-target slots.
template <int L, int SRC>
__global__ void __launch_bounds__(BLOCK) k_push(PushArgs a) {
    typedef typename Lane<L>::T T;
    T* x = reinterpret_cast<T*>(a.x);
    T* r = reinterpret_cast<T*>(a.r);
    const long long first = item_first<SRC>(a), total = item_total<SRC>(a);
    const long long ntiles = total > first ? (total - first + 31) / 32 : 0;
    // claims of up to TILE_BATCH tiles, fewer when there are not four claims per warp
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long per_claim =
        a.claim_tiles > 0 ? a.claim_tiles : max(1ll, min((long long)TILE_BATCH, ntiles / (4 * nwarps)));
    const long long nbatch = (ntiles + per_claim - 1) / per_claim;
    // with fewer batches than warps, only the first blocks claim: the others leave before they
    // zero and flush their hub-target slots (a small launch then costs only its active blocks)
    if ((long long)blockIdx.x * (blockDim.x >> 5) >= nbatch) return;
    T* hacc = hacc_init<T>(a.hub_k);
    // streamed and gathered lists: each tile's short lists arrive in shared memory by one bulk copy
    constexpr bool STAGED = SRC == SRC_CHUNK || SRC == SRC_GATHER;
    __shared__ __align__(16) int s_stage[STAGED ? BLOCK / 32 : 1][STAGED ? STAGE_INTS : 4];
    __shared__ unsigned long long s_bar[BLOCK / 32];
    __shared__ const int* s_nb[BLOCK / 32][32];
    __shared__ unsigned s_ex[BLOCK / 32][32];
    __shared__ T s_p[BLOCK / 32][32];
    __shared__ ull s_pushed[3][BLOCK / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    bool stage_on = STAGED && a.stage;
    unsigned bar_phase = 0;
    if (stage_on) {
        if (lane == 0) bar_init(&s_bar[wib]);
        __syncwarp();
    }
    ull pushed = 0, hpushed = 0, lanes = 0, taken = 0;
    for (;;) {
    // claim the next batch of tiles (and count this warp as working on it)
    ull claim = 0;
    if (lane == 0) claim = atomicAdd(&a.q->claim, 1ull << 32);
    const long long batch = (long long)(__shfl_sync(FULL, claim, 0) >> 32);
    const long long tile_end = batch < nbatch ? min((batch + 1) * per_claim, ntiles) : 0;
    for (long long tile = batch * per_claim; tile < tile_end; tile++) {
        int v = 0;
        const int* nb = nullptr;
        ull deg = 0;
        T p{};
        bool act = false;
        if (get_item<SRC>(a, first + tile * 32 + lane, v, nb, deg) &&
            !(a.lists == LISTS_SHORT && deg > HUB_MIN) && !(a.lists == LISTS_LONG && deg <= HUB_MIN)) {
            p = take(x, r, v, deg, a.M);
            act = nonzero(p) && deg > 0;
        }
        if (act) {
            const unsigned nz = measures_in(p);
            pushed += deg;
            lanes += deg * nz;
            taken += nz;
            if ((SRC == SRC_TABLE || SRC == SRC_HUBS) && a.hcache && a.idx[v] >= a.cache_edges) hpushed += deg;
        }
        const bool large = act && deg > HUB_MIN;
        // one queue reservation per warp for all its long lists (the counter is shared by the grid)
        const unsigned nseg = large ? (unsigned)((deg + HUB_SEG - 1) / HUB_SEG) : 0u;
        const unsigned sincl = warp_incl_scan(nseg, lane);
        const unsigned stot = __shfl_sync(FULL, sincl, 31);
        ull sbase = 0;
        if (stot) {
            if (lane == 0) sbase = atomicAdd(&a.q->tail, (ull)stot);
            sbase = __shfl_sync(FULL, sbase, 0);
        }
        if (large) {
            const ull base = sbase + (sincl - nseg);
            if (base + nseg <= a.hub_cap) {
                HubSeg* q = a.hubq + base;
                for (unsigned s = 0; s < nseg; s++) {
                    HubSeg h;
                    h.nb = nb + (ull)s * HUB_SEG;
                    h.len = (unsigned)min((ull)HUB_SEG, deg - (ull)s * HUB_SEG);
                    h.pad = 0;
                    if constexpr (L == 1) h.p = make_float4(p, 0.f, 0.f, 0.f); else h.p = p;
                    q[s] = h;
                }
            } else {
                atomicExch(&a.ctrl->err, 1);
            }
        }
        // every other list of the tile, edge-balanced: the tile's lists are
        // concatenated and lane j handles entry j of each 32-entry slice, UNROLL
        // slices at a time so each lane has UNROLL index loads in flight
        const unsigned ds = (act && !large) ? (unsigned)deg : 0u;
        const unsigned nz = __ballot_sync(FULL, ds != 0);
        if (nz) {
            const unsigned incl = warp_incl_scan(ds, lane);
            const unsigned tot = __shfl_sync(FULL, incl, 31);
            const unsigned ex = incl - ds;
            const int rank = __popc(nz & ((1u << lane) - 1u));
            if (ds) { s_nb[wib][rank] = nb; s_ex[wib][rank] = ex; s_p[wib][rank] = p; }
            __syncwarp();
            // streamed / gathered tiles: consecutive items' lists lie back to back, so the
            // short ones span one stretch; when it fits, one bulk copy brings it (16-byte
            // aligned, the buffers are padded) and the entries are read from shared memory
            const int* st_base = nullptr;
            if (stage_on) {
                unsigned long long lo = ds ? (unsigned long long)(uintptr_t)nb : ~0ull;
                unsigned long long hi = ds ? (unsigned long long)(uintptr_t)(nb + ds) : 0ull;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    lo = min(lo, __shfl_xor_sync(FULL, lo, o));
                    hi = max(hi, __shfl_xor_sync(FULL, hi, o));
                }
                const unsigned long long a0 = lo & ~15ull, a1 = (hi + 15ull) & ~15ull;
                if (a1 - a0 <= (unsigned long long)STAGE_INTS * sizeof(int)) {
                    if (lane == 0) bulk_stage(&s_bar[wib], s_stage[wib], (const void*)(uintptr_t)a0, (unsigned)(a1 - a0));
                    const bool ok = __all_sync(FULL, bar_wait(&s_bar[wib], bar_phase, SPIN_LIMIT));
                    bar_phase ^= 1u;
                    if (ok) st_base = (const int*)(uintptr_t)a0;
                    else {   // never expected: leave the stage alone from here on
                        if (lane == 0) atomicExch(&a.ctrl->err, 3);
                        stage_on = false;
                    }
                }
            }
            const unsigned le = lane == 31 ? FULL : (2u << lane) - 1u;
            for (unsigned j0 = 0; j0 < tot; j0 += 32 * UNROLL) {
                int u[UNROLL];
                int own[UNROLL];
#pragma unroll
                for (int k = 0; k < UNROLL; k++) {
                    // owner of entry wb+lane: the last nonempty list starting at or before it
                    // (bit i of `starts`: a list begins at entry wb+i)
                    const unsigned wb = j0 + 32 * k;
                    const unsigned j = wb + lane;
                    const unsigned starts =
                        __reduce_or_sync(FULL, (ds && ex >= wb && ex - wb < 32) ? 1u << (ex - wb) : 0u);
                    const int o = __popc(__ballot_sync(FULL, ds && ex <= wb)) - 1 + __popc(starts & le & ~1u);
                    own[k] = j < tot ? o : -1;
                    if constexpr (STAGED) {
                        if (st_base) u[k] = j < tot ? s_stage[wib][(s_nb[wib][o] - st_base) + (j - s_ex[wib][o])] : 0;
                        else u[k] = j < tot ? ld_edge(s_nb[wib][o] + (j - s_ex[wib][o])) : 0;
                    } else {
                        u[k] = j < tot ? ld_edge(s_nb[wib][o] + (j - s_ex[wib][o])) : 0;
                    }
                }
#pragma unroll
                for (int k = 0; k < UNROLL; k++)
                    if (own[k] >= 0) scatter_one(r, u[k], s_p[wib][own[k]], hacc);
            }
            __syncwarp();
        }
    }
    if (batch >= nbatch) break;
    }
    pushed = warp_sum(pushed);
    lanes = warp_sum(lanes);
    taken = warp_sum(taken);
    if (lane == 0) { s_pushed[0][wib] = pushed; s_pushed[1][wib] = lanes; s_pushed[2][wib] = taken; }
    if (a.hcache) {   // rare path (zero-copy host lists): one atomic per warp
        hpushed = warp_sum(hpushed);
        if (lane == 0 && hpushed) atomicAdd(&a.ctrl->host_pushed, hpushed);
    }
    hacc_flush(hacc, r, a.hub_id, a.hub_k);
    if (threadIdx.x < 3) {
        ull t = 0;
        for (int i = 0; i < BLOCK / 32; i++) t += s_pushed[threadIdx.x][i];
        if (t) atomicAdd(threadIdx.x == 0 ? &a.ctrl->pushed : threadIdx.x == 1 ? &a.ctrl->lanes : &a.ctrl->taken, t);
    }
}

// Pending hot vertices among hot ids [lo, hi) at launch time, appended with
// one global atomic per block (src/excent.cu:178-182).
template <int L>
__global__ void __launch_bounds__(BLOCK) k_compact_hot(int lo, int hi, const int* hids, const void* rv, DevMeasures M,
                                                       int* out, Ctrl* ctrl) {
    typedef typename Lane<L>::T T;
    const T* r = reinterpret_cast<const T*>(rv);
    __shared__ unsigned s_cnt, s_base;
    __shared__ unsigned s_w[BLOCK / 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (long long i0 = lo + (long long)blockIdx.x * BLOCK; i0 < hi; i0 += (long long)gridDim.x * BLOCK) {
        const long long i = i0 + threadIdx.x;
        const bool p = i < hi && pending_of(r[hids[i]], M);
        const uint32_t b = __ballot_sync(FULL, p);
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        if (lane == 0) s_w[wib] = atomicAdd(&s_cnt, (unsigned)__popc(b));
        __syncthreads();
        if (threadIdx.x == 0) s_base = s_cnt ? atomicAdd(&ctrl->hcount, s_cnt) : 0;
        __syncthreads();
        if (p) out[s_base + s_w[wib] + __popc(b & ((1u << lane) - 1u))] = (int)i;
        __syncthreads();
    }
}

// Pass 0: copy the lists of hot ids [lo, hi) out of a chunk staged at src
// (edges from e0), one warp per vertex (src/excent.cu:211-220).
__global__ void k_fill_hot(int lo, int hi, const int* hids, const ull* hoff, const ull* idx, ull e0, const int* src,
                           int* hedges) {
    const long long w = lo + ((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= hi) return;
    const int* from = src + (idx[hids[w]] - e0);
    int* to = hedges + hoff[w];
    for (ull i = lane, d = hoff[w + 1] - hoff[w]; i < d; i += 32) to[i] = from[i];
}


// Vertices whose lists are longer than HUB_MIN, appended in any order.
__global__ void k_hub_list(int n, const ull* idx, int* out, ull* cnt) {
    const int lane = threadIdx.x & 31;
    for (long long v0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) & ~31ll; v0 < n;
         v0 += (long long)gridDim.x * blockDim.x) {
        const long long v = v0 + lane;
        const bool h = v < n && idx[v + 1] - idx[v] > HUB_MIN;
        const unsigned b = __ballot_sync(FULL, h);
        if (!b) continue;
        ull base = 0;
        if (lane == 0) base = atomicAdd(cnt, (ull)__popc(b));
        base = __shfl_sync(FULL, base, 0);
        if (h && out) out[base + __popc(b & ((1u << lane) - 1u))] = (int)v;
    }
}

// Encode / decode the edge cache for hub-target aggregation.
// hub_id is sorted: a binary search in shared memory gives an entry's slot.
__global__ void k_hub_encode(ull m, int* adj, const int* hub_id, int hub_k) {
    extern __shared__ int s_ids[];
    for (int i = threadIdx.x; i < hub_k; i += blockDim.x) s_ids[i] = hub_id[i];
    __syncthreads();
    for (ull e = blockIdx.x * (ull)blockDim.x + threadIdx.x; e < m; e += (ull)gridDim.x * blockDim.x) {
        const int u = adj[e];
        if (u < 0) continue;
        int lo = 0, hi = hub_k - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (s_ids[mid] < u) lo = mid + 1; else hi = mid;
        }
        if (s_ids[lo] == u) adj[e] = (int)(0x80000000u | (unsigned)lo);
    }
}
__global__ void k_hub_decode(ull m, int* adj, const int* hub_id, int hub_k) {
    for (ull e = blockIdx.x * (ull)blockDim.x + threadIdx.x; e < m; e += (ull)gridDim.x * blockDim.x) {
        const int u = adj[e];
        if (u < 0 && (u & HUB_MASK) < hub_k) adj[e] = hub_id[u & HUB_MASK];
    }
}

// Measure i of a float4 layout into a float array, for readback.
__global__ void k_extract(int n, const float4* s, int i, float* out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const float4 q = s[v];
        out[v] = i == 0 ? q.x : i == 1 ? q.y : q.z;
    }
}
__global__ void k_insert(int n, float4* s, int i, const float* in) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        float4 q = s[v];
        if (i == 0) q.x = in[v]; else if (i == 1) q.y = in[v]; else q.z = in[v];
        s[v] = q;
    }
}

}  // namespace excent

using namespace excent;

// ------------------------------------------------------------------ engine

struct Slot {
    int* h_edges = nullptr; int* d_edges = nullptr;
    int* h_vids = nullptr; int* d_vids = nullptr;
    ull* h_off = nullptr; ull* d_off = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
};

struct excent_engine {
    int dev = 0, sms = 0;
    int n = 0;
    ull m = 0;
    int nm = 0, L = 1;
    excent_measures meas{};
    DevMeasures M{};
    int nc = 0;
    std::vector<int> cv0;
    std::vector<ull> ce;
    std::vector<uint8_t> loaded;
    // device state
    ull* d_idx = nullptr;
    void* d_x = nullptr;
    void* d_r = nullptr;
    uint32_t* d_bitmap = nullptr;
    ull* d_cnt = nullptr;
    int* d_cv0 = nullptr;
    int* d_list = nullptr;
    Ctrl* d_ctrl = nullptr;
    uint8_t* d_cmode = nullptr;
    uint8_t* d_wt_type = nullptr;
    unsigned* d_wt_prefix = nullptr;
    HubSeg* d_hubq[3] = {nullptr, nullptr, nullptr};  // per stream: main, slot 0, slot 1
    ull hub_cap[3] = {0, 0, 0};
    PushQueue* d_queue = nullptr;                      // per stream: main, slot 0, slot 1
    bool hot_skip = false;                             // this pass skips cached high-degree vertices
    PassRec* d_log = nullptr;
    int log_cap = 0;
    uint16_t* d_trace = nullptr;
    bool trace_on = false;
    float* d_tmp = nullptr;  // n floats for readback of the float4 layout
    float* d_v1 = nullptr;   // unit principal eigenvector for the EV normalisation step
    int* d_hub_id = nullptr; // hub-target aggregation: vertex of each slot
    int hub_k = 0;           // slots in use (0: off)
    int* h_hcache = nullptr; // pinned, mapped host copy of the entries past the device cache
    ull hcache_edges = 0;
    const int* d_hcache = nullptr;  // its device address, once all of it is pinned
    // registered in pieces (excent_engine_host_cache_begin/_pin): an anonymous mapping
    size_t hcache_map_bytes = 0;
    std::vector<std::pair<char*, size_t>> hcache_pieces;
    size_t hcache_pinned = 0;       // bytes registered so far, from the start
    int* d_hubv = nullptr;   // high-degree-first order: vertices with lists longer than HUB_MIN
    ull* d_hubv_cnt = nullptr;
    ull hubv_cap = 0;
    int hub_order = -1;      // high-degree lists: 0 in table order, 1 first, 2 last, -1 by the chunk count
    int claim_tiles = 0;     // tiles per claim of k_push (0: by the launch's size)
    int sweep_mode = -1;     // cached pushes chunk by chunk (1), in one launch (0), -1 by the chunk count
    double sweep_frac = 0.5; // ... only in passes whose pending entries reach sweep_frac * m
    cudaGraphConditionalHandle* d_chunk_if = nullptr;  // per chunk: does this pass push it (graph IF nodes)
    std::vector<cudaGraphConditionalHandle> h_chunk_if;
    bool hubv_stale = true;
    bool ev_proj = false;
    double ev_skip = 0;      // carry (do not write) a v1 correction of at most this size
    int ev_index = -1;
    int* d_cache = nullptr;
    ull cache_edges = 0;
    // hot cache
    int nh = 0;
    int* d_hids = nullptr; ull* d_hoff = nullptr; int* d_hedges = nullptr; uint32_t* d_hot = nullptr;
    int* d_hlist = nullptr;
    // pinned host mirrors
    ull* h_cnt = nullptr;
    Ctrl* h_ctrl = nullptr;
    uint8_t* h_wt_type = nullptr;
    unsigned* h_wt_prefix = nullptr;
    // streams
    cudaStream_t s_main = nullptr;
    Slot slot[2];
    bool slots_ok = false, zc = false;
    ull max_chunk_edges = 0;
    int max_chunk_verts = 0;
    // graph
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    int graph_max_passes = -1;
    double graph_list_frac = -1;
    // per-kernel timing of the host-driven device solve (excent_engine_profile)
    bool prof = false;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    double prof_ms[4] = {0, 0, 0, 0};  // snapshot, plan, push, hub
    ull prof_passes = 0;
    // launch grids
    int grid_push = 0, grid_snap = 0, groups_per_warp = 1;
    ull launches = 0;
    ull n_list = 0, n_range = 0;
};

// Device pointers and launch parameters are baked into the solve graph:
// any reallocation or option change drops it.
static void invalidate_graph(excent_engine* e) {
    if (e->gexec) { cudaGraphExecDestroy(e->gexec); e->gexec = nullptr; }
    if (e->graph) { cudaGraphDestroy(e->graph); e->graph = nullptr; }
}

static void scrub_queues(excent_engine* e);
// Release the host cache, pinned whole (cudaHostAlloc) or in pieces of an anonymous mapping.
static void free_host_cache(excent_engine* e) {
    if (!e->h_hcache) return;
    if (e->hcache_map_bytes) {
        for (auto& pc : e->hcache_pieces) cudaHostUnregister(pc.first);
        munmap(e->h_hcache, e->hcache_map_bytes);
    } else {
        cudaFreeHost(e->h_hcache);
    }
    e->h_hcache = nullptr;
    e->d_hcache = nullptr;
    e->hcache_edges = 0;
    e->hcache_map_bytes = 0;
    e->hcache_pieces.clear();
    e->hcache_pinned = 0;
}
static const char* ctrl_error(int err) {
    return err == 3 ? "a push kernel's wait for a bulk copy of its lists timed out"
                    : "device capacity check failed (hub queue overflow)";
}
static int ensure_hubv(excent_engine* e);

// Pass order. By default a graph cut into several chunks is pushed chunk by
// chunk, which is how the reference launches its resident chunks
// (src/excent.cu:684-688): every chunk then sees what the earlier ones pushed
// in the same pass, and a solve pushes about as many entries as the
// reference's. Inside each launch the chunk's long lists go first (a launch
// otherwise leaves them to k_segments, after its short lists; first measured
// smaller errors). A single chunk pushes the graph's high-degree lists first
// (measured: fewer entries and smaller errors than table order there). Both
// can be set explicitly.
static bool sweep_of(const excent_engine* e) { return e->sweep_mode >= 0 ? e->sweep_mode != 0 : e->nc > 1; }
// A sweeping engine sweeps the passes whose pending entries reach this many.
static ull sweep_min_entries(const excent_engine* e) { return (ull)(e->sweep_frac * (double)e->m); }
static int order_of(const excent_engine* e) { return e->hub_order >= 0 ? e->hub_order : (sweep_of(e) ? 3 : 1); }
// the order a pass can run: a high-degree order needs the listed high-degree vertices
static int effective_order(const excent_engine* e);

static int free_engine(excent_engine* e) {
    if (!e) return EXCENT_OK;
    cudaSetDevice(e->dev);
    cudaDeviceSynchronize();
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    if (e->graph) cudaGraphDestroy(e->graph);
    void* dptrs[] = {e->d_chunk_if, e->d_hub_id, e->d_hubv, e->d_hubv_cnt, e->d_v1, e->d_idx, e->d_x, e->d_r, e->d_bitmap, e->d_cnt, e->d_cv0, e->d_list, e->d_ctrl, e->d_cmode,
                     e->d_wt_type, e->d_wt_prefix, e->d_hubq[0], e->d_hubq[1], e->d_hubq[2], e->d_queue, e->d_log, e->d_trace, e->d_tmp, e->d_cache,
                     e->d_hids, e->d_hoff, e->d_hedges, e->d_hot, e->d_hlist};
    for (void* p : dptrs) if (p) cudaFree(p);
    void* hptrs[] = {e->h_cnt, e->h_ctrl, e->h_wt_type, e->h_wt_prefix};
    for (void* p : hptrs) if (p) cudaFreeHost(p);
    for (Slot& s : e->slot) {
        if (s.h_edges) cudaFreeHost(s.h_edges);
        if (s.h_vids) cudaFreeHost(s.h_vids);
        if (s.h_off) cudaFreeHost(s.h_off);
        if (!e->zc) {
            if (s.d_edges) cudaFree(s.d_edges);
            if (s.d_vids) cudaFree(s.d_vids);
            if (s.d_off) cudaFree(s.d_off);
        }
        if (s.st) cudaStreamDestroy(s.st);
        if (s.done) cudaEventDestroy(s.done);
    }
    for (cudaEvent_t ev : e->ev) if (ev) cudaEventDestroy(ev);
    free_host_cache(e);
    if (e->s_main) cudaStreamDestroy(e->s_main);
    delete e;
    return EXCENT_OK;
}

#define EX_ALLOC(ptr, bytes) do { if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) { cudaGetLastError(); \
    ::excent::set_error("device allocation of %llu bytes failed (%s)", (ull)(bytes), #ptr); return EXCENT_ERR_NOMEM; } } while (0)
#define EX_HALLOC(ptr, bytes) do { if (cudaMallocHost((void**)&(ptr), (bytes)) != cudaSuccess) { cudaGetLastError(); \
    ::excent::set_error("pinned allocation of %llu bytes failed (%s)", (ull)(bytes), #ptr); return EXCENT_ERR_NOMEM; } } while (0)

static int engine_setup(excent_engine* e, int device, int n, ull m, const excent_measures* ms, int nc,
                        const int* chunk_v0, const ull* chunk_e) {
    EX_CUDA(cudaSetDevice(device));
    e->dev = device;
    EX_CUDA(cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, device));
    e->n = n; e->m = m; e->nm = ms->nm; e->L = ms->nm == 1 ? 1 : 4;
    e->meas = *ms;
    e->M.nm = ms->nm;
    for (int k = 0; k < MAXM; k++) {
        e->M.eps[k] = k < ms->nm ? ms->eps[k] : 0.f;
        e->M.scale[k] = k < ms->nm ? ms->scale[k] : 0.f;
        e->M.divdeg[k] = k < ms->nm ? ms->divdeg[k] : 0;
    }
    e->nc = nc;
    e->cv0.assign(chunk_v0, chunk_v0 + nc);
    e->ce.assign(chunk_e, chunk_e + nc + 1);
    e->loaded.assign(nc, 0);
    for (int c = 0; c < nc; c++) {
        const int v1 = c + 1 < nc ? chunk_v0[c + 1] : n;
        EX_CHECK_ARG(chunk_v0[c] >= 0 && chunk_v0[c] < v1 && v1 <= n, "chunk %d has an empty or bad range", c);
        EX_CHECK_ARG(chunk_e[c] <= chunk_e[c + 1], "chunk %d has bad edge bounds", c);
        e->max_chunk_verts = std::max(e->max_chunk_verts, v1 - chunk_v0[c]);
        e->max_chunk_edges = std::max(e->max_chunk_edges, chunk_e[c + 1] - chunk_e[c]);
    }
    EX_CHECK_ARG(chunk_v0[0] == 0 && chunk_e[0] == 0 && chunk_e[nc] == m, "chunks must cover the graph");
    EX_CUDA(cudaStreamCreateWithFlags(&e->s_main, cudaStreamNonBlocking));
    const size_t words = ((size_t)n + 31) / 32;
    const size_t vbytes = (size_t)n * (e->L == 1 ? sizeof(float) : sizeof(float4));
    EX_ALLOC(e->d_idx, ((size_t)n + 1) * sizeof(ull));
    EX_ALLOC(e->d_x, vbytes);
    EX_ALLOC(e->d_r, vbytes);
    EX_ALLOC(e->d_bitmap, words * sizeof(uint32_t));
    EX_ALLOC(e->d_cnt, 2 * (size_t)nc * sizeof(ull));
    EX_ALLOC(e->d_cv0, (size_t)nc * sizeof(int));
    EX_ALLOC(e->d_list, (size_t)n * sizeof(int));
    EX_ALLOC(e->d_ctrl, sizeof(Ctrl));
    EX_ALLOC(e->d_cmode, (size_t)nc);
    EX_ALLOC(e->d_wt_type, (size_t)nc);
    EX_ALLOC(e->d_wt_prefix, ((size_t)nc + 1) * sizeof(unsigned));
    e->hub_cap[0] = m / HUB_SEG + m / HUB_MIN + 64;
    EX_ALLOC(e->d_hubq[0], e->hub_cap[0] * sizeof(HubSeg));
    EX_ALLOC(e->d_queue, 3 * sizeof(PushQueue));
    e->log_cap = 1 << 17;
    EX_ALLOC(e->d_log, (size_t)e->log_cap * sizeof(PassRec));
    if (e->L == 4) EX_ALLOC(e->d_tmp, (size_t)n * sizeof(float));
    EX_HALLOC(e->h_cnt, 2 * (size_t)nc * sizeof(ull));
    EX_HALLOC(e->h_ctrl, sizeof(Ctrl));
    EX_HALLOC(e->h_wt_type, (size_t)nc);
    EX_HALLOC(e->h_wt_prefix, ((size_t)nc + 1) * sizeof(unsigned));
    EX_CUDA(cudaMemcpy(e->d_cv0, chunk_v0, (size_t)nc * sizeof(int), cudaMemcpyHostToDevice));
    EX_CUDA(cudaMemset(e->d_ctrl, 0, sizeof(Ctrl)));
    EX_CUDA(cudaMemset(e->d_cnt, 0, 2 * (size_t)nc * sizeof(ull)));
    EX_CUDA(cudaMemset(e->d_cmode, 0, (size_t)nc));
    EX_CUDA(cudaMemset(e->d_queue, 0, 3 * sizeof(PushQueue)));
    int occ = 0;
    if (e->L == 1) EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_push<1, SRC_TABLE>, BLOCK, 0));
    else EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_push<4, SRC_TABLE>, BLOCK, 0));
    e->grid_push = e->sms * std::max(1, occ);
    int occs = 0;
    if (e->L == 1) EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occs, k_snapshot<1>, BLOCK, 0));
    else EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occs, k_snapshot<4>, BLOCK, 0));
    const long long groups = ((long long)words + SNAP_GROUP - 1) / SNAP_GROUP;
    const long long max_warps = (long long)e->sms * std::max(1, occs) * (BLOCK / 32);
    e->groups_per_warp = (int)std::max(1LL, (groups + max_warps - 1) / max_warps);
    const long long warps = (groups + e->groups_per_warp - 1) / e->groups_per_warp;
    e->grid_snap = (int)std::max(1LL, (warps + BLOCK / 32 - 1) / (BLOCK / 32));
    return EXCENT_OK;
}

// Encode cache entries [e0, e1) for hub-target aggregation (no-op when off).
static void hub_encode(excent_engine* e, ull e0, ull e1, cudaStream_t st) {
    if (!e->hub_k || e1 <= e0) return;
    k_hub_encode<<<e->sms * 4, BLOCK, (size_t)e->hub_k * sizeof(int), st>>>(e1 - e0, e->d_cache + e0, e->d_hub_id,
                                                                            e->hub_k);
    e->launches++;
}

static size_t hub_smem(const excent_engine* e) {
    return (size_t)e->hub_k * (e->L == 1 ? sizeof(float) : sizeof(float4));
}

extern "C" int excent_measures_make(excent_measures* out, const char* measure, double alpha, double beta,
                                    double lambda, double eps_pr, double eps_katz, double eps_ev) {
    EX_CHECK_ARG(out && measure, "null argument");
    excent_measures M{};
    int kinds[3], nm = 0;
    if (!strcmp(measure, "pr")) kinds[nm++] = EXCENT_PR;
    else if (!strcmp(measure, "katz")) kinds[nm++] = EXCENT_KATZ;
    else if (!strcmp(measure, "ev")) kinds[nm++] = EXCENT_EV;
    else if (!strcmp(measure, "all")) { kinds[nm++] = EXCENT_PR; kinds[nm++] = EXCENT_KATZ; kinds[nm++] = EXCENT_EV; }
    else EX_FAIL(EXCENT_ERR_ARG, "--measure must be pr, katz, ev or all");
    for (int i = 0; i < nm; i++) {
        if (kinds[i] == EXCENT_KATZ && (alpha <= 0 || eps_katz <= 0)) EX_FAIL(EXCENT_ERR_ARG, "katz needs --alpha and --eps-katz");
        if (kinds[i] == EXCENT_EV && (lambda <= 0 || eps_ev <= 0)) EX_FAIL(EXCENT_ERR_ARG, "ev needs --lambda and --eps-ev");
    }
    M.nm = nm;
    for (int i = 0; i < nm; i++) {
        const int k = kinds[i];
        M.kind[i] = k;
        M.eps[i] = (float)(k == EXCENT_PR ? eps_pr : k == EXCENT_KATZ ? eps_katz : eps_ev);
        M.scale[i] = (float)(k == EXCENT_PR ? 0.85f : k == EXCENT_KATZ ? alpha : 1.0 / lambda);
        M.divdeg[i] = k == EXCENT_PR;
    }
    M.beta = beta;
    M.lambda = lambda;
    M.flags = 0;
    *out = M;
    return EXCENT_OK;
}

extern "C" int excent_engine_create(int device, int n, unsigned long long m, const excent_measures* measures, int nc,
                                    const int* chunk_v0, const unsigned long long* chunk_e, excent_engine** out) {
    EX_CHECK_ARG(out && measures && chunk_v0 && chunk_e, "null argument");
    EX_CHECK_ARG(n >= 1, "n must be >= 1");
    EX_CHECK_ARG(nc >= 1 && nc <= n, "bad chunk count %d", nc);
    EX_CHECK_ARG(measures->nm >= 1 && measures->nm <= 3, "nm must be 1..3");
    *out = nullptr;
    excent_engine* e = new excent_engine();
    const int rc = engine_setup(e, device, n, m, measures, nc, chunk_v0, chunk_e);
    if (rc != EXCENT_OK) {
        std::string msg = excent::get_error();
        free_engine(e);
        excent::set_error("%s", msg.c_str());
        return rc;
    }
    *out = e;
    return EXCENT_OK;
}

extern "C" int excent_engine_destroy(excent_engine* e) { return free_engine(e); }

extern "C" int excent_engine_upload_offsets(excent_engine* e, const unsigned long long* idx, unsigned long long v0,
                                            unsigned long long count) {
    EX_CHECK_ARG(e && idx, "null argument");
    EX_CHECK_ARG(v0 + count <= (ull)e->n + 1, "offsets out of range");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaMemcpyAsync(e->d_idx + v0, idx, count * sizeof(ull), cudaMemcpyHostToDevice, e->s_main));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    e->hubv_stale = true;
    return EXCENT_OK;
}

extern "C" int excent_engine_upload_device(excent_engine* e, const unsigned long long* d_idx, const int32_t* d_adj) {
    EX_CHECK_ARG(e && d_idx && (d_adj || e->m == 0), "null argument");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaMemcpyAsync(e->d_idx, d_idx, ((size_t)e->n + 1) * sizeof(ull), cudaMemcpyDeviceToDevice, e->s_main));
    if (e->cache_edges != e->m) EX_TRY(excent_engine_reserve_cache(e, e->m));
    if (e->m) EX_CUDA(cudaMemcpyAsync(e->d_cache, d_adj, e->m * sizeof(int), cudaMemcpyDeviceToDevice, e->s_main));
    hub_encode(e, 0, e->m, e->s_main);
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    EX_CUDA(cudaGetLastError());
    e->hubv_stale = true;
    std::fill(e->loaded.begin(), e->loaded.end(), 1);
    return EXCENT_OK;
}

extern "C" int excent_engine_reserve_cache(excent_engine* e, unsigned long long edges) {
    EX_CHECK_ARG(e && edges <= e->m, "bad cache size");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    EX_CUDA(cudaDeviceSynchronize());
    if (e->d_cache) { cudaFree(e->d_cache); e->d_cache = nullptr; e->cache_edges = 0; }
    e->hub_k = 0;   // a fresh cache holds plain ids
    free_host_cache(e);
    if (edges == 0) return EXCENT_OK;
    // 4 entries of padding: a bulk copy of a stretch rounds its end up to 16 bytes
    if (cudaMalloc((void**)&e->d_cache, (edges + 4) * sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        e->d_cache = nullptr;
        EX_FAIL(EXCENT_ERR_NOMEM, "edge cache of %llu edges does not fit", edges);
    }
    e->cache_edges = edges;
    std::fill(e->loaded.begin(), e->loaded.end(), 0);
    return EXCENT_OK;
}

extern "C" int excent_engine_load_cache(excent_engine* e, unsigned long long e0, unsigned long long e1,
                                        const int32_t* edges) {
    EX_CHECK_ARG(e && edges && e0 <= e1 && e1 <= e->cache_edges, "edges [%llu, %llu) outside the cache", e0, e1);
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaMemcpyAsync(e->d_cache + e0, edges, (e1 - e0) * sizeof(int), cudaMemcpyHostToDevice, e->s_main));
    hub_encode(e, e0, e1, e->s_main);
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    EX_CUDA(cudaGetLastError());
    for (int c = 0; c < e->nc; c++) if (e->ce[c] >= e0 && e->ce[c + 1] <= e1) e->loaded[c] = 1;
    return EXCENT_OK;
}

extern "C" int excent_engine_set_loaded(excent_engine* e, int c, int loaded) {
    EX_CHECK_ARG(e && c >= 0 && c < e->nc, "bad chunk");
    EX_CHECK_ARG(!loaded || e->ce[c + 1] <= e->cache_edges, "chunk %d is not inside the edge cache", c);
    e->loaded[c] = loaded ? 1 : 0;
    return EXCENT_OK;
}

extern "C" int excent_engine_trace(excent_engine* e, int enable) {
    EX_CHECK_ARG(e, "null engine");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    if (enable && !e->d_trace) EX_ALLOC(e->d_trace, (size_t)e->n * sizeof(uint16_t));
    e->trace_on = enable != 0;
    if (e->d_trace) EX_CUDA(cudaMemset(e->d_trace, 0, (size_t)e->n * sizeof(uint16_t)));
    return EXCENT_OK;
}

extern "C" int excent_engine_read_trace(excent_engine* e, uint16_t* out) {
    EX_CHECK_ARG(e && out && e->d_trace, "trace not enabled");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    EX_CUDA(cudaMemcpy(out, e->d_trace, (size_t)e->n * sizeof(uint16_t), cudaMemcpyDeviceToHost));
    return EXCENT_OK;
}

static int reset_counters(excent_engine* e) {
    EX_CUDA(cudaMemsetAsync(e->d_ctrl, 0, sizeof(Ctrl), e->s_main));
    EX_CUDA(cudaMemsetAsync(e->d_queue, 0, 3 * sizeof(PushQueue), e->s_main));
    EX_CUDA(cudaMemsetAsync(e->d_cnt, 0, 2 * (size_t)e->nc * sizeof(ull), e->s_main));
    if (e->d_trace && e->trace_on) EX_CUDA(cudaMemsetAsync(e->d_trace, 0, (size_t)e->n * sizeof(uint16_t), e->s_main));
    e->hot_skip = false;
    e->n_list = e->n_range = 0;
    return EXCENT_OK;
}

static int init_state(excent_engine* e) {
    const excent_measures& ms = e->meas;
    // The reference passes lambda1 to k_init as a float (src/excent.cu:41, 372);
    // EXCENT_EV_INIT_FP64 keeps the FP64 value.
    const double lam = (ms.flags & EXCENT_EV_INIT_FP64) ? ms.lambda : (double)(float)ms.lambda;
    const int g = e->sms * 8;
    if (e->L == 1)
        k_init<1><<<g, BLOCK, 0, e->s_main>>>(e->n, e->d_idx, (float*)e->d_x, (float*)e->d_r, e->nm,
                                               ms.kind[0], 0, 0, (float)ms.beta, lam);
    else
        k_init<4><<<g, BLOCK, 0, e->s_main>>>(e->n, e->d_idx, (float4*)e->d_x, (float4*)e->d_r, e->nm,
                                               ms.kind[0], ms.kind[1], ms.kind[2], (float)ms.beta, lam);
    e->launches++;
    EX_CUDA(cudaGetLastError());
    return reset_counters(e);
}

extern "C" int excent_engine_init(excent_engine* e) {
    EX_CHECK_ARG(e, "null engine");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_TRY(init_state(e));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    return EXCENT_OK;
}

static SnapArgs snap_args(excent_engine* e, bool use_hot) {
    SnapArgs a{};
    a.n = e->n; a.nc = e->nc; a.words = (int)(((size_t)e->n + 31) / 32); a.groups_per_warp = e->groups_per_warp;
    a.r = e->d_r; a.M = e->M; a.idx = e->d_idx; a.cv0 = e->d_cv0;
    a.v1 = e->ev_proj ? e->d_v1 : nullptr;
    a.ev = e->ev_index;
    a.ev_skip = e->ev_skip;
    a.hot = use_hot ? e->d_hot : nullptr;
    a.bitmap = e->d_bitmap; a.cnt = e->d_cnt; a.list = e->d_list;
    a.trace = e->trace_on ? e->d_trace : nullptr;
    a.ctrl = e->d_ctrl;
    return a;
}

static void launch_snapshot(excent_engine* e, bool use_hot, cudaStream_t st) {
    SnapArgs a = snap_args(e, use_hot);
    if (e->L == 1) k_snapshot<1><<<e->grid_snap, BLOCK, 0, st>>>(a);
    else k_snapshot<4><<<e->grid_snap, BLOCK, 0, st>>>(a);
    e->launches++;
}

extern "C" int excent_engine_snapshot(excent_engine* e, int use_hot, unsigned long long* cnt,
                                      unsigned long long* hotpend, double* rsum) {
    EX_CHECK_ARG(e, "null engine");
    EX_CHECK_ARG(!use_hot || e->d_hot, "hot snapshot without a hot cache");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaMemsetAsync(e->d_cnt, 0, 2 * (size_t)e->nc * sizeof(ull), e->s_main));
    EX_CUDA(cudaMemsetAsync(&e->d_ctrl->hotpend, 0, sizeof(ull), e->s_main));
    EX_CUDA(cudaMemsetAsync(e->d_ctrl->rsum, 0, sizeof(double) * MAXM, e->s_main));
    e->hot_skip = use_hot != 0;
    launch_snapshot(e, use_hot != 0, e->s_main);
    EX_CUDA(cudaGetLastError());
    EX_CUDA(cudaMemcpyAsync(e->h_cnt, e->d_cnt, 2 * (size_t)e->nc * sizeof(ull), cudaMemcpyDeviceToHost, e->s_main));
    EX_CUDA(cudaMemcpyAsync(e->h_ctrl, e->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, e->s_main));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    if (e->ev_proj) {   // next snapshot removes the component measured by this one
        Ctrl* hc = e->h_ctrl;
        hc->ev_corr = hc->ev_dot;
        hc->ev_dot = 0;
        EX_CUDA(cudaMemcpyAsync(&e->d_ctrl->ev_dot, &hc->ev_dot, 2 * sizeof(double), cudaMemcpyHostToDevice, e->s_main));
        EX_CUDA(cudaStreamSynchronize(e->s_main));
    }
    if (cnt) memcpy(cnt, e->h_cnt, 2 * (size_t)e->nc * sizeof(ull));
    if (hotpend) *hotpend = e->h_ctrl->hotpend;
    if (rsum) for (int k = 0; k < e->nm; k++) rsum[k] = e->h_ctrl->rsum[k];
    return EXCENT_OK;
}

extern "C" int excent_engine_bitmap(excent_engine* e, uint32_t* words) {
    EX_CHECK_ARG(e && words, "null argument");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    EX_CUDA(cudaMemcpy(words, e->d_bitmap, (((size_t)e->n + 31) / 32) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return EXCENT_OK;
}

extern "C" int excent_engine_chunk_list(excent_engine* e, int c, int32_t* ids, unsigned int* k) {
    EX_CHECK_ARG(e && ids && k && c >= 0 && c < e->nc, "bad argument");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    ull cnt = 0;
    EX_CUDA(cudaMemcpy(&cnt, e->d_cnt + 2 * c, sizeof(ull), cudaMemcpyDeviceToHost));
    *k = (unsigned)cnt;
    if (cnt) EX_CUDA(cudaMemcpy(ids, e->d_list + e->cv0[c], cnt * sizeof(int), cudaMemcpyDeviceToHost));
    return EXCENT_OK;
}

static PushArgs push_args(excent_engine* e, int q) {
    PushArgs a{};
    a.x = e->d_x; a.r = e->d_r; a.M = e->M; a.idx = e->d_idx; a.hot = nullptr;
    a.nc = e->nc; a.cv0 = e->d_cv0; a.wt_type = e->d_wt_type; a.wt_prefix = e->d_wt_prefix; a.list = e->d_list;
    a.cache = e->d_cache;
    a.hids = e->d_hids; a.hoff = e->d_hoff; a.hedges = e->d_hedges; a.hlist = e->d_hlist;
    a.hubq = e->d_hubq[q]; a.hub_cap = e->hub_cap[q]; a.q = e->d_queue + q; a.ctrl = e->d_ctrl;
    a.hub_id = e->d_hub_id; a.hub_k = e->hub_k;
    a.hubv = e->d_hubv; a.hubv_cnt = e->d_hubv_cnt; a.lists = LISTS_ALL; a.chunk = -1; a.stage = 0;
    a.claim_tiles = e->claim_tiles;
    a.hcache = nullptr; a.cache_edges = e->cache_edges;
    a.hcache = e->d_hcache;
    return a;
}

// One push launch: its work queue zeroed, then the kernel (which scatters its
// own long-list segments).
template <int SRC>
static void launch_push(excent_engine* e, const PushArgs& a, int grid, cudaStream_t st) {
    cudaMemsetAsync(a.q, 0, sizeof(PushQueue), st);
    // a launch of short lists only queues no segments: no k_segments after it
    const bool segs = a.lists != LISTS_SHORT;
    if (e->L == 1) {
        k_push<1, SRC><<<grid, BLOCK, hub_smem(e), st>>>(a);
        if (segs) k_segments<1><<<e->grid_push, BLOCK, hub_smem(e), st>>>(e->d_r, a);
    } else {
        k_push<4, SRC><<<grid, BLOCK, hub_smem(e), st>>>(a);
        if (segs) k_segments<4><<<e->grid_push, BLOCK, hub_smem(e), st>>>(e->d_r, a);
    }
    e->launches += segs ? 2 : 1;
}

// A streamed or gathered chunk in the pass's high-degree order: with the long
// lists first (last), one launch takes only those, the next only the others,
// as the cached push sends its high-degree vertices first (last).
template <int SRC>
static void launch_ordered(excent_engine* e, PushArgs a, int grid, cudaStream_t st) {
    const int order = order_of(e);
    if (order != 0) {
        const bool long_first = order != 2;
        a.lists = long_first ? LISTS_LONG : LISTS_SHORT;
        launch_push<SRC>(e, a, grid, st);
        a.lists = long_first ? LISTS_SHORT : LISTS_LONG;
    }
    launch_push<SRC>(e, a, grid, st);
}

static int grid_for(excent_engine* e, ull items) {
    const ull warps = (items + 31) / 32;
    const ull blocks = (warps + BLOCK / 32 - 1) / (BLOCK / 32);
    return (int)std::max<ull>(1, std::min<ull>(blocks, (ull)e->grid_push));
}

extern "C" int excent_engine_push_cached(excent_engine* e, const unsigned char* mode, const unsigned long long* cnt,
                                         double list_frac) {
    EX_CHECK_ARG(e && mode && cnt, "null argument");
    EX_CHECK_ARG(e->d_cache, "no edge cache");
    EX_CUDA(cudaSetDevice(e->dev));
    unsigned total = 0;
    e->h_wt_prefix[0] = 0;
    for (int c = 0; c < e->nc; c++) {
        uint8_t ty = WT_NONE;
        unsigned items = 0;
        if (mode[c] == 1 && cnt[2 * c] > 0) {
            EX_CHECK_ARG(e->ce[c + 1] <= e->cache_edges, "chunk %d is not in the edge cache", c);
            const int nv = (c + 1 < e->nc ? e->cv0[c + 1] : e->n) - e->cv0[c];
            if ((double)cnt[2 * c] < list_frac * nv) { ty = WT_LIST; items = (unsigned)cnt[2 * c]; e->n_list++; }
            else { ty = WT_RANGE; items = (unsigned)nv; e->n_range++; }
        }
        e->h_wt_type[c] = ty;
        total += items;
        e->h_wt_prefix[c + 1] = total;
    }
    if (total == 0) return EXCENT_OK;
    EX_CUDA(cudaMemcpyAsync(e->d_wt_type, e->h_wt_type, e->nc, cudaMemcpyHostToDevice, e->s_main));
    EX_CUDA(cudaMemcpyAsync(e->d_wt_prefix, e->h_wt_prefix, ((size_t)e->nc + 1) * sizeof(unsigned),
                            cudaMemcpyHostToDevice, e->s_main));
    // a high-degree order needs every chunk with work in the cache (the hub list spans the graph);
    // the hub list is built before the push arguments are taken, which point at it
    bool all_cached = true;
    for (int c = 0; c < e->nc; c++) all_cached &= cnt[2 * c] == 0 || mode[c] == 1;
    int order = 0;
    if (order_of(e) == 3) order = 3;
    else if (all_cached && order_of(e) && !sweep_of(e)) {
        EX_TRY(ensure_hubv(e));
        order = effective_order(e);
    }
    PushArgs a = push_args(e, 0);
    a.hot = e->hot_skip ? e->d_hot : nullptr;
    if (order == 1) launch_push<SRC_HUBS>(e, a, e->grid_push, e->s_main);
    a.lists = order == 1 || order == 2 ? LISTS_SHORT : LISTS_ALL;   // the long lists go by SRC_HUBS
    // order 3: each launch's long lists first, then its short ones
    auto table = [&](unsigned items) {
        if (order == 3) {
            a.lists = LISTS_LONG;
            launch_push<SRC_TABLE>(e, a, grid_for(e, items), e->s_main);
            a.lists = LISTS_SHORT;
        }
        launch_push<SRC_TABLE>(e, a, grid_for(e, items), e->s_main);
    };
    ull demand = 0;
    for (int c = 0; c < e->nc; c++) demand += cnt[2 * c + 1];
    if (sweep_of(e) && demand >= sweep_min_entries(e)) {   // one launch per chunk, in chunk order
        for (int c = 0; c < e->nc; c++) {
            const unsigned items = e->h_wt_prefix[c + 1] - e->h_wt_prefix[c];
            if (!items) continue;
            a.chunk = c;
            table(items);
        }
    } else {
        table(total);
    }
    a.lists = LISTS_ALL;
    if (order == 2) launch_push<SRC_HUBS>(e, a, e->grid_push, e->s_main);
    EX_CUDA(cudaGetLastError());
    return EXCENT_OK;
}

extern "C" int excent_engine_slots_create(excent_engine* e, unsigned long long max_chunk_edges, int max_chunk_verts,
                                          int zero_copy) {
    EX_CHECK_ARG(e && max_chunk_verts >= 1, "bad argument");
    EX_CHECK_ARG(!e->slots_ok, "slots already created");
    EX_CUDA(cudaSetDevice(e->dev));
    e->zc = zero_copy != 0;
    for (Slot& s : e->slot) {
        const size_t eb = (std::max<ull>(max_chunk_edges, 1) + 4) * sizeof(int);   // + padding for bulk copies
        const size_t vb = (size_t)max_chunk_verts * sizeof(int), ob = ((size_t)max_chunk_verts + 1) * sizeof(ull);
        if (e->zc) {
            if (cudaHostAlloc((void**)&s.h_edges, eb, cudaHostAllocMapped) != cudaSuccess ||
                cudaHostAlloc((void**)&s.h_vids, vb, cudaHostAllocMapped) != cudaSuccess ||
                cudaHostAlloc((void**)&s.h_off, ob, cudaHostAllocMapped) != cudaSuccess) {
                cudaGetLastError();
                EX_FAIL(EXCENT_ERR_NOMEM, "mapped staging allocation failed");
            }
            EX_CUDA(cudaHostGetDevicePointer((void**)&s.d_edges, s.h_edges, 0));
            EX_CUDA(cudaHostGetDevicePointer((void**)&s.d_vids, s.h_vids, 0));
            EX_CUDA(cudaHostGetDevicePointer((void**)&s.d_off, s.h_off, 0));
        } else {
            EX_HALLOC(s.h_edges, eb);
            EX_HALLOC(s.h_vids, vb);
            EX_HALLOC(s.h_off, ob);
            EX_ALLOC(s.d_edges, eb);
            EX_ALLOC(s.d_vids, vb);
            EX_ALLOC(s.d_off, ob);
        }
        EX_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
        EX_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
    }
    for (int q = 1; q < 3; q++) {
        const ull me = std::max<ull>(max_chunk_edges, 1);
        e->hub_cap[q] = me / HUB_SEG + me / HUB_MIN + 64;
        EX_ALLOC(e->d_hubq[q], e->hub_cap[q] * sizeof(HubSeg));
        EX_CUDA(cudaMemset(e->d_hubq[q], 0, e->hub_cap[q] * sizeof(HubSeg)));
    }
    e->max_chunk_edges = std::max<ull>(e->max_chunk_edges, max_chunk_edges);
    e->slots_ok = true;
    return EXCENT_OK;
}

extern "C" int excent_engine_slot_buffers(excent_engine* e, int s, int32_t** edges, int32_t** vids,
                                          unsigned long long** off) {
    EX_CHECK_ARG(e && e->slots_ok && (s == 0 || s == 1), "no such slot");
    if (edges) *edges = e->slot[s].h_edges;
    if (vids) *vids = e->slot[s].h_vids;
    if (off) *off = e->slot[s].h_off;
    return EXCENT_OK;
}

extern "C" int excent_engine_slot_wait(excent_engine* e, int s) {
    EX_CHECK_ARG(e && e->slots_ok && (s == 0 || s == 1), "no such slot");
    EX_CUDA(cudaSetDevice(e->dev));
    Slot& sl = e->slot[s];
    if (sl.busy) { EX_CUDA(cudaEventSynchronize(sl.done)); sl.busy = false; }
    return EXCENT_OK;
}

extern "C" int excent_engine_push_stream(excent_engine* e, int s, int c, const unsigned long long* cnt,
                                         double list_frac, int cache_fill, int hlo, int hhi) {
    EX_CHECK_ARG(e && e->slots_ok && (s == 0 || s == 1) && cnt, "bad argument");
    EX_CHECK_ARG(c >= 0 && c < e->nc, "bad chunk %d", c);
    EX_CUDA(cudaSetDevice(e->dev));
    Slot& sl = e->slot[s];
    const ull e0 = e->ce[c], e1 = e->ce[c + 1], ne = e1 - e0;
    EX_CHECK_ARG(ne <= e->max_chunk_edges, "chunk %d larger than the slots", c);
    const bool to_cache = cache_fill && e->d_cache && e1 <= e->cache_edges;
    int* dst = to_cache ? e->d_cache + e0 : sl.d_edges;
    if (!e->zc) { if (ne) EX_CUDA(cudaMemcpyAsync(dst, sl.h_edges, ne * sizeof(int), cudaMemcpyHostToDevice, sl.st)); }
    else if (to_cache && ne) EX_CUDA(cudaMemcpyAsync(dst, sl.d_edges, ne * sizeof(int), cudaMemcpyDeviceToDevice, sl.st));
    if (e->d_hedges && hhi > hlo) {
        const unsigned grid = (unsigned)(((long long)(hhi - hlo) * 32 + BLOCK - 1) / BLOCK);
        k_fill_hot<<<grid, BLOCK, 0, sl.st>>>(hlo, hhi, e->d_hids, e->d_hoff, e->d_idx, e0, dst, e->d_hedges);
        e->launches++;
    }
    if (to_cache) hub_encode(e, e0, e1, sl.st);   // the cached copy carries the hub-target slots
    const int v0 = e->cv0[c], nv = (c + 1 < e->nc ? e->cv0[c + 1] : e->n) - v0;
    const ull k = cnt[2 * c];
    PushArgs a = push_args(e, 1 + s);
    a.hot = e->hot_skip ? e->d_hot : nullptr;
    a.cv_0 = v0; a.ebase = dst; a.e0 = e0;
    a.stage = e->zc ? 0 : 1;   // mapped host slots are read in place
    if ((double)k < list_frac * nv) { a.ctype = WT_LIST; a.ccount = (unsigned)k; e->n_list++; }
    else { a.ctype = WT_RANGE; a.ccount = (unsigned)nv; e->n_range++; }
    if (a.ccount) launch_ordered<SRC_CHUNK>(e, a, grid_for(e, a.ccount), sl.st);
    EX_CUDA(cudaGetLastError());
    if (to_cache) e->loaded[c] = 1;
    EX_CUDA(cudaEventRecord(sl.done, sl.st));
    sl.busy = true;
    return EXCENT_OK;
}

extern "C" int excent_engine_push_gather(excent_engine* e, int s, int k, unsigned long long ne) {
    EX_CHECK_ARG(e && e->slots_ok && (s == 0 || s == 1), "no such slot");
    EX_CHECK_ARG(k >= 0 && k <= e->max_chunk_verts && ne <= e->max_chunk_edges, "gather larger than the slots");
    EX_CUDA(cudaSetDevice(e->dev));
    Slot& sl = e->slot[s];
    if (!e->zc) {
        EX_CUDA(cudaMemcpyAsync(sl.d_vids, sl.h_vids, (size_t)k * sizeof(int), cudaMemcpyHostToDevice, sl.st));
        EX_CUDA(cudaMemcpyAsync(sl.d_off, sl.h_off, ((size_t)k + 1) * sizeof(ull), cudaMemcpyHostToDevice, sl.st));
        if (ne) EX_CUDA(cudaMemcpyAsync(sl.d_edges, sl.h_edges, ne * sizeof(int), cudaMemcpyHostToDevice, sl.st));
    }
    if (k) {
        PushArgs a = push_args(e, 1 + s);
        a.vids = sl.d_vids; a.off = sl.d_off; a.gedges = sl.d_edges; a.gk = (unsigned)k;
        a.stage = e->zc ? 0 : 1;
        launch_ordered<SRC_GATHER>(e, a, grid_for(e, (ull)k), sl.st);
        EX_CUDA(cudaGetLastError());
    }
    EX_CUDA(cudaEventRecord(sl.done, sl.st));
    sl.busy = true;
    return EXCENT_OK;
}

extern "C" int excent_engine_hot_setup(excent_engine* e, int nh, const int32_t* ids, const unsigned long long* off,
                                       const uint32_t* hot_bitmap) {
    EX_CHECK_ARG(e && nh >= 1 && ids && off && hot_bitmap, "bad argument");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CHECK_ARG(!e->d_hedges, "hot cache already set up");
    invalidate_graph(e);
    const size_t words = ((size_t)e->n + 31) / 32;
    const ull he = off[nh];
    bool ok = cudaMalloc((void**)&e->d_hedges, std::max<ull>(he, 1) * sizeof(int)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&e->d_hids, (size_t)nh * sizeof(int)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&e->d_hoff, ((size_t)nh + 1) * sizeof(ull)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&e->d_hot, words * sizeof(uint32_t)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&e->d_hlist, (size_t)nh * sizeof(int)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        void* ps[] = {e->d_hedges, e->d_hids, e->d_hoff, e->d_hot, e->d_hlist};
        for (void* p : ps) if (p) cudaFree(p);
        e->d_hedges = nullptr; e->d_hids = nullptr; e->d_hoff = nullptr; e->d_hot = nullptr; e->d_hlist = nullptr;
        e->nh = 0;
        EX_FAIL(EXCENT_ERR_NOMEM, "degree cache: could not allocate %d lists (%.2f GB)", nh, he * 4.0 / 1e9);
    }
    EX_CUDA(cudaMemcpy(e->d_hids, ids, (size_t)nh * sizeof(int), cudaMemcpyHostToDevice));
    EX_CUDA(cudaMemcpy(e->d_hoff, off, ((size_t)nh + 1) * sizeof(ull), cudaMemcpyHostToDevice));
    EX_CUDA(cudaMemcpy(e->d_hot, hot_bitmap, words * sizeof(uint32_t), cudaMemcpyHostToDevice));
    e->nh = nh;
    return EXCENT_OK;
}

extern "C" int excent_engine_push_hot(excent_engine* e, int lo, int hi, int after_slots) {
    EX_CHECK_ARG(e && e->d_hedges, "no hot cache");
    EX_CHECK_ARG(lo >= 0 && lo <= hi && hi <= e->nh, "bad hot range");
    EX_CUDA(cudaSetDevice(e->dev));
    if (after_slots && e->slots_ok)
        for (Slot& s : e->slot) if (s.busy) EX_CUDA(cudaStreamWaitEvent(e->s_main, s.done, 0));
    if (hi == lo) return EXCENT_OK;
    EX_CUDA(cudaMemsetAsync(&e->d_ctrl->hcount, 0, sizeof(unsigned), e->s_main));
    const int grid = (int)std::min<long long>(((long long)(hi - lo) + BLOCK - 1) / BLOCK, (long long)e->sms * 8);
    if (e->L == 1) k_compact_hot<1><<<grid, BLOCK, 0, e->s_main>>>(lo, hi, e->d_hids, e->d_r, e->M, e->d_hlist, e->d_ctrl);
    else k_compact_hot<4><<<grid, BLOCK, 0, e->s_main>>>(lo, hi, e->d_hids, e->d_r, e->M, e->d_hlist, e->d_ctrl);
    e->launches++;
    PushArgs a = push_args(e, 0);
    launch_push<SRC_HOT>(e, a, grid_for(e, (ull)(hi - lo)), e->s_main);
    EX_CUDA(cudaGetLastError());
    return EXCENT_OK;
}

extern "C" int excent_engine_hot_pending(excent_engine* e, int lo, int hi, int32_t* out, unsigned int* k) {
    EX_CHECK_ARG(e && e->d_hedges && out && k, "no hot cache or null argument");
    EX_CHECK_ARG(lo >= 0 && lo <= hi && hi <= e->nh, "bad hot range");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaMemsetAsync(&e->d_ctrl->hcount, 0, sizeof(unsigned), e->s_main));
    if (hi > lo) {
        const int grid = (int)std::min<long long>(((long long)(hi - lo) + BLOCK - 1) / BLOCK, (long long)e->sms * 8);
        if (e->L == 1) k_compact_hot<1><<<grid, BLOCK, 0, e->s_main>>>(lo, hi, e->d_hids, e->d_r, e->M, e->d_hlist, e->d_ctrl);
        else k_compact_hot<4><<<grid, BLOCK, 0, e->s_main>>>(lo, hi, e->d_hids, e->d_r, e->M, e->d_hlist, e->d_ctrl);
        e->launches++;
        EX_CUDA(cudaGetLastError());
    }
    unsigned cnt = 0;
    EX_CUDA(cudaMemcpyAsync(&cnt, &e->d_ctrl->hcount, sizeof(unsigned), cudaMemcpyDeviceToHost, e->s_main));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    *k = cnt;
    if (cnt) EX_CUDA(cudaMemcpy(out, e->d_hlist, (size_t)cnt * sizeof(int), cudaMemcpyDeviceToHost));
    return EXCENT_OK;
}

extern "C" int excent_engine_hot_edges(excent_engine* e, int32_t* out) {
    EX_CHECK_ARG(e && e->d_hedges && out, "no hot cache or null argument");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaDeviceSynchronize());
    ull he = 0;
    EX_CUDA(cudaMemcpy(&he, e->d_hoff + e->nh, sizeof(ull), cudaMemcpyDeviceToHost));
    if (he) EX_CUDA(cudaMemcpy(out, e->d_hedges, he * sizeof(int), cudaMemcpyDeviceToHost));
    return EXCENT_OK;
}

extern "C" int excent_engine_sync(excent_engine* e) {
    EX_CHECK_ARG(e, "null engine");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    if (e->slots_ok) for (Slot& s : e->slot) { EX_CUDA(cudaStreamSynchronize(s.st)); s.busy = false; }
    int err = 0;
    EX_CUDA(cudaMemcpy(&err, &e->d_ctrl->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) scrub_queues(e);
    if (err) EX_FAIL(EXCENT_ERR_STATE, "%s", ctrl_error(err));
    return EXCENT_OK;
}

// Open an IF node on the stream being captured (condition `h`, set per pass
// by k_plan) and start capturing its body on `body`; close_if ends the body.
static cudaError_t open_if(cudaStream_t st, cudaStream_t body, cudaGraphConditionalHandle* h) {
    cudaStreamCaptureStatus status;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaError_t rc = cudaStreamGetCaptureInfo(st, &status, nullptr, &g, &deps, &nd);
    if (rc != cudaSuccess) return rc;
    if (status != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
    rc = cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault);
    if (rc != cudaSuccess) return rc;
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = *h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    rc = cudaGraphAddNode(&node, g, deps, nd, &cp);
    if (rc != cudaSuccess) return rc;
    rc = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (rc != cudaSuccess) return rc;
    return cudaStreamBeginCaptureToGraph(body, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeRelaxed);
}
static cudaError_t close_if(cudaStream_t body) {
    cudaGraph_t g = nullptr;
    return cudaStreamEndCapture(body, &g);
}

// Kernels of one pass outside the per-chunk launches of a chunk sweep, and per
// chunk launch (for the launch count of a graph solve).
static void pass_kernels(const excent_engine* e, int order, ull* fixed, ull* per_chunk) {
    // kernels of one table push: with segments 2, short lists only 1 (no k_segments)
    const ull table = order == 3 ? 3 : (order == 1 || order == 2 ? 1 : 2);
    *fixed = 2 + (order == 1 || order == 2 ? 2 : 0) + (sweep_of(e) ? 0 : table);
    *per_chunk = sweep_of(e) ? table : 0;
}


// One pass of the device solve: snapshot -> plan -> push -> hub segments.
// With ev, events are recorded between the kernels. chunk_body (a second
// stream) is given while the pass is captured into a graph with a chunk
// sweep: each chunk's launches then sit in an IF node that k_plan switches
// on for chunks with something to push in a sweeping pass, and the
// whole-table launch sits in one more IF node, switched on in the other
// passes; e->h_chunk_if receives the nc + 1 handles.
static void enqueue_plan(excent_engine* e, double list_frac, int max_passes, cudaGraphConditionalHandle cond,
                         int use_cond, cudaStream_t st, cudaEvent_t* ev, bool use_if) {
    if (ev) cudaEventRecord(ev[0], st);
    launch_snapshot(e, false, st);
    if (ev) cudaEventRecord(ev[1], st);
    k_plan<<<1, 1024, 0, st>>>(e->nc, e->d_cv0, e->n, e->d_cnt, e->d_cmode, list_frac, max_passes, e->d_wt_type,
                               e->d_wt_prefix, e->d_ctrl, e->d_queue, e->d_log, e->log_cap, cond, use_cond,
                               use_if ? e->d_chunk_if : nullptr, sweep_of(e) ? 1 : 0, sweep_min_entries(e));
    e->launches++;
    if (ev) cudaEventRecord(ev[2], st);
}

// The pushes of a pass. sweep_pass: whether k_plan chose a chunk-by-chunk pass
// (known to the host-driven loop, which reads it back first); ignored while
// capturing with IF nodes, which hold both forms.
static cudaError_t enqueue_push(excent_engine* e, cudaStream_t st, cudaEvent_t* ev, cudaStream_t chunk_body,
                                bool sweep_pass) {
    PushArgs a = push_args(e, 0);
    const bool use_if = chunk_body && sweep_of(e);
    // high-degree order: 1 = the lists longer than HUB_MIN first, so their (large) share of the
    // pass's residual reaches every other vertex before that vertex is taken; 2 = last, so they
    // collect the pass's residual and push it once; 0 = in table order with the rest
    const int order = effective_order(e);
    auto table1 = [&](cudaStream_t s) { launch_push<SRC_TABLE>(e, a, e->grid_push, s); };
    // order 3: each launch's long lists first, then its short ones
    auto table = [&](cudaStream_t s) {
        if (order == 3) {
            a.lists = LISTS_LONG;
            table1(s);
            a.lists = LISTS_SHORT;
            table1(s);
            a.lists = LISTS_ALL;
        } else {
            table1(s);
        }
    };
    auto hub_phase = [&]() {
        cudaMemsetAsync(a.q, 0, sizeof(PushQueue), st);
        if (e->L == 1) {
            k_push<1, SRC_HUBS><<<e->grid_push, BLOCK, hub_smem(e), st>>>(a);
            k_segments<1><<<e->grid_push, BLOCK, hub_smem(e), st>>>(e->d_r, a);
        } else {
            k_push<4, SRC_HUBS><<<e->grid_push, BLOCK, hub_smem(e), st>>>(a);
            k_segments<4><<<e->grid_push, BLOCK, hub_smem(e), st>>>(e->d_r, a);
        }
        e->launches += 2;
    };
    // one launch under an IF node (c = -1: the whole table)
    auto guarded = [&](int c) -> cudaError_t {
        a.chunk = c;
        cudaError_t rc = open_if(st, chunk_body, &e->h_chunk_if[c >= 0 ? c : e->nc]);
        if (rc != cudaSuccess) return rc;
        table(chunk_body);
        rc = close_if(chunk_body);
        a.chunk = -1;
        return rc;
    };
    if (order == 1) hub_phase();
    a.lists = order == 1 || order == 2 ? LISTS_SHORT : LISTS_ALL;   // the table push skips the high-degree vertices
    if (use_if) {
        // chunk by chunk: each chunk's push (with its long lists) completes before the next
        // chunk's vertices are taken, so they see everything pushed so far; or the whole table
        for (int c = 0; c < e->nc; c++) {
            const cudaError_t rc = guarded(c);
            if (rc != cudaSuccess) return rc;
        }
        const cudaError_t rc = guarded(-1);
        if (rc != cudaSuccess) return rc;
    } else if (sweep_of(e) && sweep_pass) {
        for (int c = 0; c < e->nc; c++) {
            a.chunk = c;
            table(st);
        }
        a.chunk = -1;
    } else {
        table(st);
    }
    a.lists = LISTS_ALL;
    if (ev) cudaEventRecord(ev[3], st);
    if (order == 2) hub_phase();
    if (ev) cudaEventRecord(ev[4], st);
    return cudaGetLastError();
}

static cudaError_t enqueue_pass(excent_engine* e, double list_frac, int max_passes, cudaGraphConditionalHandle cond,
                                int use_cond, cudaStream_t st, cudaStream_t chunk_body) {
    enqueue_plan(e, list_frac, max_passes, cond, use_cond, st, nullptr, chunk_body && sweep_of(e));
    return enqueue_push(e, st, nullptr, chunk_body, true);
}

static int build_graph(excent_engine* e, double list_frac, int max_passes) {
    if (e->gexec && e->graph_max_passes == max_passes && e->graph_list_frac == list_frac) return EXCENT_OK;
    invalidate_graph(e);
    if (sweep_of(e) && !e->d_chunk_if)
        EX_ALLOC(e->d_chunk_if, (size_t)(e->nc + 1) * sizeof(cudaGraphConditionalHandle));
    e->h_chunk_if.assign(e->nc + 1, 0);
    cudaGraph_t g;
    EX_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    EX_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    EX_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    // capture one pass into the body graph
    cudaStream_t cs, cb;
    EX_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    EX_CUDA(cudaStreamCreateWithFlags(&cb, cudaStreamNonBlocking));
    EX_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const ull before = e->launches;
    const cudaError_t pe = enqueue_pass(e, list_frac, max_passes, h, 1, cs, sweep_of(e) ? cb : nullptr);
    e->launches = before;
    cudaGraph_t captured;
    const cudaError_t ce = cudaStreamEndCapture(cs, &captured);
    cudaStreamDestroy(cs);
    cudaStreamDestroy(cb);
    if (pe != cudaSuccess || ce != cudaSuccess) {
        cudaGraphDestroy(g);
        cudaGetLastError();
        EX_CUDA(pe != cudaSuccess ? pe : ce);
    }
    if (sweep_of(e))
        EX_CUDA(cudaMemcpy(e->d_chunk_if, e->h_chunk_if.data(), (size_t)(e->nc + 1) * sizeof(cudaGraphConditionalHandle),
                           cudaMemcpyHostToDevice));
    const cudaError_t ie = cudaGraphInstantiate(&e->gexec, g, 0);
    if (ie != cudaSuccess) { cudaGraphDestroy(g); e->gexec = nullptr; EX_CUDA(ie); }
    e->graph = g;
    e->graph_max_passes = max_passes;
    e->graph_list_frac = list_frac;
    return EXCENT_OK;
}

// After a device-side failure (a segment queue overflow, a bulk-copy wait that
// gave up): wait for the device, then clear the queue counters and the flag so
// the next solve starts clean.
static void scrub_queues(excent_engine* e) {
    cudaDeviceSynchronize();
    cudaMemset(e->d_queue, 0, 3 * sizeof(PushQueue));
    cudaMemset(&e->d_ctrl->err, 0, sizeof(int));
    cudaDeviceSynchronize();
}

static int solve_impl(excent_engine* e, double list_frac, int max_passes, int use_graph, bool init);

extern "C" int excent_engine_solve(excent_engine* e, double list_frac, int max_passes, int use_graph) {
    return solve_impl(e, list_frac, max_passes, use_graph, true);
}

extern "C" int excent_engine_resume(excent_engine* e, double list_frac, int max_passes, int use_graph) {
    return solve_impl(e, list_frac, max_passes, use_graph, false);
}

__global__ void k_seed(int k, const int* vids, const float* vals, float* r) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) atomicAdd(&r[vids[i]], vals[i]);
}

extern "C" int excent_engine_seed(excent_engine* e, int k, const int32_t* vids, const float* vals) {
    EX_CHECK_ARG(e && k >= 0 && (k == 0 || (vids && vals)), "bad argument");
    EX_CHECK_ARG(e->L == 1, "seeded solves need a single-measure engine");
    for (int i = 0; i < k; i++) EX_CHECK_ARG(vids[i] >= 0 && vids[i] < e->n, "seed vertex %d out of range", vids[i]);
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaMemsetAsync(e->d_x, 0, (size_t)e->n * sizeof(float), e->s_main));
    EX_CUDA(cudaMemsetAsync(e->d_r, 0, (size_t)e->n * sizeof(float), e->s_main));
    if (k) {
        // seed lists ride in the pending-list buffer (n ints), which the next snapshot rewrites
        EX_CHECK_ARG((size_t)k * 2 <= (size_t)e->n, "too many seeds (%d) for n = %d", k, e->n);
        EX_CUDA(cudaMemcpyAsync(e->d_list, vids, (size_t)k * sizeof(int), cudaMemcpyHostToDevice, e->s_main));
        EX_CUDA(cudaMemcpyAsync(e->d_list + k, vals, (size_t)k * sizeof(float), cudaMemcpyHostToDevice, e->s_main));
        k_seed<<<std::min(1024, (k + 255) / 256), 256, 0, e->s_main>>>(k, e->d_list, (const float*)(e->d_list + k),
                                                                       (float*)e->d_r);
        e->launches++;
        EX_CUDA(cudaGetLastError());
    }
    EX_TRY(reset_counters(e));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    return EXCENT_OK;
}

// The vertices whose lists are longer than HUB_MIN (for a high-degree order),
// listed once per graph; without room for the list the solve runs in table order.
static int effective_order(const excent_engine* e) {
    if (order_of(e) == 3) return 3;   // inside each launch: needs no high-degree list
    return order_of(e) && e->d_hubv && !e->hubv_stale ? order_of(e) : 0;
}

static int ensure_hubv(excent_engine* e) {
    if (e->hubv_stale) {
        // count the high-degree vertices, then list them in a buffer of that size
        if (!e->d_hubv_cnt) EX_ALLOC(e->d_hubv_cnt, sizeof(ull));
        EX_CUDA(cudaMemsetAsync(e->d_hubv_cnt, 0, sizeof(ull), e->s_main));
        k_hub_list<<<e->sms * 8, BLOCK, 0, e->s_main>>>(e->n, e->d_idx, nullptr, e->d_hubv_cnt);
        ull h = 0;
        EX_CUDA(cudaMemcpyAsync(&h, e->d_hubv_cnt, sizeof(ull), cudaMemcpyDeviceToHost, e->s_main));
        EX_CUDA(cudaStreamSynchronize(e->s_main));
        if (h > e->hubv_cap || !e->d_hubv) {
            invalidate_graph(e);
            if (e->d_hubv) cudaFree(e->d_hubv);
            e->d_hubv = nullptr;
            e->hubv_cap = 0;
            if (cudaMalloc((void**)&e->d_hubv, std::max<ull>(h, 1) * sizeof(int)) != cudaSuccess) {
                cudaGetLastError();   // no room: this solve runs in plain order
                e->d_hubv = nullptr;
            } else {
                e->hubv_cap = std::max<ull>(h, 1);
            }
        }
        if (e->d_hubv) {
            EX_CUDA(cudaMemsetAsync(e->d_hubv_cnt, 0, sizeof(ull), e->s_main));
            k_hub_list<<<e->sms * 8, BLOCK, 0, e->s_main>>>(e->n, e->d_idx, e->d_hubv, e->d_hubv_cnt);
            e->launches += 2;
            EX_CUDA(cudaGetLastError());
            e->hubv_stale = false;
        }
    }
    return EXCENT_OK;
}

static int solve_impl(excent_engine* e, double list_frac, int max_passes, int use_graph, bool init) {
    EX_CHECK_ARG(e, "null engine");
    EX_CHECK_ARG(max_passes >= 0 && max_passes < e->log_cap, "max_passes must be < %d", e->log_cap);
    for (int c = 0; c < e->nc; c++)
        EX_CHECK_ARG(e->loaded[c] || (e->d_hcache && e->ce[c] >= e->cache_edges),
                     "chunk %d is neither in the edge cache nor in the host cache", c);
    EX_CUDA(cudaSetDevice(e->dev));
    std::vector<uint8_t> cm(e->nc, 1);
    for (int c = 0; c < e->nc; c++)
        if (e->d_hcache && e->ce[c] >= e->cache_edges) cm[c] = 2;   // lists in host memory
    EX_CUDA(cudaMemcpy(e->d_cmode, cm.data(), e->nc, cudaMemcpyHostToDevice));
    if (init) EX_TRY(init_state(e));
    else EX_TRY(reset_counters(e));
    if (order_of(e) == 1 || order_of(e) == 2) EX_TRY(ensure_hubv(e));
    if (use_graph) {
        EX_TRY(build_graph(e, list_frac, max_passes));
        EX_CUDA(cudaGraphLaunch(e->gexec, e->s_main));
        EX_CUDA(cudaStreamSynchronize(e->s_main));
        EX_CUDA(cudaMemcpy(e->h_ctrl, e->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
        ull fixed = 0, per_chunk = 0;
        pass_kernels(e, effective_order(e), &fixed, &per_chunk);
        e->launches += fixed * (e->h_ctrl->pass + 1) + per_chunk * e->h_ctrl->chunk_runs;
    } else {
        // snapshot and plan, read the plan back (one sync per pass), then the pushes it chose
        for (int p = 0; p <= max_passes; p++) {
            cudaEvent_t* ev = e->prof ? e->ev : nullptr;
            enqueue_plan(e, list_frac, max_passes, 0, 0, e->s_main, ev, false);
            EX_CUDA(cudaMemcpyAsync(e->h_ctrl, e->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, e->s_main));
            EX_CUDA(cudaStreamSynchronize(e->s_main));
            if (e->h_ctrl->done) break;
            EX_CUDA(enqueue_push(e, e->s_main, ev, nullptr, e->h_ctrl->sweep_pass != 0));
            if (ev) {
                EX_CUDA(cudaStreamSynchronize(e->s_main));
                for (int k = 0; k < 4; k++) {
                    float ms = 0;
                    EX_CUDA(cudaEventElapsedTime(&ms, e->ev[k], e->ev[k + 1]));
                    e->prof_ms[k] += ms;
                }
                e->prof_passes++;
            }
        }
    }
    EX_CUDA(cudaGetLastError());
    if (e->h_ctrl->err) scrub_queues(e);
    if (e->h_ctrl->err) EX_FAIL(EXCENT_ERR_STATE, "%s", ctrl_error(e->h_ctrl->err));
    return EXCENT_OK;
}

extern "C" int excent_engine_stats(excent_engine* e, excent_stats* st, excent_pass_log* log, int cap) {
    EX_CHECK_ARG(e, "null engine");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaDeviceSynchronize());
    Ctrl c;
    EX_CUDA(cudaMemcpy(&c, e->d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
    const int np = std::min(c.pass, e->log_cap);
    std::vector<PassRec> recs(np);
    if (np) EX_CUDA(cudaMemcpy(recs.data(), e->d_log, np * sizeof(PassRec), cudaMemcpyDeviceToHost));
    if (st) {
        memset(st, 0, sizeof(*st));
        st->passes = c.pass;
        st->pushed = c.pushed;
        ull nl = 0, nr = 0;
        for (auto& r : recs) { nl += r.n_list; nr += r.n_range; }
        st->n_list = nl + e->n_list;
        st->n_range = nr + e->n_range;
        for (int k = 0; k < MAXM; k++) st->rsum[k] = c.rsum[k];
    }
    if (log) {
        for (int p = 0; p < np && p < cap; p++) {
            excent_pass_log& L = log[p];
            L.pending = recs[p].pending; L.demand = recs[p].demand; L.hot_pending = recs[p].hot_pending;
            L.pushed = (p + 1 < np ? recs[p + 1].pushed_before : c.pushed) - recs[p].pushed_before;
            L.lanes = (p + 1 < np ? recs[p + 1].lanes_before : c.lanes) - recs[p].lanes_before;
            L.taken = (p + 1 < np ? recs[p + 1].taken_before : c.taken) - recs[p].taken_before;
            for (int k = 0; k < MAXM; k++) L.rsum[k] = recs[p].rsum[k];
            L.n_list = recs[p].n_list; L.n_range = recs[p].n_range;
        }
    }
    return EXCENT_OK;
}

extern "C" int excent_engine_read(excent_engine* e, int i, int residual, float* out, unsigned long long v0,
                                  unsigned long long count) {
    EX_CHECK_ARG(e && out && i >= 0 && i < e->nm && v0 + count <= (ull)e->n, "bad argument");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaDeviceSynchronize());
    const void* src = residual ? e->d_r : e->d_x;
    if (e->L == 1) {
        EX_CUDA(cudaMemcpy(out, (const float*)src + v0, count * sizeof(float), cudaMemcpyDeviceToHost));
    } else {
        k_extract<<<e->sms * 8, BLOCK, 0, e->s_main>>>(e->n, (const float4*)src, i, e->d_tmp);
        e->launches++;
        EX_CUDA(cudaGetLastError());
        EX_CUDA(cudaMemcpyAsync(out, e->d_tmp + v0, count * sizeof(float), cudaMemcpyDeviceToHost, e->s_main));
        EX_CUDA(cudaStreamSynchronize(e->s_main));
    }
    return EXCENT_OK;
}

extern "C" int excent_engine_write(excent_engine* e, int i, const float* x, const float* r) {
    EX_CHECK_ARG(e && i >= 0 && i < e->nm, "bad argument");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaDeviceSynchronize());
    const float* srcs[2] = {x, r};
    void* dsts[2] = {e->d_x, e->d_r};
    for (int j = 0; j < 2; j++) {
        if (!srcs[j]) continue;
        if (e->L == 1) EX_CUDA(cudaMemcpy(dsts[j], srcs[j], (size_t)e->n * sizeof(float), cudaMemcpyHostToDevice));
        else {
            EX_CUDA(cudaMemcpy(e->d_tmp, srcs[j], (size_t)e->n * sizeof(float), cudaMemcpyHostToDevice));
            k_insert<<<e->sms * 8, BLOCK>>>(e->n, (float4*)dsts[j], i, e->d_tmp);
            e->launches++;
            EX_CUDA(cudaGetLastError());
            EX_CUDA(cudaDeviceSynchronize());
        }
    }
    return EXCENT_OK;
}

extern "C" int excent_device_info(int device, excent_device_info_t* out) {
    EX_CHECK_ARG(out, "null argument");
    EX_CUDA(cudaSetDevice(device));
    size_t f = 0, t = 0;
    EX_CUDA(cudaMemGetInfo(&f, &t));
    out->free_bytes = f;
    out->total_bytes = t;
    EX_CUDA(cudaDeviceGetAttribute(&out->integrated, cudaDevAttrIntegrated, device));
    EX_CUDA(cudaDeviceGetAttribute(&out->sms, cudaDevAttrMultiProcessorCount, device));
    EX_CUDA(cudaDeviceGetAttribute(&out->cc_major, cudaDevAttrComputeCapabilityMajor, device));
    EX_CUDA(cudaDeviceGetAttribute(&out->cc_minor, cudaDevAttrComputeCapabilityMinor, device));
    return EXCENT_OK;
}

extern "C" int excent_engine_set_hub_targets(excent_engine* e, int k) {
    EX_CHECK_ARG(e && k >= 0, "bad argument");
    const int kmax = e->L == 1 ? 32768 : 8192;   // 128 KiB of shared accumulators per block
    EX_CHECK_ARG(k <= kmax, "at most %d hub targets for this layout", kmax);
    EX_CHECK_ARG(k <= e->n, "more hub targets than vertices");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaDeviceSynchronize());
    invalidate_graph(e);
    if (e->hub_k && e->d_cache && e->cache_edges) {   // back to plain ids first (loaded chunks only)
        for (int c = 0; c < e->nc; c++) {
            if (!e->loaded[c] || e->ce[c + 1] > e->cache_edges || e->ce[c + 1] == e->ce[c]) continue;
            k_hub_decode<<<e->sms * 8, BLOCK, 0, e->s_main>>>(e->ce[c + 1] - e->ce[c], e->d_cache + e->ce[c],
                                                               e->d_hub_id, e->hub_k);
            e->launches++;
        }
        EX_CUDA(cudaStreamSynchronize(e->s_main));
        EX_CUDA(cudaGetLastError());
    }
    e->hub_k = 0;
    if (k > 0) {
        EX_CHECK_ARG(e->d_cache && e->cache_edges, "reserve the edge cache before choosing hub targets");
        std::vector<ull> idx((size_t)e->n + 1);
        EX_CUDA(cudaMemcpy(idx.data(), e->d_idx, idx.size() * sizeof(ull), cudaMemcpyDeviceToHost));
        std::vector<int> ids(e->n);
        for (int v = 0; v < e->n; v++) ids[v] = v;
        auto deg = [&](int v) { return idx[v + 1] - idx[v]; };
        std::nth_element(ids.begin(), ids.begin() + (k - 1), ids.end(), [&](int a, int b) {
            return deg(a) > deg(b) || (deg(a) == deg(b) && a < b);
        });
        ids.resize(k);
        std::sort(ids.begin(), ids.end());
        if (!e->d_hub_id) EX_ALLOC(e->d_hub_id, (size_t)kmax * sizeof(int));
        EX_CUDA(cudaMemcpy(e->d_hub_id, ids.data(), (size_t)k * sizeof(int), cudaMemcpyHostToDevice));
        e->hub_k = k;
        if ((size_t)k * sizeof(int) > 48 * 1024)   // the encoder keeps the sorted ids in shared memory
            EX_CUDA(cudaFuncSetAttribute(k_hub_encode, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)((size_t)k * sizeof(int))));
        for (int c = 0; c < e->nc; c++)   // chunks loaded so far; later loads encode themselves
            if (e->loaded[c] && e->ce[c + 1] <= e->cache_edges) hub_encode(e, e->ce[c], e->ce[c + 1], e->s_main);
        EX_CUDA(cudaStreamSynchronize(e->s_main));
        EX_CUDA(cudaGetLastError());
    }
    const size_t smem = hub_smem(e);
    if (smem > 0) {   // static + dynamic above 48 KiB needs the opt-in, per kernel (the staged kernels hold ~40 KiB)
        const int sz = (int)smem;
        cudaFuncSetAttribute(k_push<1, SRC_TABLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<1, SRC_CHUNK>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<1, SRC_GATHER>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<1, SRC_HOT>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<1, SRC_HUBS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<4, SRC_TABLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<4, SRC_CHUNK>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<4, SRC_GATHER>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<4, SRC_HOT>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_push<4, SRC_HUBS>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_segments<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        cudaFuncSetAttribute(k_segments<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, sz);
        EX_CUDA(cudaGetLastError());
    }
    int occ = 0;
    if (e->L == 1) EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_push<1, SRC_TABLE>, BLOCK, smem));
    else EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_push<4, SRC_TABLE>, BLOCK, smem));
    e->grid_push = e->sms * std::max(1, occ);
    return EXCENT_OK;
}

extern "C" int excent_engine_set_hub_order(excent_engine* e, int order) {
    EX_CHECK_ARG(e && order >= -1 && order <= 3,
                 "hub order must be 0 (table order), 1 (first), 2 (last), 3 (first in each launch) or -1 (by the "
                 "chunk count)");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    e->hub_order = order;
    return EXCENT_OK;
}

// Every entry of the edge cache, in cache order, reduced into a scratch array
// shaped like r: the scatter's ceiling on this graph's target distribution.
template <int L>
__global__ void __launch_bounds__(BLOCK) k_scatter_probe(ull m, const int* cache, const int* hub_id, int hub_k,
                                                         typename Lane<L>::T* out) {
    typedef typename Lane<L>::T T;
    T* hacc = hacc_init<T>(hub_k);
    T one;
    if constexpr (L == 1) one = 1.f; else one = make_float4(1.f, 1.f, 1.f, 0.f);
    const ull stride = (ull)gridDim.x * blockDim.x;
    const ull m4 = m / 4;
    const int4* c4 = reinterpret_cast<const int4*>(cache);
    ull i = blockIdx.x * (ull)blockDim.x + threadIdx.x;
    for (; i + stride < m4; i += 2 * stride) {   // two 16-byte loads in flight per thread
        const int4 q = ld_edge4(c4 + i), w = ld_edge4(c4 + i + stride);
        scatter_one(out, q.x, one, hacc); scatter_one(out, q.y, one, hacc);
        scatter_one(out, q.z, one, hacc); scatter_one(out, q.w, one, hacc);
        scatter_one(out, w.x, one, hacc); scatter_one(out, w.y, one, hacc);
        scatter_one(out, w.z, one, hacc); scatter_one(out, w.w, one, hacc);
    }
    for (; i < m4; i += stride) {
        const int4 q = ld_edge4(c4 + i);
        scatter_one(out, q.x, one, hacc); scatter_one(out, q.y, one, hacc);
        scatter_one(out, q.z, one, hacc); scatter_one(out, q.w, one, hacc);
    }
    for (ull j = m4 * 4 + blockIdx.x * (ull)blockDim.x + threadIdx.x; j < m; j += stride)
        scatter_one(out, cache[j], one, hacc);
    hacc_flush(hacc, out, hub_id, hub_k);
}

extern "C" int excent_engine_scatter_peak(excent_engine* e, double* entries_per_second) {
    EX_CHECK_ARG(e && entries_per_second, "null argument");
    EX_CHECK_ARG(e->d_cache && e->cache_edges == e->m, "the scatter probe needs the whole graph in the edge cache");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaDeviceSynchronize());
    const size_t bytes = (size_t)e->n * (e->L == 1 ? sizeof(float) : sizeof(float4));
    void* out = nullptr;
    if (cudaMalloc(&out, bytes) != cudaSuccess) { cudaGetLastError(); EX_FAIL(EXCENT_ERR_NOMEM, "probe array of %zu bytes", bytes); }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 0.f;
    if (hub_smem(e)) {
        cudaFuncSetAttribute(k_scatter_probe<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hub_smem(e));
        cudaFuncSetAttribute(k_scatter_probe<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hub_smem(e));
    }
    for (int rep = 0; rep < 4; rep++) {   // the first launch warms up; best of the other three
        cudaEventRecord(e0, e->s_main);
        if (e->L == 1)
            k_scatter_probe<1><<<e->grid_push, BLOCK, hub_smem(e), e->s_main>>>(e->m, e->d_cache, e->d_hub_id, e->hub_k,
                                                                               (float*)out);
        else
            k_scatter_probe<4><<<e->grid_push, BLOCK, hub_smem(e), e->s_main>>>(e->m, e->d_cache, e->d_hub_id, e->hub_k,
                                                                               (float4*)out);
        cudaEventRecord(e1, e->s_main);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    const cudaError_t rc = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    EX_CUDA(rc);
    *entries_per_second = best > 0.f ? (double)e->m / (best * 1e-3) : 0.0;
    return EXCENT_OK;
}

// Setting candidates of the device solve, timed one full solve each on this
// graph (after one untimed solve that builds the graph); the fastest is kept.
extern "C" int excent_engine_autotune(excent_engine* e, double list_frac, int max_passes, excent_tune* best,
                                      excent_tune* tried, int cap, int* ntried) {
    EX_CHECK_ARG(e && best, "null argument");
    EX_CHECK_ARG(e->d_cache && e->cache_edges == e->m, "autotuning needs the whole graph in the edge cache");
    EX_CUDA(cudaSetDevice(e->dev));
    // hub-target slots: a chunk-by-chunk pass flushes them once per chunk, so it measured
    // best with fewer slots (2048 for one measure) than a one-launch pass (16384)
    auto k = [&](int want) { return std::min(e->n, want); };
    const bool one = e->L == 1;
    const excent_tune cands[] = {
        // swept while a pass's pending entries reach the demand fraction of m, each launch's long
        // lists first (one candidate in plain table order)
        {k(2048), 3, 1, 0.0, 0.5}, {k(2048), 3, 1, 0.0, 0.25}, {k(2048), 3, 1, 0.0, 1.0},
        {k(one ? 16384 : 4096), 3, 1, 0.0, 0.5}, {k(2048), 0, 1, 0.0, 0.5},
        // the high-degree lists first, one launch per pass
        {k(one ? 16384 : 4096), 1, 0, 0.0, 0.0}, {k(one ? 4096 : 2048), 1, 0, 0.0, 0.0}, {0, 1, 0, 0.0, 0.0},
    };
    const int nc = (int)(sizeof cands / sizeof cands[0]);
    cudaEvent_t t0, t1;
    EX_CUDA(cudaEventCreate(&t0));
    EX_CUDA(cudaEventCreate(&t1));
    excent_tune win{};
    win.ms = -1;
    int rc = EXCENT_OK;
    for (int i = 0; i < nc && rc == EXCENT_OK; i++) {
        excent_tune c = cands[i];
        rc = excent_engine_set_hub_targets(e, c.hub_targets);
        if (rc == EXCENT_OK) rc = excent_engine_set_hub_order(e, c.hub_order);
        if (rc == EXCENT_OK) rc = excent_engine_set_chunk_sweep(e, c.chunk_sweep);
        if (rc == EXCENT_OK && c.chunk_sweep) rc = excent_engine_set_sweep_demand(e, c.sweep_demand);
        if (rc == EXCENT_OK) rc = excent_engine_solve(e, list_frac, max_passes, 1);   // builds the graph
        if (rc != EXCENT_OK) break;
        cudaEventRecord(t0, e->s_main);
        rc = excent_engine_solve(e, list_frac, max_passes, 1);
        cudaEventRecord(t1, e->s_main);
        cudaEventSynchronize(t1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, t0, t1);
        c.ms = ms;
        if (tried && i < cap) tried[i] = c;
        if (ntried) *ntried = i + 1;
        if (win.ms < 0 || c.ms < win.ms) win = c;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    EX_TRY(rc);
    EX_TRY(excent_engine_set_hub_targets(e, win.hub_targets));
    EX_TRY(excent_engine_set_hub_order(e, win.hub_order));
    EX_TRY(excent_engine_set_chunk_sweep(e, win.chunk_sweep));
    if (win.chunk_sweep) EX_TRY(excent_engine_set_sweep_demand(e, win.sweep_demand));
    *best = win;
    return EXCENT_OK;
}

extern "C" int excent_engine_set_chunk_sweep(excent_engine* e, int on) {
    EX_CHECK_ARG(e, "null engine");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    e->sweep_mode = on < 0 ? -1 : (on != 0);
    return EXCENT_OK;
}

extern "C" int excent_engine_set_sweep_demand(excent_engine* e, double frac) {
    EX_CHECK_ARG(e && frac >= 0.0 && frac <= 1e6, "sweep demand must be a fraction of m >= 0");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    e->sweep_frac = frac;
    return EXCENT_OK;
}

extern "C" int excent_engine_set_claim_tiles(excent_engine* e, int tiles) {
    EX_CHECK_ARG(e && tiles >= 0 && tiles <= 1024, "tiles per claim must be 0 (by launch size) to 1024");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    e->claim_tiles = tiles;
    return EXCENT_OK;
}

extern "C" int excent_engine_host_cache(excent_engine* e, int32_t** host_edges, unsigned long long* first_edge) {
    EX_CHECK_ARG(e && host_edges, "null argument");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    EX_CUDA(cudaDeviceSynchronize());
    free_host_cache(e);
    *host_edges = nullptr;
    const ull cnt = e->m - e->cache_edges;
    if (first_edge) *first_edge = e->cache_edges;
    if (cnt == 0) return EXCENT_OK;
    if (cudaHostAlloc((void**)&e->h_hcache, cnt * sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        e->h_hcache = nullptr;
        EX_FAIL(EXCENT_ERR_NOMEM, "pinned host cache of %llu entries does not fit", cnt);
    }
    e->hcache_edges = cnt;
    EX_CUDA(cudaHostGetDevicePointer((void**)&e->d_hcache, e->h_hcache, 0));
    *host_edges = e->h_hcache;
    return EXCENT_OK;
}

// The host cache in ordinary (pageable) memory, pinned later in pieces: the
// caller fills it and pins each filled piece (excent_engine_host_cache_pin)
// while it reads the next, so pinning overlaps the file reads instead of
// following them (cudaHostAlloc also zero-fills the whole buffer first).
// pieces_ok = 0: this device cannot address registered memory by its host
// address, so the whole range must be pinned in one call at the end.
extern "C" int excent_engine_host_cache_begin(excent_engine* e, int32_t** host_edges, unsigned long long* first_edge,
                                              int* pieces_ok) {
    EX_CHECK_ARG(e && host_edges && pieces_ok, "null argument");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    EX_CUDA(cudaDeviceSynchronize());
    free_host_cache(e);
    *host_edges = nullptr;
    const ull cnt = e->m - e->cache_edges;
    if (first_edge) *first_edge = e->cache_edges;
    int direct = 0;
    EX_CUDA(cudaDeviceGetAttribute(&direct, cudaDevAttrCanUseHostPointerForRegisteredMem, e->dev));
    *pieces_ok = direct;
    if (cnt == 0) return EXCENT_OK;
    const size_t page = (size_t)sysconf(_SC_PAGESIZE);
    const size_t bytes = (cnt * sizeof(int) + page - 1) / page * page;
    void* p = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (p == MAP_FAILED) EX_FAIL(EXCENT_ERR_NOMEM, "host cache of %llu entries: mmap failed", cnt);
    e->h_hcache = (int*)p;
    e->hcache_edges = cnt;
    e->hcache_map_bytes = bytes;
    e->hcache_pinned = 0;
    *host_edges = e->h_hcache;
    return EXCENT_OK;
}

// Pin the host cache's entries [0, upto) (relative to its first entry), past
// what is pinned already; the last call (upto = its size) makes it usable.
extern "C" int excent_engine_host_cache_pin(excent_engine* e, unsigned long long upto) {
    EX_CHECK_ARG(e && e->h_hcache && e->hcache_map_bytes, "no host cache begun");
    EX_CHECK_ARG(upto <= e->hcache_edges, "pin range past the host cache");
    EX_CUDA(cudaSetDevice(e->dev));
    const size_t page = (size_t)sysconf(_SC_PAGESIZE);
    size_t end = upto == e->hcache_edges ? e->hcache_map_bytes : (size_t)upto * sizeof(int) / page * page;
    if (end <= e->hcache_pinned) return EXCENT_OK;
    int direct = 0;
    EX_CUDA(cudaDeviceGetAttribute(&direct, cudaDevAttrCanUseHostPointerForRegisteredMem, e->dev));
    EX_CHECK_ARG(direct || (e->hcache_pinned == 0 && end == e->hcache_map_bytes),
                 "this device pins the host cache in one piece only");
    char* at = (char*)e->h_hcache + e->hcache_pinned;
    const size_t len = end - e->hcache_pinned;
    if (cudaHostRegister(at, len, cudaHostRegisterMapped | cudaHostRegisterPortable) != cudaSuccess) {
        cudaGetLastError();
        EX_FAIL(EXCENT_ERR_NOMEM, "pinning %zu bytes of the host cache failed", len);
    }
    e->hcache_pieces.push_back({at, len});
    e->hcache_pinned = end;
    if (end == e->hcache_map_bytes) {
        if (direct) e->d_hcache = e->h_hcache;
        else EX_CUDA(cudaHostGetDevicePointer((void**)&e->d_hcache, e->h_hcache, 0));
    }
    return EXCENT_OK;
}

extern "C" int excent_engine_host_pushed(excent_engine* e, unsigned long long* entries) {
    EX_CHECK_ARG(e && entries, "null argument");
    EX_CUDA(cudaSetDevice(e->dev));
    EX_CUDA(cudaStreamSynchronize(e->s_main));
    EX_CUDA(cudaMemcpy(entries, &e->d_ctrl->host_pushed, sizeof(ull), cudaMemcpyDeviceToHost));
    return EXCENT_OK;
}

extern "C" int excent_engine_ev_project(excent_engine* e, const float* d_v1) {
    EX_CHECK_ARG(e, "null engine");
    EX_CUDA(cudaSetDevice(e->dev));
    invalidate_graph(e);
    if (!d_v1) { e->ev_proj = false; return EXCENT_OK; }
    int ev = -1;
    for (int i = 0; i < e->nm; i++) if (e->meas.kind[i] == EXCENT_EV) ev = i;
    EX_CHECK_ARG(ev >= 0, "the run has no eigenvector measure");
    if (!e->d_v1) EX_ALLOC(e->d_v1, (size_t)e->n * sizeof(float));
    EX_CUDA(cudaMemcpy(e->d_v1, d_v1, (size_t)e->n * sizeof(float), cudaMemcpyDefault));
    {
        std::vector<float> h((size_t)e->n);
        EX_CUDA(cudaMemcpy(h.data(), e->d_v1, (size_t)e->n * sizeof(float), cudaMemcpyDeviceToHost));
        float vmax = 0.f;
        for (float q : h) vmax = std::max(vmax, std::fabs(q));
        e->ev_skip = vmax > 0.f ? 1e-3 * (double)e->M.eps[ev] / (double)vmax : 0.0;
    }
    e->ev_index = ev;
    e->ev_proj = true;
    return EXCENT_OK;
}

extern "C" int excent_engine_stream(excent_engine* e, void** stream) {
    EX_CHECK_ARG(e && stream, "null argument");
    *stream = (void*)e->s_main;
    return EXCENT_OK;
}

extern "C" int excent_engine_profile(excent_engine* e, int enable) {
    EX_CHECK_ARG(e, "null engine");
    EX_CUDA(cudaSetDevice(e->dev));
    if (enable && !e->ev[0])
        for (cudaEvent_t& ev : e->ev) EX_CUDA(cudaEventCreate(&ev));
    e->prof = enable != 0;
    for (double& t : e->prof_ms) t = 0;
    e->prof_passes = 0;
    return EXCENT_OK;
}

extern "C" int excent_engine_profile_read(excent_engine* e, double* ms, unsigned long long* passes) {
    EX_CHECK_ARG(e && ms, "null argument");
    for (int k = 0; k < 4; k++) ms[k] = e->prof_ms[k];
    if (passes) *passes = e->prof_passes;
    return EXCENT_OK;
}

extern "C" int excent_engine_launches(excent_engine* e, unsigned long long* launches) {
    EX_CHECK_ARG(e && launches, "null argument");
    *launches = e->launches;
    return EXCENT_OK;
}
