// batched.cu -- many personalized PageRank (or Katz) solves at once on a
// cached graph: B lanes (queries) per vertex, residuals and values laid out
// vertex-major [n][B] in FP32 so that one adjacency entry read from HBM feeds
// all B lanes with B/4 contiguous 16-byte reductions.
//
// No reference counterpart (the reference solves one centrality at a time).
// Semantics per lane q are the delta-push of the plain engine: a lane is
// pending at v iff |r[v][q]| > eps[q]; pushing takes r[v][q] (exchange with
// zero), adds it to x[v][q] and adds scale * d / deg(v) (personalized
// PageRank) or scale * d (Katz) to every neighbour's r[u][q].
//
// Frontier: a vertex is re-examined only if its row changed. A pass scans the
// "touched" bitmap of the previous pass (clearing it), checks each touched
// row against eps, takes and pushes the pending lanes and marks every
// receiving neighbour in the other touched bitmap (check before atomic OR).
// The solve ends after a pass that pushed nothing. One persistent kernel does
// the scan, take and push; lists longer than 512 entries are split into
// segments handled by a second kernel; a one-thread kernel advances the pass
// and sets the loop condition of the CUDA graph that runs all passes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "device.cuh"

namespace excent {

static constexpr int BB = 256;              // threads per block
static constexpr unsigned BHUB_MIN = 512;   // lists longer than this go to segments
static constexpr unsigned BHUB_SEG = 512;

struct BSeg {
    const int* nb;
    unsigned len;
    unsigned slot;  // row of the hub weight buffer
};

struct BCtrl {
    int pass;                 // passes executed
    int max_passes;
    ull pushed_v[2];          // vertices pushed, by pass parity
    ull hub_rows[2], hub_segs[2];
    ull total_v, total_e, total_lane_e;  // totals over the solve
    ull rows_checked;                    // touched rows examined, over the solve
    ull total_segs;                      // hub segments queued, over the solve
    int err;
    int done;
};

struct BArgs {
    int n;
    int V;                    // float4 per row = B / 4
    float4* R;
    float4* X;
    const float4* eps;        // V entries
    const ull* idx;
    const int* adj;
    float scale;
    int divdeg;
    uint32_t* touched[2];
    int words;
    float4* P;                // hub weight rows
    ull prow_cap;
    BSeg* seg;
    ull seg_cap;
    BCtrl* ctrl;
    int greedy;               // take every nonzero lane of a pushed row, not only the pending ones
    int dense;                // hub segments of rows with more active groups scatter over the groups
};

__device__ __forceinline__ float take_lane(float* rp, float rv, float eps) {
    return fabsf(rv) > eps ? atomicExch(rp, 0.f) : 0.f;
}

// Scatter list nb[0..deg) of a pushed row with the lanes over entries: lane i
// takes entry e0 + i and adds the row's nact active 16-byte groups (indices
// gi[], weights gp[] in shared memory, the same for every lane) to that
// target's row, so a warp keeps 32 targets in flight.
__device__ __forceinline__ ull scatter_lanes(float4* R, int V, uint32_t* nxt, const int* nb, unsigned deg,
                                             const float4* gp, const int* gi, int nact, int lane) {
    ull upd = 0;
    for (unsigned e0 = 0; e0 < deg; e0 += 128) {
        int u[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {   // four index loads in flight before the reductions
            const unsigned e = e0 + 32 * k + lane;
            u[k] = e < deg ? ld_edge(nb + e) : -1;
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (u[k] < 0) continue;
            float4* row = R + (size_t)u[k] * V;
            for (int i = 0; i < nact; i++) red_add(row, gi[i], gp[i]);
            const uint32_t bit = 1u << (u[k] & 31);   // check first: most targets are marked already
            if (!(nxt[u[k] >> 5] & bit)) atomicOr(&nxt[u[k] >> 5], bit);
            upd += (ull)nact;
        }
    }
    return upd;
}

// Scatter for rows with many active groups: the lanes over the row's groups
// (lane j0 + LPR * k of each LPR-lane sub-warp), 32 / LPR target rows per
// step, so each reduction instruction covers one contiguous stretch of a
// target row instead of 32 unrelated rows.
template <int LPR, int NV>
__device__ __forceinline__ ull scatter_rowpar(float4* R, int V, uint32_t* nxt, const int* nb, unsigned deg,
                                              const float4 (&p)[NV], const bool (&act)[NV], int lane) {
    constexpr int RPW = 32 / LPR;
    const int sub = lane / LPR, j0 = lane % LPR;
    ull upd = 0;
    for (unsigned e0 = 0; e0 < deg; e0 += 32) {
        const int ul = e0 + lane < deg ? ld_edge(nb + e0 + lane) : -1;
        if (ul >= 0) {   // each lane marks its own entry's target, all 32 at once
            const uint32_t bit = 1u << (ul & 31);
            if (!(nxt[ul >> 5] & bit)) atomicOr(&nxt[ul >> 5], bit);
        }
        const unsigned cnt = min(32u, deg - e0);
        for (unsigned g = 0; g < cnt; g += RPW) {
            const int u = __shfl_sync(FULL, ul, (int)g + sub);
            if (g + sub < cnt) {
                float4* row = R + (size_t)u * V;
#pragma unroll
                for (int k = 0; k < NV; k++)
                    if (act[k]) { red_add(row, j0 + LPR * k, p[k]); upd++; }
            }
        }
    }
    return upd;
}

// Default: segments of rows with more active 16-byte groups than this scatter over their groups.
static constexpr int DENSE_GROUPS = 4;

// Compact the active groups of a row held by lanes j0 + LPR * k (k < NV) into
// the warp's shared lists; returns their count (warp-uniform).
template <int LPR, int NV>
__device__ __forceinline__ int compact_groups(const float4 (&p)[NV], const bool (&act)[NV], float4* gp, int* gi,
                                              int lane) {
    const int j0 = lane % LPR;
    int base = 0;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        const bool on = lane < LPR && act[k];
        const unsigned b = __ballot_sync(FULL, on);
        if (on) {
            const int at = base + __popc(b & ((1u << lane) - 1u));
            gp[at] = p[k];
            gi[at] = j0 + LPR * k;
        }
        base += __popc(b);
    }
    __syncwarp();
    return base;
}

// One pass: scan touched words (interleaved over warps), check, take and push.
template <int LPR, int NV>
__global__ void __launch_bounds__(BB, 4) k_bpass(BArgs a) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int j0 = lane % LPR;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    __shared__ float4 s_gp[BB / 32][LPR * NV];
    __shared__ int s_gi[BB / 32][LPR * NV];
    const int par = a.ctrl->pass & 1;
    uint32_t* cur = par ? a.touched[1] : a.touched[0];   // no run-time index into the parameters
    uint32_t* nxt = par ? a.touched[0] : a.touched[1];
    ull pushed_v = 0, pushed_e = 0, upd = 0, checked = 0;
    float4 eps[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) eps[k] = a.eps[j0 + LPR * k];
    for (long long jw = 0; gw + jw * nwarps < a.words; jw += 32) {
        // warp gw owns words gw + j * nwarps (interleaved, so dense regions spread over all
        // warps); it reads 32 of them per step, one per lane, then walks the nonzero ones
        const long long wl = gw + (jw + lane) * nwarps;
        const uint32_t mine = wl < a.words ? cur[wl] : 0u;
        if (mine) { cur[wl] = 0; checked += __popc(mine); }
        unsigned nzw = __ballot_sync(FULL, mine != 0);
        while (nzw) {
        const int src = __ffs(nzw) - 1;
        nzw &= nzw - 1;
        const long long w = gw + (jw + src) * nwarps;
        uint32_t bits = __shfl_sync(FULL, mine, src);
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const int v = (int)(w * 32 + b);
            float4* rrow = a.R + (size_t)v * a.V;
            float4 d[NV];
            bool any = false;
            // a row with any pending lane is pushed whole (greedy): every lane with a nonzero
            // residual is taken, since the one read of the list serves them all
            float4 rv[NV];
            bool pend = false;
#pragma unroll
            for (int k = 0; k < NV; k++) {
                rv[k] = lane < LPR ? rrow[j0 + LPR * k] : make_float4(0.f, 0.f, 0.f, 0.f);
                pend |= fabsf(rv[k].x) > eps[k].x || fabsf(rv[k].y) > eps[k].y || fabsf(rv[k].z) > eps[k].z ||
                        fabsf(rv[k].w) > eps[k].w;
            }
            const bool row_pend = __any_sync(FULL, pend);
            const float4 floor0 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int k = 0; k < NV; k++) {
                d[k] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (lane < LPR && row_pend) {
                    if (a.greedy) {
                        // the whole 16-byte group in one exchange when any of its lanes is nonzero
                        if (nonzero(rv[k])) d[k] = atomicExch(rrow + j0 + LPR * k, floor0);
                    } else {
                        const float4 th = eps[k];
                        float* rp = reinterpret_cast<float*>(rrow + j0 + LPR * k);
                        d[k].x = take_lane(rp, rv[k].x, th.x);
                        d[k].y = take_lane(rp + 1, rv[k].y, th.y);
                        d[k].z = take_lane(rp + 2, rv[k].z, th.z);
                        d[k].w = take_lane(rp + 3, rv[k].w, th.w);
                    }
                    if (nonzero(d[k])) {
                        float4* xp = a.X + (size_t)v * a.V + j0 + LPR * k;
                        float4 xv = *xp;
                        xv.x += d[k].x; xv.y += d[k].y; xv.z += d[k].z; xv.w += d[k].w;
                        *xp = xv;
                        any = true;
                    }
                }
            }
            if (!__any_sync(FULL, any)) continue;
            const ull b0 = a.idx[v];
            const unsigned deg = (unsigned)(a.idx[v + 1] - b0);
            if (lane == 0) { pushed_v++; pushed_e += deg; }
            if (deg == 0) continue;
            float4 p[NV];
            bool act[NV];
            const float f = a.divdeg ? a.scale / (float)deg : a.scale;
#pragma unroll
            for (int k = 0; k < NV; k++) {
                float4 q = shfl(d[k], j0);  // lanes >= LPR take the weights of lane j0
                if (a.divdeg) {  // scale * d / deg, in the order of the plain push
                    q = make_float4(a.scale * q.x / (float)deg, a.scale * q.y / (float)deg,
                                    a.scale * q.z / (float)deg, a.scale * q.w / (float)deg);
                } else {
                    q = make_float4(f * q.x, f * q.y, f * q.z, f * q.w);
                }
                p[k] = q;
                act[k] = nonzero(q);
            }
            const int* nb = a.adj + b0;
            if (deg > BHUB_MIN) {
                // queue: weight row into the hub buffer, segments of BHUB_SEG entries
                ull slot = 0, sbase = 0;
                const unsigned nseg = (deg + BHUB_SEG - 1) / BHUB_SEG;
                if (lane == 0) {
                    slot = atomicAdd(&a.ctrl->hub_rows[par], 1ull);
                    sbase = atomicAdd(&a.ctrl->hub_segs[par], (ull)nseg);
                }
                slot = __shfl_sync(FULL, slot, 0);
                sbase = __shfl_sync(FULL, sbase, 0);
                if (slot < a.prow_cap && sbase + nseg <= a.seg_cap) {
                    if (lane < LPR)
#pragma unroll
                        for (int k = 0; k < NV; k++) a.P[slot * a.V + j0 + LPR * k] = p[k];
                    for (unsigned s = lane; s < nseg; s += 32) {
                        BSeg sg;
                        sg.nb = nb + (size_t)s * BHUB_SEG;
                        sg.len = min(BHUB_SEG, deg - s * BHUB_SEG);
                        sg.slot = (unsigned)slot;
                        a.seg[sbase + s] = sg;
                    }
                } else if (lane == 0) {
                    atomicExch(&a.ctrl->err, 1);
                }
                continue;
            }
            // (lists up to BHUB_MIN: lanes over entries measured faster here at any density)
            const int nact = compact_groups<LPR, NV>(p, act, s_gp[wib], s_gi[wib], lane);
            upd += scatter_lanes(a.R, a.V, nxt, nb, deg, s_gp[wib], s_gi[wib], nact, lane);
            __syncwarp();
        }
        }
    }
    __shared__ ull s_v[BB / 32], s_e[BB / 32], s_u[BB / 32], s_c[BB / 32];
    pushed_v = warp_sum(pushed_v);
    pushed_e = warp_sum(pushed_e);
    upd = warp_sum(upd);
    checked = warp_sum(checked);
    if (lane == 0) { s_v[wib] = pushed_v; s_e[wib] = pushed_e; s_u[wib] = upd; s_c[wib] = checked; }
    __syncthreads();
    if (threadIdx.x == 0) {
        ull tv = 0, te = 0, tu = 0, tc = 0;
        for (int i = 0; i < BB / 32; i++) { tv += s_v[i]; te += s_e[i]; tu += s_u[i]; tc += s_c[i]; }
        if (tv) atomicAdd(&a.ctrl->pushed_v[par], tv);
        if (te) atomicAdd(&a.ctrl->total_e, te);
        if (tu) atomicAdd(&a.ctrl->total_lane_e, tu);
        if (tc) atomicAdd(&a.ctrl->rows_checked, tc);
    }
}

template <int LPR, int NV>
__global__ void __launch_bounds__(BB) k_bhub(BArgs a) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int j0 = lane % LPR;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int par = a.ctrl->pass & 1;
    uint32_t* nxt = par ? a.touched[0] : a.touched[1];
    ull nseg = a.ctrl->hub_segs[par];
    if (nseg > a.seg_cap) nseg = a.seg_cap;
    __shared__ float4 s_gp[BB / 32][LPR * NV];
    __shared__ int s_gi[BB / 32][LPR * NV];
    ull upd = 0;
    for (long long s = gw; s < (long long)nseg; s += nwarps) {
        const BSeg sg = a.seg[s];
        float4 p[NV];
        bool act[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) {
            p[k] = a.P[(size_t)sg.slot * a.V + j0 + LPR * k];
            act[k] = nonzero(p[k]);
        }
        const int nact = compact_groups<LPR, NV>(p, act, s_gp[wib], s_gi[wib], lane);
        if (nact > a.dense) upd += scatter_rowpar<LPR, NV>(a.R, a.V, nxt, sg.nb, sg.len, p, act, lane);
        else upd += scatter_lanes(a.R, a.V, nxt, sg.nb, sg.len, s_gp[wib], s_gi[wib], nact, lane);
        __syncwarp();
    }
    __shared__ ull s_u[BB / 32];
    upd = warp_sum(upd);
    if (lane == 0) s_u[wib] = upd;
    __syncthreads();
    if (threadIdx.x == 0) {
        ull tu = 0;
        for (int i = 0; i < BB / 32; i++) tu += s_u[i];
        if (tu) atomicAdd(&a.ctrl->total_lane_e, tu);
    }
}

// Vertices with more than thr entries.
__global__ void k_bcount(int n, const ull* idx, unsigned thr, ull* out) {
    ull c = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        c += idx[v + 1] - idx[v] > thr;
    c = warp_sum(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// End of a pass: totals, next pass's counters, loop condition.
__global__ void k_bend(BCtrl* c, cudaGraphConditionalHandle cond, int use_cond) {
    const int par = c->pass & 1;
    const ull pv = c->pushed_v[par];
    c->total_v += pv;
    c->total_segs += c->hub_segs[par];
    c->pushed_v[par ^ 1] = 0;
    c->hub_rows[par ^ 1] = 0;
    c->hub_segs[par ^ 1] = 0;
    const bool more = pv > 0 && c->pass + 1 < c->max_passes && !c->err;
    if (pv > 0) c->pass++;
    if (!more) c->done = 1;
    if (use_cond) cudaGraphSetConditional(cond, more ? 1u : 0u);
}

__global__ void k_bseed(int nq, const int* lane_off, const int* vids, const float* vals, float* R, int B,
                        uint32_t* touched) {
    const int q = blockIdx.x;
    if (q >= nq) return;
    for (int i = lane_off[q] + threadIdx.x; i < lane_off[q + 1]; i += blockDim.x) {
        const int v = vids[i];
        R[(size_t)v * B + q] += vals[i];
        atomicOr(&touched[v >> 5], 1u << (v & 31));
    }
}

__global__ void k_bcolumn(int n, const float* S, int B, int q, float* out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        out[v] = S[(size_t)v * B + q];
}

}  // namespace excent

using namespace excent;

struct excent_batch {
    int dev = 0, sms = 0;
    int n = 0, B = 0, kind = 0;
    ull m = 0;
    float scale = 0;
    const ull* d_idx = nullptr;
    const int* d_adj = nullptr;
    float* d_R = nullptr;
    float* d_X = nullptr;
    float* d_eps = nullptr;
    uint32_t* d_t[2] = {nullptr, nullptr};
    float4* d_P = nullptr;
    BSeg* d_seg = nullptr;
    ull prow_cap = 0, seg_cap = 0;
    BCtrl* d_ctrl = nullptr;
    int* d_seed_off = nullptr;
    int* d_seed_v = nullptr;
    float* d_seed_x = nullptr;
    size_t seed_cap = 0;
    float* d_col = nullptr;
    cudaStream_t st = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    int graph_max = -1;
    int grid = 0;
    ull launches = 0;
    int greedy = 1;
    int dense = DENSE_GROUPS;   // see excent_batch_set_dense
};

static void batch_free(excent_batch* b) {
    cudaSetDevice(b->dev);
    cudaDeviceSynchronize();
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    void* ps[] = {b->d_R, b->d_X, b->d_eps, b->d_t[0], b->d_t[1], b->d_P, b->d_seg, b->d_ctrl,
                  b->d_seed_off, b->d_seed_v, b->d_seed_x, b->d_col};
    for (void* p : ps) if (p) cudaFree(p);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

#define BX_ALLOC(ptr, bytes) do { if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) { cudaGetLastError(); \
    ::excent::set_error("batch: device allocation of %llu bytes failed (%s)", (ull)(bytes), #ptr); return EXCENT_ERR_NOMEM; } } while (0)

static BArgs bargs(excent_batch* b) {
    BArgs a{};
    a.n = b->n; a.V = b->B / 4;
    a.R = (float4*)b->d_R; a.X = (float4*)b->d_X; a.eps = (const float4*)b->d_eps;
    a.idx = b->d_idx; a.adj = b->d_adj;
    a.scale = b->scale; a.divdeg = b->kind == EXCENT_PR;
    a.touched[0] = b->d_t[0]; a.touched[1] = b->d_t[1];
    a.words = (int)(((size_t)b->n + 31) / 32);
    a.P = b->d_P; a.prow_cap = b->prow_cap; a.seg = b->d_seg; a.seg_cap = b->seg_cap;
    a.ctrl = b->d_ctrl;
    a.greedy = b->greedy;
    a.dense = b->dense;
    return a;
}

template <int LPR, int NV>
static void launch_pass_t(excent_batch* b, cudaStream_t st, cudaGraphConditionalHandle cond, int use_cond) {
    BArgs a = bargs(b);
    k_bpass<LPR, NV><<<b->grid, BB, 0, st>>>(a);
    k_bhub<LPR, NV><<<b->grid, BB, 0, st>>>(a);
    k_bend<<<1, 1, 0, st>>>(b->d_ctrl, cond, use_cond);
}

static void launch_pass(excent_batch* b, cudaStream_t st, cudaGraphConditionalHandle cond, int use_cond) {
    switch (b->B) {
        case 32: launch_pass_t<8, 1>(b, st, cond, use_cond); break;
        case 64: launch_pass_t<16, 1>(b, st, cond, use_cond); break;
        case 128: launch_pass_t<32, 1>(b, st, cond, use_cond); break;
        default: launch_pass_t<32, 2>(b, st, cond, use_cond); break;
    }
    b->launches += 3;
}

static int batch_setup(excent_batch* b, int device, int n, ull m, const ull* d_idx, const int* d_adj, int B, int kind,
                       double d_or_alpha) {
    EX_CUDA(cudaSetDevice(device));
    b->dev = device;
    EX_CUDA(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device));
    b->n = n; b->m = m; b->B = B; b->kind = kind;
    b->scale = (float)d_or_alpha;
    b->d_idx = d_idx; b->d_adj = d_adj;
    EX_CUDA(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    const size_t rows = (size_t)n * B * sizeof(float);
    BX_ALLOC(b->d_R, rows);
    BX_ALLOC(b->d_X, rows);
    BX_ALLOC(b->d_eps, (size_t)B * sizeof(float));
    const size_t words = ((size_t)n + 31) / 32;
    BX_ALLOC(b->d_t[0], words * 4);
    BX_ALLOC(b->d_t[1], words * 4);
    {   // rows that can be queued in one pass: the vertices with more than BHUB_MIN entries
        ull* d_cnt = nullptr;
        BX_ALLOC(d_cnt, sizeof(ull));
        cudaMemset(d_cnt, 0, sizeof(ull));
        k_bcount<<<b->sms * 8, BB, 0, b->st>>>(n, d_idx, BHUB_MIN, d_cnt);
        ull cnt = 0;
        const cudaError_t err = cudaMemcpyAsync(&cnt, d_cnt, sizeof(ull), cudaMemcpyDeviceToHost, b->st);
        cudaStreamSynchronize(b->st);
        cudaFree(d_cnt);
        EX_CUDA(err);
        b->prow_cap = cnt + 16;
    }
    b->seg_cap = 2 * (m / BHUB_SEG) + 64;
    BX_ALLOC(b->d_P, b->prow_cap * (size_t)B * sizeof(float));
    BX_ALLOC(b->d_seg, b->seg_cap * sizeof(BSeg));
    BX_ALLOC(b->d_ctrl, sizeof(BCtrl));
    BX_ALLOC(b->d_col, (size_t)n * sizeof(float));
    int occ = 0;
    switch (B) {
        case 32: EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bpass<8, 1>, BB, 0)); break;
        case 64: EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bpass<16, 1>, BB, 0)); break;
        case 128: EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bpass<32, 1>, BB, 0)); break;
        default: EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bpass<32, 2>, BB, 0)); break;
    }
    b->grid = b->sms * std::max(1, occ);
    return EXCENT_OK;
}

extern "C" int excent_batch_create(int device, int n, unsigned long long m, const unsigned long long* d_idx,
                                   const int32_t* d_adj, int B, int kind, double d_or_alpha, excent_batch** out) {
    EX_CHECK_ARG(out && d_idx && (d_adj || m == 0) && n >= 1, "bad argument");
    EX_CHECK_ARG(B == 32 || B == 64 || B == 128 || B == 256, "batch width must be 32, 64, 128 or 256");
    EX_CHECK_ARG(kind == EXCENT_PR || kind == EXCENT_KATZ, "batched solves are personalized PageRank or Katz");
    *out = nullptr;
    excent_batch* b = new excent_batch();
    const int rc = batch_setup(b, device, n, m, d_idx, d_adj, B, kind, d_or_alpha);
    if (rc != EXCENT_OK) {
        std::string msg = get_error();
        batch_free(b);
        set_error("%s", msg.c_str());
        return rc;
    }
    *out = b;
    return EXCENT_OK;
}

extern "C" int excent_batch_destroy(excent_batch* b) {
    if (b) batch_free(b);
    return EXCENT_OK;
}

extern "C" int excent_batch_seed(excent_batch* b, int nq, const int* lane_off, const int32_t* vids, const float* vals,
                                 const float* eps) {
    EX_CHECK_ARG(b && nq >= 0 && nq <= b->B && lane_off && eps, "bad argument");
    EX_CHECK_ARG(lane_off[0] == 0, "lane_off[0] must be 0");
    for (int q = 0; q < nq; q++) EX_CHECK_ARG(lane_off[q + 1] >= lane_off[q], "lane_off must not decrease");
    const int ns = lane_off[nq];
    EX_CHECK_ARG(ns == 0 || (vids && vals), "null seeds");
    for (int i = 0; i < ns; i++) EX_CHECK_ARG(vids[i] >= 0 && vids[i] < b->n, "seed vertex %d out of range", vids[i]);
    EX_CUDA(cudaSetDevice(b->dev));
    const size_t rows = (size_t)b->n * b->B * sizeof(float);
    EX_CUDA(cudaMemsetAsync(b->d_R, 0, rows, b->st));
    EX_CUDA(cudaMemsetAsync(b->d_X, 0, rows, b->st));
    const size_t words = ((size_t)b->n + 31) / 32;
    EX_CUDA(cudaMemsetAsync(b->d_t[0], 0, words * 4, b->st));
    EX_CUDA(cudaMemsetAsync(b->d_t[1], 0, words * 4, b->st));
    std::vector<float> e(b->B, INFINITY);  // unused lanes never pend
    for (int q = 0; q < nq; q++) e[q] = eps[q];
    EX_CUDA(cudaMemcpyAsync(b->d_eps, e.data(), b->B * sizeof(float), cudaMemcpyHostToDevice, b->st));
    if ((size_t)ns > b->seed_cap || !b->d_seed_off) {
        if (b->d_seed_off) cudaFree(b->d_seed_off);
        if (b->d_seed_v) cudaFree(b->d_seed_v);
        if (b->d_seed_x) cudaFree(b->d_seed_x);
        b->seed_cap = std::max<size_t>(ns, 1024);
        BX_ALLOC(b->d_seed_off, (b->B + 1) * sizeof(int));
        BX_ALLOC(b->d_seed_v, b->seed_cap * sizeof(int));
        BX_ALLOC(b->d_seed_x, b->seed_cap * sizeof(float));
    }
    EX_CUDA(cudaMemcpyAsync(b->d_seed_off, lane_off, (nq + 1) * sizeof(int), cudaMemcpyHostToDevice, b->st));
    if (ns) {
        EX_CUDA(cudaMemcpyAsync(b->d_seed_v, vids, ns * sizeof(int), cudaMemcpyHostToDevice, b->st));
        EX_CUDA(cudaMemcpyAsync(b->d_seed_x, vals, ns * sizeof(float), cudaMemcpyHostToDevice, b->st));
    }
    if (nq) {
        k_bseed<<<nq, 256, 0, b->st>>>(nq, b->d_seed_off, b->d_seed_v, b->d_seed_x, b->d_R, b->B, b->d_t[0]);
        b->launches++;
    }
    EX_CUDA(cudaGetLastError());
    EX_CUDA(cudaStreamSynchronize(b->st));
    return EXCENT_OK;
}

static int batch_graph(excent_batch* b, int max_passes) {
    if (b->gexec && b->graph_max == max_passes) return EXCENT_OK;
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
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
    cudaStream_t cs;
    EX_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    EX_CUDA(cudaStreamBeginCaptureToGraph(cs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
    const ull before = b->launches;
    launch_pass(b, cs, h, 1);
    b->launches = before;
    cudaGraph_t captured;
    const cudaError_t ce = cudaStreamEndCapture(cs, &captured);
    cudaStreamDestroy(cs);
    EX_CUDA(ce);
    EX_CUDA(cudaGraphInstantiate(&b->gexec, g, 0));
    b->graph = g;
    b->graph_max = max_passes;
    return EXCENT_OK;
}

extern "C" int excent_batch_solve(excent_batch* b, int max_passes, int use_graph) {
    EX_CHECK_ARG(b && max_passes >= 1, "bad argument");
    EX_CUDA(cudaSetDevice(b->dev));
    BCtrl c{};
    c.max_passes = max_passes;
    EX_CUDA(cudaMemcpyAsync(b->d_ctrl, &c, sizeof c, cudaMemcpyHostToDevice, b->st));
    if (use_graph) {
        EX_TRY(batch_graph(b, max_passes));
        EX_CUDA(cudaGraphLaunch(b->gexec, b->st));
        EX_CUDA(cudaStreamSynchronize(b->st));
        EX_CUDA(cudaMemcpy(&c, b->d_ctrl, sizeof c, cudaMemcpyDeviceToHost));
        b->launches += 3ull * (c.pass + 1);
    } else {
        for (int p = 0; p < max_passes; p++) {
            launch_pass(b, b->st, 0, 0);
            EX_CUDA(cudaGetLastError());
            EX_CUDA(cudaMemcpyAsync(&c, b->d_ctrl, sizeof c, cudaMemcpyDeviceToHost, b->st));
            EX_CUDA(cudaStreamSynchronize(b->st));
            if (c.done) break;
        }
    }
    if (c.err) EX_FAIL(EXCENT_ERR_STATE, "batch: hub buffer capacity exceeded");
    return EXCENT_OK;
}

extern "C" int excent_batch_stats(excent_batch* b, int* passes, unsigned long long* pushed_vertices,
                                  unsigned long long* pushed_edges, unsigned long long* lane_updates,
                                  unsigned long long* rows_checked, unsigned long long* hub_segments) {
    EX_CHECK_ARG(b, "null batch");
    EX_CUDA(cudaSetDevice(b->dev));
    BCtrl c;
    EX_CUDA(cudaStreamSynchronize(b->st));
    EX_CUDA(cudaMemcpy(&c, b->d_ctrl, sizeof c, cudaMemcpyDeviceToHost));
    if (passes) *passes = c.pass;
    if (pushed_vertices) *pushed_vertices = c.total_v;
    if (pushed_edges) *pushed_edges = c.total_e;
    if (lane_updates) *lane_updates = c.total_lane_e;
    if (rows_checked) *rows_checked = c.rows_checked;
    if (hub_segments) *hub_segments = c.total_segs;
    return EXCENT_OK;
}

extern "C" int excent_batch_read(excent_batch* b, int lane, int residual, float* out) {
    EX_CHECK_ARG(b && out && lane >= 0 && lane < b->B, "bad argument");
    EX_CUDA(cudaSetDevice(b->dev));
    k_bcolumn<<<b->sms * 8, 256, 0, b->st>>>(b->n, residual ? b->d_R : b->d_X, b->B, lane, b->d_col);
    b->launches++;
    EX_CUDA(cudaGetLastError());
    EX_CUDA(cudaMemcpyAsync(out, b->d_col, (size_t)b->n * sizeof(float), cudaMemcpyDeviceToHost, b->st));
    EX_CUDA(cudaStreamSynchronize(b->st));
    return EXCENT_OK;
}

extern "C" int excent_batch_set_dense(excent_batch* b, int groups) {
    EX_CHECK_ARG(b && groups >= 0, "bad argument");
    b->dense = groups;
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    b->graph_max = -1;
    return EXCENT_OK;
}

extern "C" int excent_batch_set_greedy(excent_batch* b, int greedy) {
    EX_CHECK_ARG(b, "null batch");
    b->greedy = greedy != 0;
    if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    b->graph_max = -1;
    return EXCENT_OK;
}

extern "C" int excent_batch_stream(excent_batch* b, void** stream) {
    EX_CHECK_ARG(b && stream, "null argument");
    *stream = (void*)b->st;
    return EXCENT_OK;
}

extern "C" int excent_batch_launches(excent_batch* b, unsigned long long* launches) {
    EX_CHECK_ARG(b && launches, "null argument");
    *launches = b->launches;
    return EXCENT_OK;
}

// Autotuner: time one batch of min(B, nq) queries at every batch width in
// {32, 64, 128, 256} (the first queries of the set, seeded as given) and pick
// the width with the lowest time per query. per_query_ms[4] receives the
// measured times (0 where a width could not be allocated).
extern "C" int excent_batch_autotune(int device, int n, unsigned long long m, const unsigned long long* d_idx,
                                     const int32_t* d_adj, int kind, double d_or_alpha, int nq, const int* lane_off,
                                     const int32_t* vids, const float* vals, const float* eps, int max_passes,
                                     int* best_B, int* best_greedy, double* per_query_ms) {
    EX_CHECK_ARG(best_B && nq >= 1 && lane_off, "bad argument");
    const int widths[4] = {32, 64, 128, 256};
    double best = 1e300;
    *best_B = 0;
    if (best_greedy) *best_greedy = 1;
    for (int i = 0; i < 8; i++) {
        if (per_query_ms) per_query_ms[i] = 0;
        const int B = widths[i >> 1], greedy = i & 1;
        excent_batch* b = nullptr;
        if (excent_batch_create(device, n, m, d_idx, d_adj, B, kind, d_or_alpha, &b) != EXCENT_OK) continue;
        int rc = excent_batch_set_greedy(b, greedy);
        const int q = std::min(B, nq);
        if (rc == EXCENT_OK) rc = excent_batch_seed(b, q, lane_off, vids, vals, eps);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        float ms = 0;
        if (rc == EXCENT_OK) {
            rc = excent_batch_solve(b, max_passes, 1);   // builds the graph; not timed
            if (rc == EXCENT_OK) rc = excent_batch_seed(b, q, lane_off, vids, vals, eps);
            if (rc == EXCENT_OK) {
                cudaEventRecord(e0, b->st);
                rc = excent_batch_solve(b, max_passes, 1);
                cudaEventRecord(e1, b->st);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&ms, e0, e1);
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        excent_batch_destroy(b);
        if (rc != EXCENT_OK) return rc;
        const double pq = ms / q;
        if (per_query_ms) per_query_ms[i] = pq;
        if (pq < best) { best = pq; *best_B = B; if (best_greedy) *best_greedy = greedy; }
    }
    if (!*best_B) EX_FAIL(EXCENT_ERR_NOMEM, "autotune: no batch width could be allocated");
    return EXCENT_OK;
}
