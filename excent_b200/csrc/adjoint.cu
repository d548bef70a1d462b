// adjoint.cu -- differentiable weighted PageRank / Katz on a directed graph.
//
// Forward (kind EXCENT_PR): x = (1 - d) t + d W^T x, with W the row-normalised
// edge weights wn[e] = w[e] / sum_{e' in row u} w[e'] of edges u -> v, so
// (W^T x)_v = sum_{u -> v} wn[u->v] x_u. Katz (kind EXCENT_KATZ):
// x = beta + alpha W^T x. Both run as a delta-push over out-lists: pushing u
// adds s * wn[e] * d_u to r_v for each edge e = u -> v (s = d or alpha).
//
// Adjoint of a scalar loss L with dL/dx = c: lambda = c + s W lambda, a push
// over the transposed lists with the permuted weights. Gradients:
//   dL/dt = (1 - d) lambda (PageRank),  dL/dbeta = lambda (Katz),
//   dL/dwn[u->v] = s x_u lambda_v,
//   dL/dw[e] = (G_e - sum_{e' in row u} wn[e'] G_e') / rowsum_u, G = dL/dwn.
// No reference counterpart (the reference has no weights and no adjoint).
//
// The push passes use a touched-vertex frontier (a vertex is re-examined
// only after its residual changed) and run as one CUDA graph with a
// conditional while node. FP64 pull (Jacobi) solvers of the same fixed
// points give finite differences and the oracle gradient for verification.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "device.cuh"

namespace excent {

static constexpr int WB = 256;

struct WCtrl {
    int pass, max_passes, done, err;
    ull pushed_v[2];
    ull total_v, total_e;
};

struct WArgs {
    int n;
    const ull* idx;
    const int* adj;
    const float* wt;    // per-edge weight (row-normalised, forward or transposed order)
    float s;
    float eps;
    float* x;
    float* r;
    uint32_t* touched[2];
    int words;
    WCtrl* ctrl;
};

__device__ __forceinline__ void wmark(uint32_t* t, int u) {
    const uint32_t bit = 1u << (u & 31);
    if (!(t[u >> 5] & bit)) atomicOr(&t[u >> 5], bit);
}

// One pass: lanes take the touched vertices of a bitmap word, then the warp
// scatters each pushed vertex's list with s * d * wt[e] per entry.
__global__ void __launch_bounds__(WB) k_wpass(WArgs a) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long gw = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int par = a.ctrl->pass & 1;
    uint32_t* cur = par ? a.touched[1] : a.touched[0];   // no run-time index into the parameters
    uint32_t* nxt = par ? a.touched[0] : a.touched[1];
    ull pv = 0, pe = 0;
    for (long long w = gw; w < a.words; w += nwarps) {
        const uint32_t bits = cur[w];
        if (!bits) continue;
        __syncwarp();
        if (lane == 0) cur[w] = 0;
        const int v = (int)(w * 32 + lane);
        float d = 0.f;
        ull b0 = 0;
        unsigned deg = 0;
        if ((bits >> lane) & 1u) {
            if (fabsf(a.r[v]) > a.eps) {
                d = atomicExch(&a.r[v], 0.f);
                a.x[v] += d;
            }
            if (d != 0.f) {
                b0 = a.idx[v];
                deg = (unsigned)(a.idx[v + 1] - b0);
                pv++;
                pe += deg;
            }
        }
        uint32_t mm = __ballot_sync(FULL, d != 0.f && deg > 0);
        while (mm) {
            const int sl = __ffs(mm) - 1;
            mm &= mm - 1;
            const ull bb = __shfl_sync(FULL, b0, sl);
            const unsigned dd = __shfl_sync(FULL, deg, sl);
            const float f = a.s * __shfl_sync(FULL, d, sl);
            for (unsigned i0 = 0; i0 < dd; i0 += 128) {
                int u[4];
                float wt[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {   // four entries per lane in flight
                    const unsigned i = i0 + 32 * k + lane;
                    u[k] = i < dd ? ld_edge(a.adj + bb + i) : -1;
                    wt[k] = i < dd ? __ldcs(a.wt + bb + i) : 0.f;
                }
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (u[k] >= 0) red_add(a.r, u[k], f * wt[k]);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (u[k] >= 0) wmark(nxt, u[k]);
            }
        }
    }
    __shared__ ull s_v[WB / 32], s_e[WB / 32];
    pv = warp_sum(pv);
    pe = warp_sum(pe);
    if (lane == 0) { s_v[wib] = pv; s_e[wib] = pe; }
    __syncthreads();
    if (threadIdx.x == 0) {
        ull tv = 0, te = 0;
        for (int i = 0; i < WB / 32; i++) { tv += s_v[i]; te += s_e[i]; }
        if (tv) atomicAdd(&a.ctrl->pushed_v[par], tv);
        if (te) atomicAdd(&a.ctrl->total_e, te);
    }
}

__global__ void k_wend(WCtrl* c, cudaGraphConditionalHandle cond, int use_cond) {
    const int par = c->pass & 1;
    const ull pv = c->pushed_v[par];
    c->total_v += pv;
    c->pushed_v[par ^ 1] = 0;
    const bool more = pv > 0 && c->pass + 1 < c->max_passes;
    if (pv > 0) c->pass++;
    if (!more) c->done = 1;
    if (use_cond) cudaGraphSetConditional(cond, more ? 1u : 0u);
}

// x = 0, r = c0 * t (t NULL: all ones), touched where r != 0.
__global__ void k_wseed(int n, const float* t, float c0, float* x, float* r, uint32_t* touched) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const float rv = c0 * (t ? t[v] : 1.f);
        x[v] = 0.f;
        r[v] = rv;
        if (rv != 0.f) atomicOr(&touched[v >> 5], 1u << (v & 31));
    }
}

// Row sums and normalised weights (FP32 for the push, FP64 for the tools).
__global__ void k_wnorm(int n, const ull* idx, const float* w, float* wn, double* wn64, double* rowsum) {
    const long long u = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (u >= n) return;
    double s = 0;
    for (ull e = idx[u] + lane; e < idx[u + 1]; e += 32) s += w[e];
    s = warp_sum(s);
    s = __shfl_sync(FULL, s, 0);
    for (ull e = idx[u] + lane; e < idx[u + 1]; e += 32) {
        const double q = (double)w[e] / s;
        wn[e] = (float)q;
        wn64[e] = q;
    }
    if (lane == 0) rowsum[u] = s;
}

__global__ void k_wpermute(ull m, const unsigned* perm, const float* wn, const double* wn64, float* wt, double* wt64) {
    for (ull e = blockIdx.x * (ull)blockDim.x + threadIdx.x; e < m; e += (ull)gridDim.x * blockDim.x) {
        wt[e] = wn[perm[e]];
        wt64[e] = wn64[perm[e]];
    }
}

// Transposed CSR from keys (dst << scale | src) sorted with the original edge ids.
__global__ void k_wtrans(int n, int shift, ull m, const uint64_t* keys, int* adjT, ull* idxT) {
    const uint64_t mask = (1ull << shift) - 1;
    for (ull e = blockIdx.x * (ull)blockDim.x + threadIdx.x; e <= m; e += (ull)gridDim.x * blockDim.x) {
        const long long s = e < m ? (long long)(keys[e] >> shift) : n;
        const long long p = e > 0 ? (long long)(keys[e - 1] >> shift) : -1;
        if (e < m) adjT[e] = (int)(keys[e] & mask);
        for (long long v = p + 1; v <= s; v++) idxT[v] = e;
    }
}

__global__ void k_wkeys(int n, int shift, const ull* idx, const int* adj, uint64_t* keys, unsigned* vals) {
    const long long u = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (u >= n) return;
    for (ull e = idx[u] + lane; e < idx[u + 1]; e += 32) {
        keys[e] = ((uint64_t)adj[e] << shift) | (uint64_t)u;
        vals[e] = (unsigned)e;
    }
}

// Gradient through the row normalisation, one warp per row u.
__global__ void k_wgrad(int n, const ull* idx, const int* adj, const float* wn, const double* rowsum, const float* x,
                        const float* lam, float s, float* gw) {
    const long long u = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (u >= n) return;
    const double xu = x[u];
    double dot = 0;
    for (ull e = idx[u] + lane; e < idx[u + 1]; e += 32) dot += (double)wn[e] * s * xu * lam[adj[e]];
    dot = warp_sum(dot);
    dot = __shfl_sync(FULL, dot, 0);
    const double rs = rowsum[u];
    for (ull e = idx[u] + lane; e < idx[u + 1]; e += 32) gw[e] = (float)(((double)s * xu * lam[adj[e]] - dot) / rs);
}

__global__ void k_wscale(int n, const float* in, float f, float* out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        out[v] = f * in[v];
}

// FP64 pull: y_v = c * t_v + s * sum_e wt[e] x[adj[e]] over the lists of v;
// mx[0] = max |y - x|, mx[1] = max |y| as ordered bit patterns.
__global__ void k_wpull64(int n, const ull* idx, const int* adj, const double* wt, const double* x, const float* t,
                          double c, double s, double* y, ull* mx) {
    const long long v = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (v >= n) return;
    double acc = 0;
    for (ull e = idx[v] + lane; e < idx[v + 1]; e += 32) acc += wt[e] * x[adj[e]];
    acc = warp_sum(acc);
    if (lane == 0) {
        const double nv = c * (t ? (double)t[v] : 1.0) + s * acc;
        y[v] = nv;
        atomicMax(&mx[0], (ull)__double_as_longlong(fabs(nv - x[v])));
        atomicMax(&mx[1], (ull)__double_as_longlong(fabs(nv)));
    }
}

__global__ void k_wdot64(int n, const double* x, const float* c, double* out) {
    double a = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        a += x[v] * (double)c[v];
    a = warp_sum(a);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, a);
}

__global__ void k_wgrad64(int n, const ull* idx, const int* adj, const double* wn64, const double* rowsum,
                          const double* x, const double* lam, double s, double* gw) {
    const long long u = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (u >= n) return;
    double dot = 0;
    for (ull e = idx[u] + lane; e < idx[u + 1]; e += 32) dot += wn64[e] * s * x[u] * lam[adj[e]];
    dot = warp_sum(dot);
    dot = __shfl_sync(FULL, dot, 0);
    for (ull e = idx[u] + lane; e < idx[u + 1]; e += 32) gw[e] = (s * x[u] * lam[adj[e]] - dot) / rowsum[u];
}

}  // namespace excent

using namespace excent;

struct excent_wgraph {
    int dev = 0, sms = 0, n = 0;
    ull m = 0;
    const ull* d_idx = nullptr;   // caller's forward CSR
    const int* d_adj = nullptr;
    const float* d_wraw = nullptr;
    float* d_wn = nullptr;        // forward order
    double* d_wn64 = nullptr;
    double* d_rowsum = nullptr;
    ull* d_idxT = nullptr;
    int* d_adjT = nullptr;
    unsigned* d_perm = nullptr;   // transposed edge -> forward edge
    unsigned* d_inv = nullptr;    // forward edge -> transposed edge
    float* d_wt = nullptr;        // transposed order
    double* d_wt64 = nullptr;
    float *d_x = nullptr, *d_r = nullptr, *d_lam = nullptr;
    uint32_t* d_t[2] = {nullptr, nullptr};
    WCtrl* d_ctrl = nullptr;
    double *d_v64[2] = {nullptr, nullptr};
    ull* d_mx = nullptr;
    double* d_red = nullptr;
    cudaStream_t st = nullptr;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};  // forward, adjoint
    cudaGraph_t graph[2] = {nullptr, nullptr};
    int gmax[2] = {-1, -1};
    float geps[2] = {-1, -1}, gs[2] = {0, 0};
    int grid = 0;
    bool have_fwd = false;
    bool host_t = false;          // transposed lists and weights in pinned, mapped host memory
    int* h_adjT = nullptr;
    float* h_wt = nullptr;
    double* h_wt64 = nullptr;
    int fwd_kind = -1;
    double fwd_s = 0;
    ull launches = 0;
};

static void wg_drop_graphs(excent_wgraph* g) {
    for (int k = 0; k < 2; k++) {
        if (g->gexec[k]) cudaGraphExecDestroy(g->gexec[k]);
        if (g->graph[k]) cudaGraphDestroy(g->graph[k]);
        g->gexec[k] = nullptr;
        g->graph[k] = nullptr;
        g->gmax[k] = -1;
    }
}

static void wg_free(excent_wgraph* g) {
    cudaSetDevice(g->dev);
    cudaDeviceSynchronize();
    wg_drop_graphs(g);
    if (g->host_t) {
        cudaFreeHost(g->h_adjT);
        cudaFreeHost(g->h_wt);
        cudaFreeHost(g->h_wt64);
        g->d_adjT = nullptr; g->d_wt = nullptr; g->d_wt64 = nullptr;
    }
    void* ps[] = {g->d_wn, g->d_wn64, g->d_rowsum, g->d_idxT, g->d_adjT, g->d_perm, g->d_inv, g->d_wt, g->d_wt64,
                  g->d_x, g->d_r, g->d_lam, g->d_t[0], g->d_t[1], g->d_ctrl, g->d_v64[0], g->d_v64[1], g->d_mx,
                  g->d_red};
    for (void* p : ps) if (p) cudaFree(p);
    if (g->st) cudaStreamDestroy(g->st);
    delete g;
}

#define WG_ALLOC(ptr, bytes) do { if (cudaMalloc((void**)&(ptr), (bytes)) != cudaSuccess) { cudaGetLastError(); \
    ::excent::set_error("wgraph: device allocation of %llu bytes failed (%s)", (ull)(bytes), #ptr); return EXCENT_ERR_NOMEM; } } while (0)

static int wg_normalise(excent_wgraph* g) {
    const unsigned wb = (unsigned)(((long long)g->n * 32 + WB - 1) / WB);
    k_wnorm<<<wb, WB, 0, g->st>>>(g->n, g->d_idx, g->d_wraw, g->d_wn, g->d_wn64, g->d_rowsum);
    if (g->m) k_wpermute<<<2048, WB, 0, g->st>>>(g->m, g->d_perm, g->d_wn, g->d_wn64, g->d_wt, g->d_wt64);
    g->launches += 2;
    EX_CUDA(cudaGetLastError());
    EX_CUDA(cudaStreamSynchronize(g->st));
    g->have_fwd = false;
    return EXCENT_OK;
}

static int wg_setup(excent_wgraph* g, int device, int n, ull m, const ull* d_idx, const int* d_adj, const float* d_w) {
    EX_CUDA(cudaSetDevice(device));
    g->dev = device;
    EX_CUDA(cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, device));
    EX_CHECK_ARG(m < (1ull << 32), "weighted graphs are limited to 2^32 - 1 edges");
    g->n = n; g->m = m; g->d_idx = d_idx; g->d_adj = d_adj; g->d_wraw = d_w;
    EX_CUDA(cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking));
    const size_t me = std::max<ull>(m, 1);
    WG_ALLOC(g->d_wn, me * 4);
    WG_ALLOC(g->d_wn64, me * 8);
    WG_ALLOC(g->d_rowsum, (size_t)n * 8);
    WG_ALLOC(g->d_idxT, ((size_t)n + 1) * 8);
    WG_ALLOC(g->d_adjT, me * 4);
    WG_ALLOC(g->d_perm, me * 4);
    WG_ALLOC(g->d_inv, me * 4);
    WG_ALLOC(g->d_wt, me * 4);
    WG_ALLOC(g->d_wt64, me * 8);
    WG_ALLOC(g->d_x, (size_t)n * 4);
    WG_ALLOC(g->d_r, (size_t)n * 4);
    WG_ALLOC(g->d_lam, (size_t)n * 4);
    const size_t words = ((size_t)n + 31) / 32;
    WG_ALLOC(g->d_t[0], words * 4);
    WG_ALLOC(g->d_t[1], words * 4);
    WG_ALLOC(g->d_ctrl, sizeof(WCtrl));
    WG_ALLOC(g->d_mx, 2 * sizeof(ull));
    WG_ALLOC(g->d_red, sizeof(double));
    // transpose: sort (dst, src) keys carrying forward edge ids
    int shift = 1;
    while ((1ll << shift) < (long long)n) shift++;
    uint64_t *k0 = nullptr, *k1 = nullptr;
    unsigned *v0 = nullptr;
    void* tmp = nullptr;
    size_t tb = 0;
    int rc = EXCENT_OK;
    do {
        if (cudaMalloc(&k0, me * 8) != cudaSuccess || cudaMalloc(&k1, me * 8) != cudaSuccess ||
            cudaMalloc(&v0, me * 4) != cudaSuccess) {
            cudaGetLastError();
            set_error("wgraph: transpose scratch does not fit");
            rc = EXCENT_ERR_NOMEM;
            break;
        }
        const unsigned wb = (unsigned)(((long long)n * 32 + WB - 1) / WB);
        k_wkeys<<<wb, WB, 0, g->st>>>(n, shift, d_idx, d_adj, k0, v0);
        cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, v0, g->d_perm, (long long)m, 0, 2 * shift, g->st);
        if (cudaMalloc(&tmp, std::max<size_t>(tb, 16)) != cudaSuccess) {
            cudaGetLastError();
            set_error("wgraph: sort scratch does not fit");
            rc = EXCENT_ERR_NOMEM;
            break;
        }
        if (cub::DeviceRadixSort::SortPairs(tmp, tb, k0, k1, v0, g->d_perm, (long long)m, 0, 2 * shift, g->st) !=
            cudaSuccess) {
            set_error("wgraph: transpose sort failed");
            rc = EXCENT_ERR_CUDA;
            break;
        }
        k_wtrans<<<2048, WB, 0, g->st>>>(n, shift, m, k1, g->d_adjT, g->d_idxT);
        if (cudaStreamSynchronize(g->st) != cudaSuccess) { set_error("wgraph: transpose failed"); rc = EXCENT_ERR_CUDA; }
    } while (0);
    if (k0) cudaFree(k0);
    if (k1) cudaFree(k1);
    if (v0) cudaFree(v0);
    if (tmp) cudaFree(tmp);
    if (rc != EXCENT_OK) return rc;
    // inverse permutation (forward edge -> transposed edge), on the host once
    if (m) {
        std::vector<unsigned> perm(m), inv(m);
        EX_CUDA(cudaMemcpy(perm.data(), g->d_perm, m * 4, cudaMemcpyDeviceToHost));
        for (ull i = 0; i < m; i++) inv[perm[i]] = (unsigned)i;
        EX_CUDA(cudaMemcpy(g->d_inv, inv.data(), m * 4, cudaMemcpyHostToDevice));
    }
    int occ = 0;
    EX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_wpass, WB, 0));
    g->grid = g->sms * std::max(1, occ);
    return wg_normalise(g);
}

extern "C" int excent_wgraph_create(int device, int n, unsigned long long m, const unsigned long long* d_idx,
                                    const int32_t* d_adj, const float* d_w, excent_wgraph** out) {
    EX_CHECK_ARG(out && n >= 1 && d_idx && (m == 0 || (d_adj && d_w)), "bad argument");
    *out = nullptr;
    excent_wgraph* g = new excent_wgraph();
    const int rc = wg_setup(g, device, n, m, d_idx, d_adj, d_w);
    if (rc != EXCENT_OK) {
        std::string msg = get_error();
        wg_free(g);
        set_error("%s", msg.c_str());
        return rc;
    }
    *out = g;
    return EXCENT_OK;
}

extern "C" int excent_wgraph_destroy(excent_wgraph* g) {
    if (g) wg_free(g);
    return EXCENT_OK;
}

extern "C" int excent_wgraph_set_weights(excent_wgraph* g, const float* d_w) {
    EX_CHECK_ARG(g && (d_w || g->m == 0), "bad argument");
    EX_CUDA(cudaSetDevice(g->dev));
    g->d_wraw = d_w;
    return wg_normalise(g);
}

static WArgs wargs(excent_wgraph* g, bool transposed, float s, float eps, float* x, float* r) {
    WArgs a{};
    a.n = g->n;
    a.idx = transposed ? g->d_idxT : g->d_idx;
    a.adj = transposed ? g->d_adjT : g->d_adj;
    a.wt = transposed ? g->d_wt : g->d_wn;
    a.s = s; a.eps = eps; a.x = x; a.r = r;
    a.touched[0] = g->d_t[0]; a.touched[1] = g->d_t[1];
    a.words = (int)(((size_t)g->n + 31) / 32);
    a.ctrl = g->d_ctrl;
    return a;
}

// Delta-push to eps of the fixed point x = c0 * seed + s * (op) x; op = W^T
// (forward lists) or W (transposed lists). Result in x.
static int wg_push(excent_wgraph* g, bool transposed, float s, float eps, int max_passes, const float* seed, float c0,
                   float* x, int* passes, ull* pushed) {
    const size_t words = ((size_t)g->n + 31) / 32;
    EX_CUDA(cudaMemsetAsync(g->d_t[0], 0, words * 4, g->st));
    EX_CUDA(cudaMemsetAsync(g->d_t[1], 0, words * 4, g->st));
    k_wseed<<<g->sms * 8, WB, 0, g->st>>>(g->n, seed, c0, x, g->d_r, g->d_t[0]);
    g->launches++;
    WCtrl c{};
    c.max_passes = max_passes;
    EX_CUDA(cudaMemcpyAsync(g->d_ctrl, &c, sizeof c, cudaMemcpyHostToDevice, g->st));
    const int k = transposed ? 1 : 0;
    WArgs a = wargs(g, transposed, s, eps, x, g->d_r);
    if (!g->gexec[k] || g->gmax[k] != max_passes || g->geps[k] != eps || g->gs[k] != s) {
        if (g->gexec[k]) { cudaGraphExecDestroy(g->gexec[k]); g->gexec[k] = nullptr; }
        if (g->graph[k]) { cudaGraphDestroy(g->graph[k]); g->graph[k] = nullptr; }
        cudaGraph_t gr;
        EX_CUDA(cudaGraphCreate(&gr, 0));
        cudaGraphConditionalHandle h;
        EX_CUDA(cudaGraphConditionalHandleCreate(&h, gr, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        EX_CUDA(cudaGraphAddNode(&node, gr, nullptr, 0, &cp));
        cudaStream_t cs;
        EX_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        EX_CUDA(cudaStreamBeginCaptureToGraph(cs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal));
        k_wpass<<<g->grid, WB, 0, cs>>>(a);
        k_wend<<<1, 1, 0, cs>>>(g->d_ctrl, h, 1);
        cudaGraph_t captured;
        const cudaError_t ce = cudaStreamEndCapture(cs, &captured);
        cudaStreamDestroy(cs);
        EX_CUDA(ce);
        EX_CUDA(cudaGraphInstantiate(&g->gexec[k], gr, 0));
        g->graph[k] = gr;
        g->gmax[k] = max_passes;
        g->geps[k] = eps;
        g->gs[k] = s;
    }
    EX_CUDA(cudaGraphLaunch(g->gexec[k], g->st));
    EX_CUDA(cudaStreamSynchronize(g->st));
    EX_CUDA(cudaMemcpy(&c, g->d_ctrl, sizeof c, cudaMemcpyDeviceToHost));
    g->launches += 2ull * (c.pass + 1);
    if (passes) *passes = c.pass;
    if (pushed) *pushed = c.total_e;
    return EXCENT_OK;
}

extern "C" int excent_wgraph_forward(excent_wgraph* g, int kind, double s, const float* d_t, float eps, int max_passes,
                                     float* d_x_out, int* passes, unsigned long long* pushed) {
    EX_CHECK_ARG(g && (kind == EXCENT_PR || kind == EXCENT_KATZ) && eps > 0 && max_passes >= 1, "bad argument");
    EX_CUDA(cudaSetDevice(g->dev));
    const float c0 = kind == EXCENT_PR ? (float)(1.0 - s) : 1.f;
    EX_TRY(wg_push(g, false, (float)s, eps, max_passes, d_t, c0, g->d_x, passes, pushed));
    if (d_x_out) EX_CUDA(cudaMemcpy(d_x_out, g->d_x, (size_t)g->n * 4, cudaMemcpyDeviceToDevice));
    g->have_fwd = true;
    g->fwd_kind = kind;
    g->fwd_s = s;
    return EXCENT_OK;
}

extern "C" int excent_wgraph_vjp(excent_wgraph* g, const float* d_c, float eps, int max_passes, float* d_grad_t,
                                 float* d_grad_w, int* passes, unsigned long long* pushed) {
    EX_CHECK_ARG(g && d_c && eps > 0 && max_passes >= 1, "bad argument");
    EX_CHECK_ARG(g->have_fwd, "vjp needs a forward solve with the current weights first");
    EX_CUDA(cudaSetDevice(g->dev));
    const float s = (float)g->fwd_s;
    EX_TRY(wg_push(g, true, s, eps, max_passes, d_c, 1.f, g->d_lam, passes, pushed));
    if (d_grad_t) {
        const float f = g->fwd_kind == EXCENT_PR ? (float)(1.0 - g->fwd_s) : 1.f;
        k_wscale<<<g->sms * 8, WB, 0, g->st>>>(g->n, g->d_lam, f, d_grad_t);
        g->launches++;
    }
    if (d_grad_w && g->m) {
        const unsigned wb = (unsigned)(((long long)g->n * 32 + WB - 1) / WB);
        k_wgrad<<<wb, WB, 0, g->st>>>(g->n, g->d_idx, g->d_adj, g->d_wn, g->d_rowsum, g->d_x, g->d_lam, s, d_grad_w);
        g->launches++;
    }
    EX_CUDA(cudaGetLastError());
    EX_CUDA(cudaStreamSynchronize(g->st));
    return EXCENT_OK;
}

extern "C" int excent_wgraph_lambda(excent_wgraph* g, float* d_out) {
    EX_CHECK_ARG(g && d_out, "bad argument");
    EX_CUDA(cudaSetDevice(g->dev));
    EX_CUDA(cudaMemcpy(d_out, g->d_lam, (size_t)g->n * 4, cudaMemcpyDeviceToDevice));
    return EXCENT_OK;
}

// FP64 Jacobi of x = c0 * t + s * (op) x by pulls: the forward operator pulls
// over the transposed lists, the adjoint over the forward lists.
static int wg_jacobi64(excent_wgraph* g, bool adjoint, double s, double c0, const float* t, double tol, int maxit,
                       double* out_dev_sel) {
    const size_t n = g->n;
    for (auto& p : g->d_v64) if (!p) WG_ALLOC(p, n * 8);
    const unsigned wb = (unsigned)(((long long)n * 32 + WB - 1) / WB);
    // x0 = c0 * t
    EX_CUDA(cudaMemsetAsync(g->d_v64[0], 0, n * 8, g->st));
    double* x = g->d_v64[0];
    double* y = g->d_v64[1];
    const ull* idx = adjoint ? g->d_idx : g->d_idxT;
    const int* adj = adjoint ? g->d_adj : g->d_adjT;
    const double* w = adjoint ? g->d_wn64 : g->d_wt64;
    double rel = 1;
    for (int it = 0; it < maxit && rel > tol; it++) {
        EX_CUDA(cudaMemsetAsync(g->d_mx, 0, 2 * sizeof(ull), g->st));
        k_wpull64<<<wb, WB, 0, g->st>>>(g->n, idx, adj, w, x, t, c0, s, y, g->d_mx);
        ull h[2];
        EX_CUDA(cudaMemcpyAsync(h, g->d_mx, sizeof h, cudaMemcpyDeviceToHost, g->st));
        EX_CUDA(cudaStreamSynchronize(g->st));
        double d, mv;
        memcpy(&d, &h[0], 8);
        memcpy(&mv, &h[1], 8);
        rel = mv > 0 ? d / mv : 0;
        std::swap(x, y);
    }
    if (x != g->d_v64[0]) std::swap(g->d_v64[0], g->d_v64[1]);  // result in d_v64[0]
    (void)out_dev_sel;
    return EXCENT_OK;
}

// Set raw weight of forward edge e to w_e + delta (or restore), renormalising row u in FP64.
static int wg_perturb(excent_wgraph* g, long long e, double delta, int* u_out, std::vector<double>& saved) {
    std::vector<ull> idx(g->n + 1);
    EX_CUDA(cudaMemcpy(idx.data(), g->d_idx, (g->n + 1) * 8, cudaMemcpyDeviceToHost));
    const int u = (int)(std::upper_bound(idx.begin(), idx.end(), (ull)e) - idx.begin()) - 1;
    const ull b = idx[u], d = idx[u + 1] - b;
    std::vector<float> w(d);
    EX_CUDA(cudaMemcpy(w.data(), g->d_wraw + b, d * 4, cudaMemcpyDeviceToHost));
    saved.resize(d);
    EX_CUDA(cudaMemcpy(saved.data(), g->d_wn64 + b, d * 8, cudaMemcpyDeviceToHost));
    std::vector<double> wd(d), q(d);
    double rs = 0;
    for (ull i = 0; i < d; i++) { wd[i] = w[i] + (b + i == (ull)e ? delta : 0.0); rs += wd[i]; }
    for (ull i = 0; i < d; i++) q[i] = wd[i] / rs;
    EX_CUDA(cudaMemcpy(g->d_wn64 + b, q.data(), d * 8, cudaMemcpyHostToDevice));
    std::vector<unsigned> inv(d);
    EX_CUDA(cudaMemcpy(inv.data(), g->d_inv + b, d * 4, cudaMemcpyDeviceToHost));
    for (ull i = 0; i < d; i++) EX_CUDA(cudaMemcpy(g->d_wt64 + inv[i], &q[i], 8, cudaMemcpyDefault));
    *u_out = u;
    return EXCENT_OK;
}

static int wg_restore(excent_wgraph* g, int u, const std::vector<double>& saved) {
    ull b[2];
    EX_CUDA(cudaMemcpy(b, g->d_idx + u, 16, cudaMemcpyDeviceToHost));
    const ull d = b[1] - b[0];
    EX_CUDA(cudaMemcpy(g->d_wn64 + b[0], saved.data(), d * 8, cudaMemcpyHostToDevice));
    std::vector<unsigned> inv(d);
    EX_CUDA(cudaMemcpy(inv.data(), g->d_inv + b[0], d * 4, cudaMemcpyDeviceToHost));
    for (ull i = 0; i < d; i++) EX_CUDA(cudaMemcpy(g->d_wt64 + inv[i], &saved[i], 8, cudaMemcpyDefault));
    return EXCENT_OK;
}

extern "C" int excent_wgraph_loss_fp64(excent_wgraph* g, int kind, double s, const float* d_t, const float* d_c,
                                       long long edge, double delta, double tol, double* loss) {
    EX_CHECK_ARG(g && d_c && loss && (kind == EXCENT_PR || kind == EXCENT_KATZ), "bad argument");
    EX_CHECK_ARG(edge < (long long)g->m, "edge out of range");
    EX_CUDA(cudaSetDevice(g->dev));
    int u = -1;
    std::vector<double> saved;
    if (edge >= 0) EX_TRY(wg_perturb(g, edge, delta, &u, saved));
    const double c0 = kind == EXCENT_PR ? 1.0 - s : 1.0;
    const int rc = wg_jacobi64(g, false, s, c0, d_t, tol, 1000000, nullptr);
    if (edge >= 0) EX_TRY(wg_restore(g, u, saved));
    EX_TRY(rc);
    EX_CUDA(cudaMemsetAsync(g->d_red, 0, 8, g->st));
    k_wdot64<<<g->sms * 8, WB, 0, g->st>>>(g->n, g->d_v64[0], d_c, g->d_red);
    EX_CUDA(cudaMemcpyAsync(loss, g->d_red, 8, cudaMemcpyDeviceToHost, g->st));
    EX_CUDA(cudaStreamSynchronize(g->st));
    return EXCENT_OK;
}

extern "C" int excent_wgraph_grad_fp64(excent_wgraph* g, int kind, double s, const float* d_t, const float* d_c,
                                       double tol, double* grad_t, double* grad_w) {
    EX_CHECK_ARG(g && d_c && (kind == EXCENT_PR || kind == EXCENT_KATZ), "bad argument");
    EX_CUDA(cudaSetDevice(g->dev));
    const size_t n = g->n;
    const double c0 = kind == EXCENT_PR ? 1.0 - s : 1.0;
    EX_TRY(wg_jacobi64(g, false, s, c0, d_t, tol, 1000000, nullptr));
    double* xf = nullptr;
    WG_ALLOC(xf, n * 8);
    EX_CUDA(cudaMemcpy(xf, g->d_v64[0], n * 8, cudaMemcpyDeviceToDevice));
    int rc = wg_jacobi64(g, true, s, 1.0, d_c, tol, 1000000, nullptr);
    double* gw = nullptr;
    if (rc == EXCENT_OK && grad_t) {
        std::vector<double> lam(n);
        cudaMemcpy(lam.data(), g->d_v64[0], n * 8, cudaMemcpyDeviceToHost);
        for (size_t v = 0; v < n; v++) grad_t[v] = (kind == EXCENT_PR ? 1.0 - s : 1.0) * lam[v];
    }
    if (rc == EXCENT_OK && grad_w && g->m) {
        if (cudaMalloc(&gw, g->m * 8) != cudaSuccess) { cudaGetLastError(); set_error("grad buffer"); rc = EXCENT_ERR_NOMEM; }
        else {
            const unsigned wb = (unsigned)(((long long)n * 32 + WB - 1) / WB);
            k_wgrad64<<<wb, WB, 0, g->st>>>(g->n, g->d_idx, g->d_adj, g->d_wn64, g->d_rowsum, xf, g->d_v64[0], s, gw);
            if (cudaMemcpyAsync(grad_w, gw, g->m * 8, cudaMemcpyDeviceToHost, g->st) != cudaSuccess ||
                cudaStreamSynchronize(g->st) != cudaSuccess) { set_error("grad copy failed"); rc = EXCENT_ERR_CUDA; }
        }
    }
    cudaFree(xf);
    if (gw) cudaFree(gw);
    return rc;
}

extern "C" int excent_wgraph_stream(excent_wgraph* g, void** stream) {
    EX_CHECK_ARG(g && stream, "null argument");
    *stream = (void*)g->st;
    return EXCENT_OK;
}

// Move the transposed lists and weights to pinned, device-mapped host memory:
// the adjoint push then reads them in place over the host link (zero copy),
// the way the engine's host cache serves graphs larger than device memory.
extern "C" int excent_wgraph_host_transposed(excent_wgraph* g) {
    EX_CHECK_ARG(g, "null graph");
    if (g->host_t || g->m == 0) return EXCENT_OK;
    EX_CUDA(cudaSetDevice(g->dev));
    EX_CUDA(cudaDeviceSynchronize());
    wg_drop_graphs(g);
    const unsigned fl = cudaHostAllocMapped | cudaHostAllocPortable;
    int* ha = nullptr;
    float* hw = nullptr;
    double* hw64 = nullptr;
    if (cudaHostAlloc((void**)&ha, g->m * 4, fl) != cudaSuccess || cudaHostAlloc((void**)&hw, g->m * 4, fl) != cudaSuccess ||
        cudaHostAlloc((void**)&hw64, g->m * 8, fl) != cudaSuccess) {
        cudaGetLastError();
        if (ha) cudaFreeHost(ha);
        if (hw) cudaFreeHost(hw);
        if (hw64) cudaFreeHost(hw64);
        EX_FAIL(EXCENT_ERR_NOMEM, "pinned host copy of the transposed graph does not fit");
    }
    EX_CUDA(cudaMemcpy(ha, g->d_adjT, g->m * 4, cudaMemcpyDeviceToHost));
    EX_CUDA(cudaMemcpy(hw, g->d_wt, g->m * 4, cudaMemcpyDeviceToHost));
    EX_CUDA(cudaMemcpy(hw64, g->d_wt64, g->m * 8, cudaMemcpyDeviceToHost));
    cudaFree(g->d_adjT);
    cudaFree(g->d_wt);
    cudaFree(g->d_wt64);
    g->h_adjT = ha; g->h_wt = hw; g->h_wt64 = hw64;
    EX_CUDA(cudaHostGetDevicePointer((void**)&g->d_adjT, ha, 0));
    EX_CUDA(cudaHostGetDevicePointer((void**)&g->d_wt, hw, 0));
    EX_CUDA(cudaHostGetDevicePointer((void**)&g->d_wt64, hw64, 0));
    g->host_t = true;
    return EXCENT_OK;
}
