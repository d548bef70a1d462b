// rmat.cu -- seeded R-MAT graph generator on the device, written from the
// recursive-quadrant definition of R-MAT: each edge descends `scale` levels,
// picking quadrant (0,0), (0,1), (1,0), (1,1) with probabilities a, b, c, d.
// Symmetric graphs add both directions; self-loops and duplicates are
// dropped and each adjacency list is sorted (CSR from a radix sort of
// (src, dst) keys). Directed graphs keep one direction. Optional per-edge
// weights are float32 uniform on [0.5, 1.5) in steps of 2^-24.
//
// Random stream: splitmix64 outputs mix64(key + (c + 1) * 0x9E3779B97F4A7C15)
// for counter c, key = mix64(seed * 0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019).
// Pair i, level l uses half (l & 1) of counter i * ceil(scale / 2) + l / 2.
// The graph is setup input, not the measured path; the sort uses CUB.
#include <cub/cub.cuh>
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <vector>

#include "common.h"

namespace excent {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t rng64(uint64_t key, uint64_t c) {
    return mix64(key + (c + 1) * 0x9E3779B97F4A7C15ull);
}
static uint64_t rmat_key(uint64_t seed) { return mix64(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull); }

static constexpr uint64_t NONE = ~0ull;

// Pair i: source r and destination c after `scale` quadrant choices.
__device__ __forceinline__ void rmat_pair(int scale, ull i, uint64_t key, uint32_t tA, uint32_t tAB, uint32_t tABC,
                                          uint32_t& r, uint32_t& c) {
    const ull W = (ull)(scale + 1) / 2;
    r = 0; c = 0;
    uint64_t h = 0;
    for (int l = 0; l < scale; l++) {
        if ((l & 1) == 0) h = rng64(key, i * W + (ull)(l >> 1));
        const uint32_t u = (l & 1) ? (uint32_t)(h >> 32) : (uint32_t)h;
        const uint32_t bit = 1u << (scale - 1 - l);
        if (u < tA) {
        } else if (u < tAB) c |= bit;
        else if (u < tABC) r |= bit;
        else { r |= bit; c |= bit; }
    }
}

__global__ void k_rmat_keys(int scale, ull npairs, uint64_t key, uint32_t tA, uint32_t tAB, uint32_t tABC, int sym,
                            uint64_t* keys) {
    for (ull i = blockIdx.x * (ull)blockDim.x + threadIdx.x; i < npairs; i += (ull)gridDim.x * blockDim.x) {
        uint32_t r, c;
        rmat_pair(scale, i, key, tA, tAB, tABC, r, c);
        const bool self = r == c;
        if (sym) {
            keys[2 * i] = self ? NONE : ((uint64_t)r << scale) | c;
            keys[2 * i + 1] = self ? NONE : ((uint64_t)c << scale) | r;
        } else {
            keys[i] = self ? NONE : ((uint64_t)r << scale) | c;
        }
    }
}

// Histogram of the source vertices of both directions of every non-loop pair,
// by source >> shift (HBINS buckets).
static constexpr int HBINS = 4096;
__global__ void k_rmat_hist(int scale, ull npairs, uint64_t key, uint32_t tA, uint32_t tAB, uint32_t tABC, int shift,
                            ull* hist) {
    __shared__ unsigned h[HBINS];
    for (int i = threadIdx.x; i < HBINS; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (ull i = blockIdx.x * (ull)blockDim.x + threadIdx.x; i < npairs; i += (ull)gridDim.x * blockDim.x) {
        uint32_t r, c;
        rmat_pair(scale, i, key, tA, tAB, tABC, r, c);
        if (r != c) { atomicAdd(&h[r >> shift], 1u); atomicAdd(&h[c >> shift], 1u); }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < HBINS; i += blockDim.x)
        if (h[i]) atomicAdd(hist + i, (ull)h[i]);
}

// The keys (both directions, no loops) whose source lies in [s_lo, s_hi),
// appended in any order with one atomic per warp.
__global__ void k_rmat_part(int scale, ull npairs, uint64_t key, uint32_t tA, uint32_t tAB, uint32_t tABC,
                            uint32_t s_lo, uint32_t s_hi, uint64_t* out, ull* cnt, ull cap) {
    const int lane = threadIdx.x & 31;
    const ull stride = (ull)gridDim.x * blockDim.x;
    // every lane of a warp runs the same number of iterations (the bound is rounded up to the warp)
    const ull bound = (npairs + 31) / 32 * 32;
    for (ull i = blockIdx.x * (ull)blockDim.x + threadIdx.x; i < bound; i += stride) {
        uint32_t r = 0, c = 0;
        if (i < npairs) rmat_pair(scale, i, key, tA, tAB, tABC, r, c);
        const bool ok = i < npairs && r != c;
        const bool k0 = ok && r >= s_lo && r < s_hi, k1 = ok && c >= s_lo && c < s_hi;
        const unsigned b0 = __ballot_sync(0xffffffffu, k0), b1 = __ballot_sync(0xffffffffu, k1);
        const unsigned tot = __popc(b0) + __popc(b1);
        ull base = 0;
        if (lane == 0 && tot) base = atomicAdd(cnt, (ull)tot);
        base = __shfl_sync(0xffffffffu, base, 0);
        const unsigned lt = (1u << lane) - 1u;
        if (k0) { const ull p = base + __popc(b0 & lt); if (p < cap) out[p] = ((uint64_t)r << scale) | c; }
        if (k1) { const ull p = base + __popc(b0) + __popc(b1 & lt); if (p < cap) out[p] = ((uint64_t)c << scale) | r; }
    }
}

// CSR of one source partition from its sorted unique keys: adj[e] = dst,
// idx[v - s_lo] = base + first entry of v, for v in [s_lo, s_hi).
__global__ void k_csr_part(int scale, ull m, const uint64_t* keys, int* adj, ull* idx, uint32_t s_lo, uint32_t s_hi,
                           ull base) {
    const uint64_t mask = (1ull << scale) - 1;
    for (ull e = blockIdx.x * (ull)blockDim.x + threadIdx.x; e <= m; e += (ull)gridDim.x * blockDim.x) {
        const long long s = e < m ? (long long)(keys[e] >> scale) : (long long)s_hi;
        const long long p = e > 0 ? (long long)(keys[e - 1] >> scale) : (long long)s_lo - 1;
        if (e < m) adj[e] = (int)(keys[e] & mask);
        for (long long v = p + 1; v <= s && v < (long long)s_hi; v++) idx[v - s_lo] = base + e;
    }
}

// CSR from sorted unique keys: adj[e] = dst, idx[v] = first edge of v.
__global__ void k_csr(int scale, ull m, const uint64_t* keys, int* adj, ull* idx, int n) {
    const uint64_t mask = (1ull << scale) - 1;
    for (ull e = blockIdx.x * (ull)blockDim.x + threadIdx.x; e <= m; e += (ull)gridDim.x * blockDim.x) {
        const long long s = e < m ? (long long)(keys[e] >> scale) : n;
        const long long p = e > 0 ? (long long)(keys[e - 1] >> scale) : -1;
        if (e < m) adj[e] = (int)(keys[e] & mask);
        for (long long v = p + 1; v <= s; v++) idx[v] = e;
    }
}

__global__ void k_weights(ull m, uint64_t key, float* w) {
    for (ull e = blockIdx.x * (ull)blockDim.x + threadIdx.x; e < m; e += (ull)gridDim.x * blockDim.x)
        w[e] = 0.5f + (float)(rng64(key, e) >> 40) * (1.0f / 16777216.0f);
}

}  // namespace excent

using namespace excent;

struct excent_dgraph {
    int dev = 0;
    int n = 0;
    ull m = 0;
    ull* d_idx = nullptr;
    int* d_adj = nullptr;
    float* d_w = nullptr;
};

extern "C" int excent_dgraph_destroy(excent_dgraph* g) {
    if (!g) return EXCENT_OK;
    cudaSetDevice(g->dev);
    if (g->d_idx) cudaFree(g->d_idx);
    if (g->d_adj) cudaFree(g->d_adj);
    if (g->d_w) cudaFree(g->d_w);
    delete g;
    return EXCENT_OK;
}

static int rmat_impl(excent_dgraph* g, int scale, int edge_factor, ull seed, double a, double b, double c,
                     int symmetric, int weights) {
    const int n = 1 << scale;
    const ull npairs = symmetric ? (ull)n * edge_factor / 2 : (ull)n * edge_factor;
    const ull nkeys = symmetric ? 2 * npairs : npairs;
    const uint32_t tA = (uint32_t)(a * 4294967296.0), tAB = (uint32_t)((a + b) * 4294967296.0),
                   tABC = (uint32_t)((a + b + c) * 4294967296.0);
    uint64_t *k0 = nullptr, *k1 = nullptr;
    void* tmp = nullptr;
    ull* d_m = nullptr;
    int rc = EXCENT_OK;
    size_t tb_sort = 0, tb_uniq = 0;
    auto fail = [&](const char* what, cudaError_t err) {
        set_error("rmat: %s failed (%s)", what, cudaGetErrorString(err));
        rc = err == cudaErrorMemoryAllocation ? EXCENT_ERR_NOMEM : EXCENT_ERR_CUDA;
    };
    cudaError_t err;
    do {
        if ((err = cudaMalloc(&k0, nkeys * 8)) != cudaSuccess) { fail("key allocation", err); break; }
        if ((err = cudaMalloc(&k1, nkeys * 8)) != cudaSuccess) { fail("key allocation", err); break; }
        if ((err = cudaMalloc(&d_m, 8)) != cudaSuccess) { fail("counter allocation", err); break; }
        k_rmat_keys<<<2048, 256>>>(scale, npairs, rmat_key(seed), tA, tAB, tABC, symmetric, k0);
        cub::DeviceRadixSort::SortKeys(nullptr, tb_sort, k0, k1, (long long)nkeys, 0, 2 * scale);
        cub::DeviceSelect::Unique(nullptr, tb_uniq, k1, k0, d_m, (long long)nkeys);
        if ((err = cudaMalloc(&tmp, std::max(tb_sort, tb_uniq))) != cudaSuccess) { fail("sort scratch", err); break; }
        // keys use 2*scale bits; self loops are all ones and sort last
        if ((err = cub::DeviceRadixSort::SortKeys(tmp, tb_sort, k0, k1, (long long)nkeys, 0, 2 * scale)) != cudaSuccess) {
            fail("sort", err); break;
        }
        if ((err = cub::DeviceSelect::Unique(tmp, tb_uniq, k1, k0, d_m, (long long)nkeys)) != cudaSuccess) {
            fail("unique", err); break;
        }
        ull mu = 0;
        if ((err = cudaMemcpy(&mu, d_m, 8, cudaMemcpyDeviceToHost)) != cudaSuccess) { fail("copy", err); break; }
        uint64_t last = 0;
        if (mu && (err = cudaMemcpy(&last, k0 + mu - 1, 8, cudaMemcpyDeviceToHost)) != cudaSuccess) { fail("copy", err); break; }
        if (mu && last == NONE) mu--;
        g->n = n;
        g->m = mu;
        if ((err = cudaMalloc(&g->d_idx, ((size_t)n + 1) * 8)) != cudaSuccess) { fail("offsets", err); break; }
        if ((err = cudaMalloc(&g->d_adj, std::max<ull>(mu, 1) * 4)) != cudaSuccess) { fail("lists", err); break; }
        k_csr<<<2048, 256>>>(scale, mu, k0, g->d_adj, g->d_idx, n);
        if (weights) {
            if ((err = cudaMalloc(&g->d_w, std::max<ull>(mu, 1) * 4)) != cudaSuccess) { fail("weights", err); break; }
            k_weights<<<2048, 256>>>(mu, rmat_key(seed ^ 0x5745494748545321ull), g->d_w);
        }
        if ((err = cudaDeviceSynchronize()) != cudaSuccess) { fail("generation", err); break; }
    } while (0);
    if (k0) cudaFree(k0);
    if (k1) cudaFree(k1);
    if (tmp) cudaFree(tmp);
    if (d_m) cudaFree(d_m);
    return rc;
}

extern "C" int excent_rmat_generate(int device, int scale, int edge_factor, unsigned long long seed, double a,
                                    double b, double c, int symmetric, int weights, excent_dgraph** out) {
    EX_CHECK_ARG(out, "null output");
    EX_CHECK_ARG(scale >= 1 && scale <= 30, "scale must be 1..30");
    EX_CHECK_ARG(edge_factor >= 1, "edge factor must be >= 1");
    EX_CHECK_ARG(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0, "bad R-MAT probabilities");
    *out = nullptr;
    EX_CUDA(cudaSetDevice(device));
    excent_dgraph* g = new excent_dgraph();
    g->dev = device;
    const int rc = rmat_impl(g, scale, edge_factor, seed, a, b, c, symmetric, weights);
    if (rc != EXCENT_OK) {
        std::string msg = get_error();
        excent_dgraph_destroy(g);
        set_error("%s", msg.c_str());
        return rc;
    }
    *out = g;
    return EXCENT_OK;
}

extern "C" int excent_dgraph_info(excent_dgraph* g, int* n, unsigned long long* m) {
    EX_CHECK_ARG(g, "null graph");
    if (n) *n = g->n;
    if (m) *m = g->m;
    return EXCENT_OK;
}

extern "C" int excent_dgraph_device_ptrs(excent_dgraph* g, unsigned long long** idx, int32_t** adj, float** w) {
    EX_CHECK_ARG(g, "null graph");
    if (idx) *idx = g->d_idx;
    if (adj) *adj = g->d_adj;
    if (w) *w = g->d_w;
    return EXCENT_OK;
}

extern "C" int excent_dgraph_download(excent_dgraph* g, unsigned long long* idx, int32_t* adj, float* w) {
    EX_CHECK_ARG(g, "null graph");
    EX_CUDA(cudaSetDevice(g->dev));
    if (idx) EX_CUDA(cudaMemcpy(idx, g->d_idx, ((size_t)g->n + 1) * 8, cudaMemcpyDeviceToHost));
    if (adj && g->m) EX_CUDA(cudaMemcpy(adj, g->d_adj, g->m * 4, cudaMemcpyDeviceToHost));
    if (w) {
        EX_CHECK_ARG(g->d_w, "graph has no weights");
        if (g->m) EX_CUDA(cudaMemcpy(w, g->d_w, g->m * 4, cudaMemcpyDeviceToHost));
    }
    return EXCENT_OK;
}

static bool write_all(int fd, const void* buf, size_t bytes, off_t off) {
    const char* p = static_cast<const char*>(buf);
    while (bytes) {
        const ssize_t w = pwrite(fd, p, std::min<size_t>(bytes, (size_t)1 << 30), off);
        if (w <= 0) return false;
        p += w; off += w; bytes -= (size_t)w;
    }
    return true;
}

extern "C" int excent_rmat_write_egr(int device, int scale, int edge_factor, unsigned long long seed, double a,
                                     double b, double c, unsigned long long max_part_keys, const char* path,
                                     unsigned long long* m_out, int* parts_out) {
    EX_CHECK_ARG(path, "null path");
    EX_CHECK_ARG(scale >= 1 && scale <= 30, "scale must be 1..30");
    EX_CHECK_ARG(edge_factor >= 1, "edge factor must be >= 1");
    EX_CHECK_ARG(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0, "bad R-MAT probabilities");
    EX_CUDA(cudaSetDevice(device));
    const int n = 1 << scale;
    const ull npairs = (ull)n * edge_factor / 2;
    const uint32_t tA = (uint32_t)(a * 4294967296.0), tAB = (uint32_t)((a + b) * 4294967296.0),
                   tABC = (uint32_t)((a + b + c) * 4294967296.0);
    const uint64_t key = rmat_key(seed);
    const int shift = scale > 12 ? scale - 12 : 0;
    const int nbins = n >> shift;
    // 1. keys per source bucket
    ull* d_hist = nullptr;
    EX_CUDA(cudaMalloc(&d_hist, HBINS * sizeof(ull)));
    std::vector<ull> hist(HBINS);
    cudaError_t err = cudaMemset(d_hist, 0, HBINS * sizeof(ull));
    if (err == cudaSuccess) {
        k_rmat_hist<<<2048, 256>>>(scale, npairs, key, tA, tAB, tABC, shift, d_hist);
        err = cudaMemcpy(hist.data(), d_hist, HBINS * sizeof(ull), cudaMemcpyDeviceToHost);
    }
    cudaFree(d_hist);
    EX_CUDA(err);
    // 2. partition size: two key buffers, sort scratch, this partition's offsets
    ull cap = max_part_keys;
    if (!cap) {
        size_t fr = 0, tot = 0;
        EX_CUDA(cudaMemGetInfo(&fr, &tot));
        const double usable = (double)fr * 0.85 - (double)n * 8 - (1u << 30);
        EX_CHECK_ARG(usable > 0, "not enough device memory");
        cap = (ull)(usable / 26.0);   // 8 + 8 key bytes, ~8 sort scratch, margin
    }
    ull biggest = 0;
    for (int i = 0; i < nbins; i++) biggest = std::max(biggest, hist[i]);
    EX_CHECK_ARG(biggest <= cap, "a source bucket holds %llu keys, above the partition size %llu", biggest, cap);
    std::vector<int> cut{0};   // partition p covers buckets [cut[p], cut[p+1])
    {
        ull acc = 0;
        for (int i = 0; i < nbins; i++) {
            if (acc + hist[i] > cap) { cut.push_back(i); acc = 0; }
            acc += hist[i];
        }
        cut.push_back(nbins);
    }
    const int parts = (int)cut.size() - 1;
    ull maxk = 0, maxr = 0;
    for (int p = 0; p < parts; p++) {
        ull k = 0;
        for (int i = cut[p]; i < cut[p + 1]; i++) k += hist[i];
        maxk = std::max(maxk, k);
        maxr = std::max(maxr, (ull)(cut[p + 1] - cut[p]) << shift);
    }
    maxk = std::max<ull>(maxk, 1);
    const int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    EX_CHECK_ARG(fd >= 0, "cannot create %s", path);
    uint64_t *k0 = nullptr, *k1 = nullptr;
    ull *d_cnt = nullptr, *d_idx = nullptr;
    void* tmp = nullptr;
    int rc = EXCENT_OK;
    auto fail = [&](int code, const char* what, cudaError_t e2) {
        if (code == EXCENT_ERR_IO) set_error("rmat egr: writing %s failed", path);
        else set_error("rmat egr: %s failed (%s)", what, cudaGetErrorString(e2));
        rc = e2 == cudaErrorMemoryAllocation ? EXCENT_ERR_NOMEM : code;
    };
    ull m = 0;
    const off_t adj_off = 16 + (off_t)8 * ((off_t)n + 1);
    do {
        size_t tb_sort = 0, tb_uniq = 0;
        if ((err = cudaMalloc(&k0, maxk * 8)) != cudaSuccess) { fail(EXCENT_ERR_CUDA, "key allocation", err); break; }
        if ((err = cudaMalloc(&k1, maxk * 8)) != cudaSuccess) { fail(EXCENT_ERR_CUDA, "key allocation", err); break; }
        if ((err = cudaMalloc(&d_cnt, 8)) != cudaSuccess) { fail(EXCENT_ERR_CUDA, "counter allocation", err); break; }
        if ((err = cudaMalloc(&d_idx, maxr * 8)) != cudaSuccess) { fail(EXCENT_ERR_CUDA, "offset allocation", err); break; }
        cub::DeviceRadixSort::SortKeys(nullptr, tb_sort, k0, k1, (long long)maxk, 0, 2 * scale);
        cub::DeviceSelect::Unique(nullptr, tb_uniq, k1, k0, d_cnt, (long long)maxk);
        if ((err = cudaMalloc(&tmp, std::max(tb_sort, tb_uniq))) != cudaSuccess) { fail(EXCENT_ERR_CUDA, "sort scratch", err); break; }
        std::vector<int> h_adj;
        std::vector<ull> h_idx;
        for (int p = 0; p < parts && rc == EXCENT_OK; p++) {
            const uint32_t s_lo = (uint32_t)cut[p] << shift, s_hi = (uint32_t)((ull)cut[p + 1] << shift);
            ull k = 0;
            for (int i = cut[p]; i < cut[p + 1]; i++) k += hist[i];
            if ((err = cudaMemset(d_cnt, 0, 8)) != cudaSuccess) { fail(EXCENT_ERR_CUDA, "memset", err); break; }
            k_rmat_part<<<4096, 256>>>(scale, npairs, key, tA, tAB, tABC, s_lo, s_hi, k0, d_cnt, maxk);
            if ((err = cub::DeviceRadixSort::SortKeys(tmp, tb_sort, k0, k1, (long long)k, 0, 2 * scale)) != cudaSuccess) {
                fail(EXCENT_ERR_CUDA, "sort", err); break;
            }
            if ((err = cub::DeviceSelect::Unique(tmp, tb_uniq, k1, k0, d_cnt, (long long)k)) != cudaSuccess) {
                fail(EXCENT_ERR_CUDA, "unique", err); break;
            }
            ull mu = 0;
            if ((err = cudaMemcpy(&mu, d_cnt, 8, cudaMemcpyDeviceToHost)) != cudaSuccess) { fail(EXCENT_ERR_CUDA, "copy", err); break; }
            int* d_adjp = reinterpret_cast<int*>(k1);   // k1 is free after the unique
            k_csr_part<<<2048, 256>>>(scale, mu, k0, d_adjp, d_idx, s_lo, s_hi, m);
            h_adj.resize(std::max<ull>(mu, 1));
            h_idx.resize(s_hi - s_lo);
            if ((err = cudaMemcpy(h_adj.data(), d_adjp, mu * 4, cudaMemcpyDeviceToHost)) != cudaSuccess) {
                fail(EXCENT_ERR_CUDA, "download", err); break;
            }
            if ((err = cudaMemcpy(h_idx.data(), d_idx, (size_t)(s_hi - s_lo) * 8, cudaMemcpyDeviceToHost)) != cudaSuccess) {
                fail(EXCENT_ERR_CUDA, "download", err); break;
            }
            if (!write_all(fd, h_adj.data(), mu * 4, adj_off + (off_t)4 * (off_t)m) ||
                !write_all(fd, h_idx.data(), (size_t)(s_hi - s_lo) * 8, 16 + (off_t)8 * s_lo)) {
                fail(EXCENT_ERR_IO, "", cudaSuccess); break;
            }
            m += mu;
        }
        if (rc != EXCENT_OK) break;
        int32_t head[2] = {n, -1};
        const int64_t mm = (int64_t)m;
        const ull last = m;
        if (!write_all(fd, head, 8, 0) || !write_all(fd, &mm, 8, 8) || !write_all(fd, &last, 8, 16 + (off_t)8 * n) ||
            fsync(fd) != 0) {
            fail(EXCENT_ERR_IO, "", cudaSuccess);
        }
    } while (0);
    close(fd);
    if (k0) cudaFree(k0);
    if (k1) cudaFree(k1);
    if (d_cnt) cudaFree(d_cnt);
    if (d_idx) cudaFree(d_idx);
    if (tmp) cudaFree(tmp);
    if (rc == EXCENT_OK) {
        if (m_out) *m_out = m;
        if (parts_out) *parts_out = parts;
    }
    return rc;
}
