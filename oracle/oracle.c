/*
 * oracle.c -- CPU restatement of the ExCent delta-push centrality path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker: only the test suite, the
 * smoke check and the CPU-baseline leg of the benchmark load it. The product
 * (libexcent_b200.so and the excent CLI) never links, loads or calls it.
 *
 * Every function restates one piece of the reference (SPADE-IITJ/ExCent) and
 * cites the file:line it follows. Paths are relative to the reference project.
 *   - FP64 Jacobi / power-iteration oracle:   tools/centrality_reference.cu:31-59, 184-214
 *   - given constants (lambda1, means):       tools/excent_params.cu:133-163
 *   - engine init and push semantics:         src/excent.cu:41-124
 *   - demand snapshot:                        src/excent.cu:49-98
 *   - fetch plan:                             src/excent.cu:666-678
 *   - gather list build:                      src/excent.cu:711-730
 *   - chunk planner:                          include/StaticGraph.h:128-139, src/excent.cu:321-327
 *   - gather page-run dedup:                  include/StaticGraph.h:90-114
 *   - GPU cache sizing (chunks / hot):        src/excent.cu:400-513
 *   - stream/gather crossover tau:            src/excent.cu:566-572
 * Things the reference does not have (batched PPR, the adjoint, the R-MAT
 * generator) are restated from their mathematical definitions.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -shared -fPIC).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef unsigned long long ull;

/* ------------------------------------------------------------------ R-MAT */

/* splitmix64 finalizer; the generator's counter-based stream is
 * mix64(key + (c + 1) * golden) for counter c. */
static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline uint64_t rng64(uint64_t key, uint64_t c) { return mix64(key + (c + 1) * 0x9E3779B97F4A7C15ull); }
uint64_t or_rmat_key(uint64_t seed) { return mix64(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull); }

/* R-MAT pair i: `scale` levels, each picks a quadrant of the adjacency matrix
 * from one 32-bit uniform u: u < tA -> (0,0), u < tAB -> (0,1), u < tABC -> (1,0),
 * else (1,1). Level l sets bit (scale-1-l) of (row, col). Level l draws half
 * (l & 1) of rng64(key, i * W + l / 2), W = (scale + 1) / 2. */
void or_rmat_pairs(int scale, ull npairs, uint64_t seed, uint32_t tA, uint32_t tAB, uint32_t tABC,
                   int32_t* src, int32_t* dst) {
    const uint64_t key = or_rmat_key(seed);
    const ull W = (ull)(scale + 1) / 2;
    #pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)npairs; i++) {
        uint32_t r = 0, c = 0;
        uint64_t h = 0;
        for (int l = 0; l < scale; l++) {
            if ((l & 1) == 0) h = rng64(key, (ull)i * W + (ull)(l >> 1));
            const uint32_t u = (l & 1) ? (uint32_t)(h >> 32) : (uint32_t)h;
            const uint32_t bit = 1u << (scale - 1 - l);
            if (u < tA) {}
            else if (u < tAB) c |= bit;
            else if (u < tABC) r |= bit;
            else { r |= bit; c |= bit; }
        }
        src[i] = (int32_t)r;
        dst[i] = (int32_t)c;
    }
}

/* Edge weights: float32 uniform on [0.5, 1.5) in steps of 2^-24, edge e in CSR order. */
void or_rmat_weights(ull m, uint64_t seed, float* w) {
    const uint64_t key = or_rmat_key(seed ^ 0x5745494748545321ull);
    #pragma omp parallel for schedule(static)
    for (long long e = 0; e < (long long)m; e++)
        w[e] = 0.5f + (float)(rng64(key, (ull)e) >> 40) * (1.0f / 16777216.0f);
}

/* ------------------------------------------------------- FP64 Jacobi oracle */

/* y[w] = c + s * sum_{u in N(w)} x[u] (/ L(u) if divdeg); stop when
 * max|y - x| / max|y| < tol or after maxit sweeps. Restates
 * tools/centrality_reference.cu:31-49 (k_step) and :184-195, 208-213 (loop).
 * x0 = 0.15 for PageRank and 1.0 otherwise (:184). Pull over CSR lists, so the
 * graph must be symmetric (:3-4). Returns the number of sweeps. */
int or_jacobi(int n, const ull* idx, const int32_t* adj, double c, double s, int divdeg,
              double x0, double tol, int maxit, double* x_out, double* rel_out) {
    double* x = (double*)malloc(sizeof(double) * (size_t)n);
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) x[i] = x0;
    int it = 0; double rel = 1;
    for (; it < maxit && rel > tol; it++) {
        double mx0 = 0, mx1 = 0;
        #pragma omp parallel for schedule(dynamic, 1024) reduction(max : mx0, mx1)
        for (int w = 0; w < n; w++) {
            double acc = 0;
            for (ull e = idx[w]; e < idx[w + 1]; e++) {
                int u = adj[e];
                acc += divdeg ? x[u] / (double)(idx[u + 1] - idx[u]) : x[u];
            }
            double nv = c + s * acc;
            y[w] = nv;
            double d = fabs(nv - x[w]);
            if (d > mx0) mx0 = d;
            if (fabs(nv) > mx1) mx1 = fabs(nv);
        }
        rel = mx0 / mx1;
        double* t = x; x = y; y = t;
    }
    memcpy(x_out, x, sizeof(double) * (size_t)n);
    if (rel_out) *rel_out = rel;
    free(x); free(y);
    return it;
}

/* unit L2 norm with the sign fixed by the sum: tools/centrality_reference.cu:71-76 */
void or_unit(int n, double* v) {
    double s = 0, t = 0;
    for (int i = 0; i < n; i++) { s += v[i] * v[i]; t += v[i]; }
    double f = (t < 0 ? -1.0 : 1.0) / sqrt(s);
    for (int i = 0; i < n; i++) v[i] *= f;
}

/* Eigenvector oracle: x0 = 1, y = A x, y /= ||y||, rel = max|x - y|; the first
 * sweep is sign-fixed and forces rel = 1. tools/centrality_reference.cu:193-207. */
int or_power(int n, const ull* idx, const int32_t* adj, double tol, int maxit, double* x_out, double* lam_out) {
    double* x = (double*)malloc(sizeof(double) * (size_t)n);
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) x[i] = 1.0;
    int it = 0; double rel = 1, lam = 0;
    for (; it < maxit && rel > tol; it++) {
        double ss = 0;
        #pragma omp parallel for schedule(dynamic, 1024) reduction(+ : ss)
        for (int w = 0; w < n; w++) {
            double acc = 0;
            for (ull e = idx[w]; e < idx[w + 1]; e++) acc += x[adj[e]];
            y[w] = acc;
            ss += acc * acc;
        }
        lam = sqrt(ss);
        double mx = 0;
        #pragma omp parallel for schedule(static) reduction(max : mx)
        for (int w = 0; w < n; w++) {
            y[w] *= 1.0 / lam;
            double d = fabs(x[w] - y[w]);
            if (d > mx) mx = d;
        }
        rel = mx;
        if (it == 0) { or_unit(n, y); rel = 1; }
        double* t = x; x = y; y = t;
    }
    memcpy(x_out, x, sizeof(double) * (size_t)n);
    if (lam_out) *lam_out = lam;
    free(x); free(y);
    return it;
}

/* ------------------------------------------------------- given constants */

/* lambda1 by power iteration from the unit all-ones vector, stopping when
 * |lam - lamPrev| / lam < 1e-12 after 10 sweeps (<= 5000); eigenvector mean
 * (v1 . 1)^2 / n; Katz alpha = 0.85 / lambda1, beta = 1 and the Katz fixed
 * point's mean (stop at relative mean change < 1e-12, <= 5000).
 * Restates tools/excent_params.cu:133-163. out = {lambda, alpha, meanEV, meanK, pit}. */
void or_params(int n, const ull* idx, const int32_t* adj, double* out) {
    double* v0 = (double*)malloc(sizeof(double) * (size_t)n);
    double* v1 = (double*)malloc(sizeof(double) * (size_t)n);
    double nrm = sqrt((double)n);
    for (int i = 0; i < n; i++) v0[i] = 1.0 / nrm;
    double lam = 0, lamPrev = 0;
    int pit = 0;
    for (; pit < 5000; pit++) {
        double ss = 0;
        #pragma omp parallel for schedule(dynamic, 1024) reduction(+ : ss)
        for (int w = 0; w < n; w++) {
            double acc = 0;
            for (ull e = idx[w]; e < idx[w + 1]; e++) acc += v0[adj[e]];
            v1[w] = acc; ss += acc * acc;
        }
        lam = sqrt(ss);
        for (int w = 0; w < n; w++) v1[w] *= 1.0 / lam;
        double* t = v0; v0 = v1; v1 = t;
        if (pit > 10 && fabs(lam - lamPrev) / lam < 1e-12) break;
        lamPrev = lam;
    }
    double vsum = 0;
    for (int i = 0; i < n; i++) vsum += v0[i];
    const double meanEV = vsum * vsum / n;
    const double alpha = 0.85 / lam, beta = 1.0;
    for (int i = 0; i < n; i++) v0[i] = beta;
    double meanK = 0;
    for (int it = 0; it < 5000; it++) {
        double sum = 0;
        #pragma omp parallel for schedule(dynamic, 1024) reduction(+ : sum)
        for (int w = 0; w < n; w++) {
            double acc = 0;
            for (ull e = idx[w]; e < idx[w + 1]; e++) acc += v0[adj[e]];
            v1[w] = acc * alpha + beta;
            sum += v1[w];
        }
        double* t = v0; v0 = v1; v1 = t;
        double newMean = sum / n;
        if (fabs(newMean - meanK) / newMean < 1e-12) { meanK = newMean; break; }
        meanK = newMean;
    }
    out[0] = lam; out[1] = alpha; out[2] = meanEV; out[3] = meanK; out[4] = pit;
    free(v0); free(v1);
}

/* ------------------------------------------------------- demand snapshot */

/* Bitmap word per 32 vertices (every word written), per-chunk interleaved
 * (pending count, sum of pending degrees), hot pending count, trace counter.
 * Pending iff |r_k| > eps_k for any measure; a pending hot vertex counts in
 * hotpend and is left out of the bitmap and cnt. r is measure-major: r[k*n + v].
 * Restates src/excent.cu:49-98 (chunk_of 49-56, pending 58-64, hot_bit 66-68). */
void or_snapshot(int n, int nm, const float* r, const float* eps, const ull* idx, const int* cv0, int nc,
                 const uint32_t* hot, uint32_t* bitmap, ull* cnt, ull* hotpend, uint16_t* trace) {
    const size_t words = ((size_t)n + 31) / 32;
    memset(bitmap, 0, words * sizeof(uint32_t));
    memset(cnt, 0, 2 * (size_t)nc * sizeof(ull));
    ull hp = 0;
    int c = 0;
    for (int v = 0; v < n; v++) {
        int p = 0;
        for (int k = 0; k < nm; k++) p |= fabsf(r[(size_t)k * n + v]) > eps[k];
        if (trace && p) trace[v]++;
        if (hot && p && ((hot[v >> 5] >> (v & 31)) & 1u)) { hp++; p = 0; }
        if (!p) continue;
        bitmap[v >> 5] |= 1u << (v & 31);
        while (c + 1 < nc && cv0[c + 1] <= v) c++;
        cnt[2 * c] += 1;
        cnt[2 * c + 1] += idx[v + 1] - idx[v];
    }
    *hotpend = hp;
}

/* -------------------------------------------------- CPU delta-push port */

static inline float xchg0(float* a) {
    uint32_t old = __atomic_exchange_n((uint32_t*)a, 0u, __ATOMIC_RELAXED);
    float f; memcpy(&f, &old, 4); return f;
}
static inline void fadd(float* a, float v) {
    uint32_t* p = (uint32_t*)a;
    uint32_t old = __atomic_load_n(p, __ATOMIC_RELAXED), nw;
    do { float f; memcpy(&f, &old, 4); f += v; memcpy(&nw, &f, 4); }
    while (!__atomic_compare_exchange_n(p, &old, nw, 1, __ATOMIC_RELAXED, __ATOMIC_RELAXED));
}

/* Per-measure push of vertex v (src/excent.cu:100-124): for each measure with
 * |r| > eps take d = exchange(r[v], 0), x[v] += d (one writer), weight
 * p = scale*d/(float)deg (divdeg) or scale*d, then add p to r[u] for every
 * neighbour; a degree-0 vertex only absorbs its residual (:116). */
static ull push_one(int v, int nm, int n, float* x, float* r, const float* eps, const float* scale,
                    const int* divdeg, const ull* idx, const int32_t* adj) {
    float p[3] = {0, 0, 0};
    int any = 0;
    const ull deg = idx[v + 1] - idx[v];
    for (int k = 0; k < nm; k++) {
        float* rk = r + (size_t)k * n;
        uint32_t bits = __atomic_load_n((uint32_t*)&rk[v], __ATOMIC_RELAXED);
        float cur; memcpy(&cur, &bits, 4);
        if (fabsf(cur) > eps[k]) {
            float d = xchg0(&rk[v]);
            x[(size_t)k * n + v] += d;
            if (d != 0.f) { any = 1; p[k] = divdeg[k] ? scale[k] * d / (float)deg : scale[k] * d; }
        }
    }
    if (!any || deg == 0) return 0;
    for (ull e = idx[v]; e < idx[v + 1]; e++) {
        const int u = adj[e];
        for (int k = 0; k < nm; k++) if (p[k] != 0.f) fadd(&r[(size_t)k * n + u], p[k]);
    }
    return deg;
}

/* Initial values per measure kind (0 pr, 1 katz, 2 ev): src/excent.cu:41-47.
 * EV's r is computed in double and rounded to float. */
void or_init(int n, int kind, const ull* idx, double beta, double lambda, float* x, float* r) {
    for (int v = 0; v < n; v++) {
        if (kind == 0) { x[v] = 0.f; r[v] = 1.f - 0.85f; }
        else if (kind == 1) { x[v] = 0.f; r[v] = (float)beta; }
        else { x[v] = 1.f; r[v] = (float)((double)(idx[v + 1] - idx[v]) / (float)lambda - 1.0); }
    }
}

/* Whole-run CPU port of the engine for a fully cached graph: per pass a
 * demand snapshot, then each chunk with pending vertices pushed either as its
 * snapshot-pending list (k < list_frac * nv) or as its whole vertex range with
 * the push-time re-check (src/excent.cu:634-652, 656-760). Chunks run in order;
 * within a chunk vertices run in parallel with atomic residual updates.
 * x, r are measure-major [nm][n] and must be initialised by or_init.
 * Stops when nothing is pending or after max_passes passes (or when
 * max_edges pushed edges are reached, 0 = unbounded; used to bound the timed
 * CPU sample). Returns passes; *pushed_out = adjacency entries pushed. */
int or_delta_push(int n, int nm, const ull* idx, const int32_t* adj, const int* cv0, int nc,
                  const float* eps, const float* scale, const int* divdeg, double list_frac,
                  int max_passes, ull max_edges, int threads, float* x, float* r, ull* pushed_out) {
    const size_t words = ((size_t)n + 31) / 32;
    uint32_t* bitmap = (uint32_t*)malloc(words * sizeof(uint32_t));
    ull* cnt = (ull*)malloc(2 * (size_t)nc * sizeof(ull));
    int* list = (int*)malloc(sizeof(int) * (size_t)n);
    ull pushed = 0;
    int pass = 0;
    if (threads <= 0) threads = omp_get_max_threads();
    for (; pass < max_passes; pass++) {
        memset(cnt, 0, 2 * (size_t)nc * sizeof(ull));
        memset(bitmap, 0, words * sizeof(uint32_t));
        ull pend = 0;
        #pragma omp parallel for num_threads(threads) schedule(static) reduction(+ : pend)
        for (long long wd = 0; wd < (long long)words; wd++) {
            uint32_t b = 0;
            for (int l = 0; l < 32; l++) {
                long long v = wd * 32 + l;
                if (v >= n) break;
                int p = 0;
                for (int k = 0; k < nm; k++) p |= fabsf(r[(size_t)k * n + v]) > eps[k];
                if (p) b |= 1u << l;
            }
            bitmap[wd] = b;
            pend += (ull)__builtin_popcount(b);
        }
        if (pend == 0) break;
        for (int c = 0; c < nc; c++) {
            const int v0 = cv0[c], v1 = c + 1 < nc ? cv0[c + 1] : n;
            int k = 0;
            for (int v = v0; v < v1; v++) if ((bitmap[v >> 5] >> (v & 31)) & 1u) list[k++] = v;
            cnt[2 * c] = (ull)k;
            if (k == 0) continue;
            ull pc = 0;
            if ((double)k < list_frac * (v1 - v0)) {
                #pragma omp parallel for num_threads(threads) schedule(dynamic, 64) reduction(+ : pc)
                for (int i = 0; i < k; i++) pc += push_one(list[i], nm, n, x, r, eps, scale, divdeg, idx, adj);
            } else {
                #pragma omp parallel for num_threads(threads) schedule(dynamic, 256) reduction(+ : pc)
                for (int v = v0; v < v1; v++) pc += push_one(v, nm, n, x, r, eps, scale, divdeg, idx, adj);
            }
            pushed += pc;
        }
        if (max_edges && pushed >= max_edges) { pass++; break; }
    }
    free(bitmap); free(cnt); free(list);
    *pushed_out = pushed;
    return pass;
}

/* ------------------------------------------------------------ host logic */

/* Greedy contiguous chunks of <= max_edges edges, at least one vertex each:
 * include/StaticGraph.h:128-139. out holds 4 ull per chunk {v0, v1, e0, e1};
 * returns the chunk count (out may be NULL to count only). */
int or_plan_chunks(int n, const ull* off, ull max_edges, ull* out) {
    int v = 0, nc = 0;
    while (v < n) {
        const ull limit = off[v] + max_edges;
        /* upper_bound over off[v+1 .. n] for limit, minus one */
        int lo = v + 1, hi = n + 1;
        while (lo < hi) { int mid = lo + (hi - lo) / 2; if (off[mid] <= limit) lo = mid + 1; else hi = mid; }
        int v1 = lo - 1;
        if (v1 <= v) v1 = v + 1;
        if (out) { out[4 * nc] = (ull)v; out[4 * nc + 1] = (ull)v1; out[4 * nc + 2] = off[v]; out[4 * nc + 3] = off[v1]; }
        nc++;
        v = v1;
    }
    return nc;
}

/* Chunk edge cap: --chunk-medges if > 0, else clamp(ceil(m / target_chunks),
 * min_chunk_medges * 1e6, 64e6). src/excent.cu:321-326. */
ull or_chunk_cap(ull m, double chunk_medges, double target_chunks, double min_chunk_medges) {
    if (chunk_medges > 0) return (ull)(chunk_medges * 1e6);
    const ull lo = (ull)(min_chunk_medges * 1e6), hi = 64000000ull;
    ull t = (ull)ceil((double)m / target_chunks);
    if (t < lo) t = lo;
    if (t > hi) t = hi;
    return t;
}

/* Per-chunk mode (0 skip, 1 resident, 2 stream, 3 gather), pending total,
 * demand total and whether the bitmap must be read back. src/excent.cu:666-678. */
void or_fetch_plan(int nc, const ull* cnt, const uint8_t* resident, const uint8_t* loaded, double stream_ratio,
                   const ull* chunk_edges, int hot_mode, int pass, const int* hlo, const int* hhi,
                   uint8_t* mode, ull* pend_v, ull* demand, int* need_bitmap) {
    ull pv = 0, dm = 0; int nb = 0;
    for (int c = 0; c < nc; c++) {
        const ull cv = cnt[2 * c], ce = cnt[2 * c + 1];
        pv += cv; dm += ce;
        mode[c] = 0;
        if (cv == 0) continue;
        if (resident[c] && loaded[c]) mode[c] = 1;
        else if (resident[c] || (double)ce >= stream_ratio * (double)chunk_edges[c]) mode[c] = 2;
        else if (hot_mode && pass == 0 && hhi[c] > hlo[c]) mode[c] = 2;
        else { mode[c] = 3; nb = 1; }
    }
    *pend_v = pv; *demand = dm; *need_bitmap = nb;
}

/* Ascending pending vertex ids of [v0, v1) from the bitmap and the prefix sums
 * of their degrees: src/excent.cu:711-723. Returns k; off has k + 1 entries. */
int or_gather_list(int v0, int v1, const uint32_t* bitmap, const ull* idx, int* vids, ull* off) {
    int k = 0;
    for (int v = v0; v < v1; v++) if ((bitmap[v >> 5] >> (v & 31)) & 1u) vids[k++] = v;
    off[0] = 0;
    for (int i = 0; i < k; i++) off[i + 1] = off[i] + (idx[vids[i] + 1] - idx[vids[i]]);
    return k;
}

/* Page runs of the gathered lists, merged per part, parts = clamp(k/1024, 1,
 * io_threads), parts split [k*t/parts, k*(t+1)/parts): include/StaticGraph.h:90-114.
 * nlist_off is the byte offset of nlist in the file. */
void or_prefetch_runs(const int* vids, int k, const ull* idx, ull nlist_off, ull page, int io_threads,
                      ull* pages, ull* runs) {
    ull np = 0, nr = 0;
    int parts = k / 1024;
    if (parts > io_threads) parts = io_threads;
    if (parts < 1) parts = 1;
    for (int t = 0; t < parts; t++) {
        const int i0 = (int)((long long)k * t / parts), i1 = (int)((long long)k * (t + 1) / parts);
        ull r0 = 0, r1 = 0; int open = 0;
        for (int i = i0; i < i1; i++) {
            const ull d = idx[vids[i] + 1] - idx[vids[i]];
            if (!d) continue;
            const ull b0 = nlist_off + idx[vids[i]] * 4, b1 = b0 + d * 4;
            const ull p0 = b0 / page, p1 = (b1 + page - 1) / page;
            if (open && p0 <= r1) { if (p1 > r1) r1 = p1; }
            else { if (open) { np += r1 - r0; nr++; } r0 = p0; r1 = p1; open = 1; }
        }
        if (open) { np += r1 - r0; nr++; }
    }
    *pages = np; *runs = nr;
}

/* Chunk cache: whole chunks in file order while each fits in what is left of
 * free - reserve; returns the resident count. src/excent.cu:410-421. */
int or_cache_chunks(int nc, const ull* chunk_edges, ull free_bytes, ull reserve) {
    ull avail = free_bytes > reserve ? free_bytes - reserve : 0;
    int c = 0;
    for (; c < nc; c++) {
        const ull need = chunk_edges[c] * 4;
        if (need > avail) break;
        avail -= need;
    }
    return c;
}

/* Degree cache selection without --hot-rank: cost(d) = 4d + 16 bytes; the
 * degrees >= 2^20 are taken greedily in descending order, then histogram
 * buckets from 2^20-1 down, each bucket taking as many as the budget allows;
 * the threshold T and quota of degree-T vertices pick the set in vertex order.
 * src/excent.cu:428-457, 475-491. Returns the count, ids ascending (may be NULL),
 * *T_out the threshold. */
static int cmp_desc(const void* a, const void* b) {
    ull x = *(const ull*)a, y = *(const ull*)b;
    return x < y ? 1 : x > y ? -1 : 0;
}
int or_hot_select(int n, const ull* idx, ull budget, int* ids, ull* T_out, ull* edges_out) {
    const ull CAP = 1ull << 20;
    ull* hist = (ull*)calloc(CAP, sizeof(ull));
    ull* big = (ull*)malloc(sizeof(ull) * (size_t)(n > 0 ? n : 1));
    size_t nbig = 0;
    for (int v = 0; v < n; v++) { ull d = idx[v + 1] - idx[v]; if (d >= CAP) big[nbig++] = d; else hist[d]++; }
    qsort(big, nbig, sizeof(ull), cmp_desc);
#define COST(d) ((d) * 4ull + 16ull)
    ull used = 0, T = 0, quota = 0; int done = 0;
    for (size_t i = 0; i < nbig; i++) {
        ull d = big[i];
        if (used + COST(d) > budget) { T = d; quota = 0; done = 1; break; }
        used += COST(d); T = d; quota++;
    }
    if (!done) { quota = 0; T = CAP - 1; }
    for (ull d = CAP - 1; !done && d >= 1; d--) {
        if (!hist[d]) continue;
        ull take = (budget - used) / COST(d);
        if (take > hist[d]) take = hist[d];
        used += take * COST(d);
        T = d; quota = take;
        if (take < hist[d]) done = 1;
    }
    int nh = 0; ull he = 0;
    for (int v = 0; v < n; v++) {
        ull d = idx[v + 1] - idx[v];
        if (d == 0) continue;
        int take = d > T || (d == T && quota > 0);
        if (!take) continue;
        if (d == T) quota--;
        if (ids) ids[nh] = v;
        nh++; he += d;
    }
#undef COST
    free(hist); free(big);
    *T_out = T; *edges_out = he;
    return nh;
}

/* Stream/gather crossover from one stream timing and three gather timings at
 * demand fractions f[0..2]: src/excent.cu:566-572. */
double or_tau(double t_stream, const double* t_g, const double* f) {
    double tau;
    if (t_g[0] >= t_stream) tau = f[0] * t_stream / t_g[0];
    else if (t_g[2] < t_stream) tau = f[2] * t_stream / t_g[2];
    else {
        int j = t_g[1] >= t_stream ? 1 : 2;
        tau = f[j - 1] + (f[j] - f[j - 1]) * (t_stream - t_g[j - 1]) / (t_g[j] - t_g[j - 1]);
    }
    if (tau > 1.0) tau = 1.0;
    if (tau < 0.005) tau = 0.005;
    return tau;
}

/* ------------------------------------------ personalized PR / Katz (FP64) */

/* Column of personalized PageRank for one query: x = (1-d) s + d * sum x_u/L(u)
 * over a symmetric graph, s the seed indicator divided by the seed count;
 * Jacobi until max|dx| / max|x| < tol. Katz with a per-vertex beta vector:
 * x = beta + alpha * sum x_u (kind 1). Returns sweeps. */
int or_ppr(int n, const ull* idx, const int32_t* adj, int kind, double d_or_alpha, const double* teleport,
           double tol, int maxit, double* x_out) {
    double* x = (double*)calloc((size_t)n, sizeof(double));
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    const double c = kind == 0 ? 1.0 - d_or_alpha : 1.0;
    int it = 0; double rel = 1;
    for (int i = 0; i < n; i++) x[i] = c * teleport[i];
    for (; it < maxit && rel > tol; it++) {
        double mx0 = 0, mx1 = 0;
        #pragma omp parallel for schedule(dynamic, 1024) reduction(max : mx0, mx1)
        for (int w = 0; w < n; w++) {
            double acc = 0;
            for (ull e = idx[w]; e < idx[w + 1]; e++) {
                int u = adj[e];
                acc += kind == 0 ? x[u] / (double)(idx[u + 1] - idx[u]) : x[u];
            }
            double nv = c * teleport[w] + d_or_alpha * acc;
            y[w] = nv;
            double dd = fabs(nv - x[w]);
            if (dd > mx0) mx0 = dd;
            if (fabs(nv) > mx1) mx1 = fabs(nv);
        }
        rel = mx1 > 0 ? mx0 / mx1 : 0;
        double* t = x; x = y; y = t;
    }
    memcpy(x_out, x, sizeof(double) * (size_t)n);
    free(x); free(y);
    return it;
}

/* ---------------------------------------------- weighted directed PR (FP64) */

/* Row-normalised weights wn[e] = w[e] / sum of w over the row of e. */
void or_row_normalise(int n, const ull* idx, const float* w, double* wn) {
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int u = 0; u < n; u++) {
        double s = 0;
        for (ull e = idx[u]; e < idx[u + 1]; e++) s += w[e];
        for (ull e = idx[u]; e < idx[u + 1]; e++) wn[e] = w[e] / s;
    }
}

/* Forward weighted PageRank / Katz on a directed CSR (out-lists):
 * x = c * t + s * W^T x, with (W^T x)_v = sum over edges u->v of wn[e] x_u.
 * Push-free FP64 Jacobi by scattering over out-lists. Returns sweeps. */
int or_wfwd(int n, const ull* idx, const int32_t* adj, const double* wn, double c, double s, const double* t,
            double tol, int maxit, double* x_out) {
    double* x = (double*)malloc(sizeof(double) * (size_t)n);
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) x[i] = c * t[i];
    int it = 0; double rel = 1;
    for (; it < maxit && rel > tol; it++) {
        for (int i = 0; i < n; i++) y[i] = c * t[i];
        for (int u = 0; u < n; u++) {
            const double xu = x[u];
            if (xu == 0) continue;
            for (ull e = idx[u]; e < idx[u + 1]; e++) y[adj[e]] += s * wn[e] * xu;
        }
        double mx0 = 0, mx1 = 0;
        for (int i = 0; i < n; i++) {
            double d = fabs(y[i] - x[i]); if (d > mx0) mx0 = d;
            if (fabs(y[i]) > mx1) mx1 = fabs(y[i]);
        }
        rel = mx1 > 0 ? mx0 / mx1 : 0;
        double* tt = x; x = y; y = tt;
    }
    memcpy(x_out, x, sizeof(double) * (size_t)n);
    free(x); free(y);
    return it;
}

/* Adjoint of or_wfwd: lam = g + s * W lam, (W lam)_u = sum over edges u->v of
 * wn[e] lam_v (a pull over out-lists). Returns sweeps. */
int or_wadj(int n, const ull* idx, const int32_t* adj, const double* wn, double s, const double* g,
            double tol, int maxit, double* lam_out) {
    double* x = (double*)malloc(sizeof(double) * (size_t)n);
    double* y = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) x[i] = g[i];
    int it = 0; double rel = 1;
    for (; it < maxit && rel > tol; it++) {
        double mx0 = 0, mx1 = 0;
        #pragma omp parallel for schedule(dynamic, 1024) reduction(max : mx0, mx1)
        for (int u = 0; u < n; u++) {
            double acc = 0;
            for (ull e = idx[u]; e < idx[u + 1]; e++) acc += wn[e] * x[adj[e]];
            double nv = g[u] + s * acc;
            y[u] = nv;
            double d = fabs(nv - x[u]); if (d > mx0) mx0 = d;
            if (fabs(nv) > mx1) mx1 = fabs(nv);
        }
        rel = mx1 > 0 ? mx0 / mx1 : 0;
        double* tt = x; x = y; y = tt;
    }
    memcpy(lam_out, x, sizeof(double) * (size_t)n);
    free(x); free(y);
    return it;
}

/* Gradient w.r.t. the raw weights w of L = g . x through the row
 * normalisation wn = w / rowsum(w): with G_e = s * x_u * lam_v,
 * dL/dw_e = (G_e - sum_{e' in row u} wn_e' G_e') / rowsum_u. */
void or_wgrad(int n, const ull* idx, const int32_t* adj, const float* w, const double* wn, double s,
              const double* x, const double* lam, double* gw) {
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int u = 0; u < n; u++) {
        double rs = 0, dot = 0;
        for (ull e = idx[u]; e < idx[u + 1]; e++) { rs += w[e]; dot += wn[e] * s * x[u] * lam[adj[e]]; }
        for (ull e = idx[u]; e < idx[u + 1]; e++) gw[e] = (s * x[u] * lam[adj[e]] - dot) / rs;
    }
}

/* ------------------------------------------- CSR construction (OpenMP) */

static int cmp_i32(const void* a, const void* b) {
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* CSR of npairs (src, dst) pairs over n vertices: both directions when
 * symmetric, self-loops and duplicates dropped, each list sorted. idx has
 * n + 1 entries; adj must hold 2 * npairs (symmetric) or npairs entries.
 * Returns m. Same result as csr_from_pairs() in oracle/__init__.py. */
ull or_csr_build(int n, ull npairs, const int32_t* src, const int32_t* dst, int symmetric, ull* idx, int32_t* adj) {
    ull* deg = (ull*)calloc((size_t)n + 1, sizeof(ull));
    #pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)npairs; i++) {
        if (src[i] == dst[i]) continue;
        __atomic_fetch_add(&deg[src[i]], 1ull, __ATOMIC_RELAXED);
        if (symmetric) __atomic_fetch_add(&deg[dst[i]], 1ull, __ATOMIC_RELAXED);
    }
    ull* pos = (ull*)malloc(((size_t)n + 1) * sizeof(ull));
    pos[0] = 0;
    for (int v = 0; v < n; v++) pos[v + 1] = pos[v] + deg[v];
    ull* fill = (ull*)malloc(((size_t)n + 1) * sizeof(ull));
    memcpy(fill, pos, ((size_t)n + 1) * sizeof(ull));
    #pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)npairs; i++) {
        const int s = src[i], d = dst[i];
        if (s == d) continue;
        adj[__atomic_fetch_add(&fill[s], 1ull, __ATOMIC_RELAXED)] = d;
        if (symmetric) adj[__atomic_fetch_add(&fill[d], 1ull, __ATOMIC_RELAXED)] = s;
    }
    /* sort and dedup each list in place; deg[v] becomes the unique count */
    #pragma omp parallel for schedule(dynamic, 256)
    for (int v = 0; v < n; v++) {
        int32_t* l = adj + pos[v];
        const ull k = pos[v + 1] - pos[v];
        if (k > 1) qsort(l, k, sizeof(int32_t), cmp_i32);
        ull u = 0;
        for (ull j = 0; j < k; j++) if (j == 0 || l[j] != l[j - 1]) l[u++] = l[j];
        deg[v] = u;
    }
    idx[0] = 0;
    for (int v = 0; v < n; v++) idx[v + 1] = idx[v] + deg[v];
    /* compact lists towards the front (sequential: ranges move left only) */
    for (int v = 0; v < n; v++)
        if (idx[v] != pos[v] && deg[v]) memmove(adj + idx[v], adj + pos[v], deg[v] * sizeof(int32_t));
    const ull m = idx[n];
    free(deg); free(pos); free(fill);
    return m;
}

/* lambda1 of a symmetric graph by FP64 power iteration from the unit
 * all-ones vector, stopping when the relative change is below tol. */
double or_lambda1(int n, const ull* idx, const int32_t* adj, double tol, int maxit) {
    double* v0 = (double*)malloc(sizeof(double) * (size_t)n);
    double* v1 = (double*)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) v0[i] = 1.0 / sqrt((double)n);
    double lam = 0, prev = 0;
    for (int it = 0; it < maxit; it++) {
        double ss = 0;
        #pragma omp parallel for schedule(dynamic, 4096) reduction(+ : ss)
        for (int w = 0; w < n; w++) {
            double acc = 0;
            for (ull e = idx[w]; e < idx[w + 1]; e++) acc += v0[adj[e]];
            v1[w] = acc; ss += acc * acc;
        }
        lam = sqrt(ss);
        #pragma omp parallel for schedule(static)
        for (int w = 0; w < n; w++) v1[w] /= lam;
        double* t = v0; v0 = v1; v1 = t;
        if (it > 10 && fabs(lam - prev) / lam < tol) break;
        prev = lam;
    }
    free(v0); free(v1);
    return lam;
}
