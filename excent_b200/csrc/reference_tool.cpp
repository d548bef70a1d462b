// reference_tool.cpp -- bin/excent_reference: the FP64 oracle of a graph as a
// GPU tool, and the comparison of a float32 dump against it. Same modes and
// file formats as the reference's tools/centrality_reference.cu:
//   excent_reference graph.egr pr|katz|ev ref.bin [--alpha A] [--beta B]
//       FP64 Jacobi (PR, Katz) or power iteration (EV) to a relative change of
//       1e-9 (at most 20000 sweeps) on the GPU (excent_reference_fp64); ref.bin
//       gets n doubles.
//   excent_reference --compare pr|katz|ev ref.bin dump.bin
//       L1 error relative to |ref|_1, L2 error and top-100 overlap of a float32
//       dump (EV: both as unit vectors, sign fixed by their sums).
//   excent_reference --rank pr|katz|ev ref.bin dump.bin
//       P@k of the dump's top k against the reference's (k = 10 .. 100000) and
//       Kendall tau over the reference's top 1000.
//   excent_reference --compare-dumps pr|katz|ev a.bin b.bin   (two float32 dumps)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "common.h"
#include "egr.h"

namespace excent {
namespace {

bool load_file(const char* path, std::vector<char>& out) {
    FILE* f = fopen(path, "rb");
    if (!f) { perror(path); return false; }
    fseek(f, 0, SEEK_END);
    const long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    out.resize((size_t)std::max(sz, 0L));
    const bool ok = fread(out.data(), 1, out.size(), f) == out.size();
    fclose(f);
    if (!ok) perror(path);
    return ok;
}

// Unit L2 norm with the sign that makes the sum positive.
void to_unit(std::vector<double>& v) {
    double ss = 0, sum = 0;
    for (double a : v) { ss += a * a; sum += a; }
    if (ss <= 0) return;
    const double f = (sum < 0 ? -1.0 : 1.0) / std::sqrt(ss);
    for (double& a : v) a *= f;
}

bool load_pair(const char* refp, const char* dumpp, bool ref_is_float, std::vector<double>& r, std::vector<double>& x) {
    std::vector<char> rb, xb;
    if (!load_file(refp, rb) || !load_file(dumpp, xb)) return false;
    const size_t n = rb.size() / (ref_is_float ? sizeof(float) : sizeof(double));
    if (xb.size() != n * sizeof(float)) {
        fprintf(stderr, "size mismatch: ref n=%zu, dump %zu floats\n", n, xb.size() / 4);
        return false;
    }
    r.resize(n);
    x.resize(n);
    for (size_t i = 0; i < n; i++) {
        if (ref_is_float) { float t; memcpy(&t, rb.data() + 4 * i, 4); r[i] = t; }
        else memcpy(&r[i], rb.data() + 8 * i, 8);
        float t;
        memcpy(&t, xb.data() + 4 * i, 4);
        x[i] = t;
    }
    return true;
}

// Indices of the k largest values (ties: lower index first), as a sorted set.
std::vector<int> top_set(const std::vector<double>& v, size_t k) {
    std::vector<int> id(v.size());
    std::iota(id.begin(), id.end(), 0);
    k = std::min(k, v.size());
    std::partial_sort(id.begin(), id.begin() + k, id.end(),
                      [&](int a, int b) { return v[a] > v[b] || (v[a] == v[b] && a < b); });
    id.resize(k);
    return id;
}

size_t overlap(std::vector<int> a, std::vector<int> b) {
    std::sort(a.begin(), a.end());
    std::sort(b.begin(), b.end());
    std::vector<int> c;
    std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(c));
    return c.size();
}

int compare_mode(const std::string& measure, const char* refp, const char* dumpp, bool ref_is_float) {
    std::vector<double> r, x;
    if (!load_pair(refp, dumpp, ref_is_float, r, x)) return 1;
    if (measure == "ev") { to_unit(r); to_unit(x); }
    double l1 = 0, r1 = 0, l2 = 0;
    for (size_t i = 0; i < r.size(); i++) {
        const double d = std::fabs(x[i] - r[i]);
        l1 += d;
        r1 += std::fabs(r[i]);
        l2 += d * d;
    }
    const int K = 100;
    const size_t common = overlap(top_set(r, K), top_set(x, K));
    printf("%s: n=%zu  L1 rel err %.3e  L2 err %.3e%s  top-%d overlap %zu/%d\n", measure.c_str(), r.size(), l1 / r1,
           std::sqrt(l2), measure == "ev" ? " (unit vectors)" : "", K, common, K);
    return 0;
}

int rank_mode(const std::string& measure, const char* refp, const char* dumpp) {
    std::vector<double> r, x;
    if (!load_pair(refp, dumpp, false, r, x)) return 1;
    if (measure == "ev") { to_unit(r); to_unit(x); }
    const size_t kmax = std::min<size_t>(100000, r.size());
    const std::vector<int> tr = top_set(r, kmax), tx = top_set(x, kmax);
    printf("%s:", measure.c_str());
    for (size_t k : {10, 100, 1000, 10000, 100000}) {
        if (k > kmax) break;
        const size_t c = overlap(std::vector<int>(tr.begin(), tr.begin() + k), std::vector<int>(tx.begin(), tx.begin() + k));
        printf("  P@%zu %.4f", k, (double)c / (double)k);
    }
    // Kendall tau over the reference's top T: concordant minus discordant pairs
    const int T = (int)std::min<size_t>(1000, r.size());
    long long conc = 0, disc = 0;
    for (int i = 0; i < T; i++)
        for (int j = i + 1; j < T; j++) {
            const double dr = r[tr[i]] - r[tr[j]], dx = x[tr[i]] - x[tr[j]];
            if (dr * dx > 0) conc++;
            else if (dr * dx < 0) disc++;
        }
    printf("  tau@1000 %.4f\n", (double)(conc - disc) / ((double)T * (T - 1) / 2));
    return 0;
}

int solve_mode(int argc, char** argv) {
    const std::string measure = argv[2];
    double alpha = -1, beta = 1;
    for (int i = 4; i + 1 < argc; i += 2) {
        if (!strcmp(argv[i], "--alpha")) alpha = atof(argv[i + 1]);
        else if (!strcmp(argv[i], "--beta")) beta = atof(argv[i + 1]);
    }
    const int kind = measure == "pr" ? 0 : measure == "katz" ? 1 : measure == "ev" ? 2 : -1;
    if (kind < 0) { fprintf(stderr, "measure must be pr, katz or ev\n"); return 1; }
    if (kind == 1 && alpha <= 0) { fprintf(stderr, "katz needs --alpha\n"); return 1; }
    GraphFile g;
    if (g.open(argv[1], 16, true, true) != EXCENT_OK) { fprintf(stderr, "%s: %s\n", argv[1], excent_last_error()); return 1; }
    const int n = g.n;
    const ull m = g.m;
    ull* d_idx = nullptr;
    int32_t* d_adj = nullptr;
    std::vector<int32_t> stage;
    std::vector<double> x((size_t)n);
    int it = 0, rc = 0;
    do {
        if (cudaMalloc((void**)&d_idx, ((size_t)n + 1) * sizeof(ull)) != cudaSuccess ||
            cudaMalloc((void**)&d_adj, std::max<ull>(m, 1) * sizeof(int32_t)) != cudaSuccess) {
            fprintf(stderr, "excent_reference: the graph does not fit on the GPU\n");
            rc = 1;
            break;
        }
        cudaMemcpy(d_idx, g.offsets(), ((size_t)n + 1) * sizeof(ull), cudaMemcpyHostToDevice);
        const ull piece = (ull)1 << 26;
        stage.resize((size_t)std::min<ull>(piece, std::max<ull>(m, 1)));
        for (ull e0 = 0; e0 < m && !rc; e0 += piece) {
            const ull e1 = std::min(m, e0 + piece);
            if (g.fetch_entries(e0, e1, stage.data()) != EXCENT_OK ||
                cudaMemcpy(d_adj + e0, stage.data(), (e1 - e0) * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
                rc = 1;
        }
        if (rc) { fprintf(stderr, "excent_reference: reading %s failed\n", argv[1]); break; }
        if (excent_reference_fp64(0, n, d_idx, d_adj, kind, alpha, beta, 1e-9, 20000, x.data(), &it) != EXCENT_OK) {
            fprintf(stderr, "excent_reference: %s\n", excent_last_error());
            rc = 1;
        }
    } while (0);
    if (d_idx) cudaFree(d_idx);
    if (d_adj) cudaFree(d_adj);
    if (rc) return rc;
    double sum = 0;
    for (double v : x) sum += v;
    printf("reference %s: %d iterations, sum %.6e%s\n", measure.c_str(), it, sum, kind == 2 ? " (unit L2)" : "");
    FILE* o = fopen(argv[3], "wb");
    if (!o || fwrite(x.data(), sizeof(double), x.size(), o) != x.size()) { perror(argv[3]); if (o) fclose(o); return 1; }
    fclose(o);
    return 0;
}

}  // namespace
}  // namespace excent

using namespace excent;

extern "C" int excent_reference_main(int argc, char** argv) {
    if (argc >= 5 && !strcmp(argv[1], "--compare")) return compare_mode(argv[2], argv[3], argv[4], false);
    if (argc >= 5 && !strcmp(argv[1], "--rank")) return rank_mode(argv[2], argv[3], argv[4]);
    if (argc >= 5 && !strcmp(argv[1], "--compare-dumps")) return compare_mode(argv[2], argv[3], argv[4], true);
    if (argc < 4) {
        fprintf(stderr, "usage: %s graph.egr pr|katz|ev ref.bin [--alpha A] [--beta B]\n"
                        "       %s --compare pr|katz|ev ref.bin dump.bin\n", argv[0], argv[0]);
        return 1;
    }
    return solve_mode(argc, argv);
}
