// params_tool.cpp -- bin/excent_params: the "given constants" of a symmetric
// graph (lambda1 and the Katz / eigenvector fixed-point means, the thresholds
// derived from them) computed in FP64 on the device, written as the .env file
// the CLI and run.sh read. Same arguments, stdout lines and .env keys as the
// reference's tools/excent_params.cu:73-172; the computation is
// excent_params_fp64 (fp64.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.h"
#include "egr.h"

namespace excent {
namespace {

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Sampled symmetry check (tools/excent_params.cu:106-118): for random entries
// e = (v -> u), u's sorted list must hold v. Returns the number of misses.
int symmetry_misses(const GraphFile& g, int samples) {
    uint64_t s = 42;
    const ull* off = g.offsets();
    int bad = 0;
    for (int i = 0; i < samples; i++) {
        const ull e = splitmix(s) % g.m;
        const int v = (int)(std::upper_bound(off, off + (size_t)g.n + 1, e) - off) - 1;
        const int u = g.list(0)[e];
        const int32_t* b = g.list(u);
        const int32_t* en = b + g.degree(u);
        const bool sorted = std::is_sorted(b, en);
        const bool found = sorted ? std::binary_search(b, en, v) : std::find(b, en, v) != en;
        if (!found) bad++;
    }
    return bad;
}

}  // namespace
}  // namespace excent

using namespace excent;

extern "C" int excent_params_main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s graph.egr out.env\n", argv[0]);
        return 1;
    }
    int device = 0;
    for (int i = 3; i + 1 < argc; i += 2) {
        if (!strcmp(argv[i], "--device")) device = atoi(argv[i + 1]);
        else { fprintf(stderr, "unknown option %s\n", argv[i]); return 1; }
    }
    const auto t0 = std::chrono::steady_clock::now();
    GraphFile g;
    if (g.open(argv[1], 16, true, true) != EXCENT_OK) { fprintf(stderr, "%s: %s\n", argv[1], excent_last_error()); return 1; }
    const int n = g.n;
    const ull m = g.m;
    printf("graph: n=%d m=%llu  load %.1fs\n", n, m,
           std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    if (m > 0) {
        const int S = 200000;
        const int bad = symmetry_misses(g, S);
        if (bad) {
            fprintf(stderr, "graph is not symmetric (%d/%d sampled edges lack a reverse edge)\n", bad, S);
            return 1;
        }
    }
    ull* d_idx = nullptr;
    int32_t* d_adj = nullptr;
    int32_t* stage = nullptr;
    int rc = 0;
    double out[5] = {0, 0, 0, 0, 0};
    do {
        if (cudaSetDevice(device) != cudaSuccess ||
            cudaMalloc((void**)&d_idx, ((size_t)n + 1) * sizeof(ull)) != cudaSuccess ||
            cudaMalloc((void**)&d_adj, std::max<ull>(m, 1) * sizeof(int32_t)) != cudaSuccess ||
            cudaMallocHost((void**)&stage, (size_t)1 << 28) != cudaSuccess) {
            fprintf(stderr, "excent_params: the graph does not fit on device %d\n", device);
            rc = 1;
            break;
        }
        if (cudaMemcpy(d_idx, g.offsets(), ((size_t)n + 1) * sizeof(ull), cudaMemcpyHostToDevice) != cudaSuccess) { rc = 1; break; }
        const ull piece = ((size_t)1 << 28) / sizeof(int32_t);
        for (ull e0 = 0; e0 < m && !rc; e0 += piece) {
            const ull e1 = std::min(m, e0 + piece);
            if (g.fetch_entries(e0, e1, stage) != EXCENT_OK ||
                cudaMemcpy(d_adj + e0, stage, (e1 - e0) * sizeof(int32_t), cudaMemcpyHostToDevice) != cudaSuccess)
                rc = 1;
        }
        if (rc) { fprintf(stderr, "excent_params: reading %s failed\n", argv[1]); break; }
        if (excent_params_fp64(device, n, d_idx, d_adj, 0.85, out, nullptr) != EXCENT_OK) {
            fprintf(stderr, "excent_params: %s\n", excent_last_error());
            rc = 1;
        }
    } while (0);
    if (stage) cudaFreeHost(stage);
    if (d_idx) cudaFree(d_idx);
    if (d_adj) cudaFree(d_adj);
    if (rc) return rc;
    const double lam = out[0], alpha = out[1], mean_ev = out[2], mean_katz = out[3];
    const int sweeps = (int)out[4];
    printf("lambda1 = %.10f after %d power iterations; eigenvector fixed-point mean = %.6g\n", lam, sweeps, mean_ev);
    printf("Katz: alpha = 0.85/lambda1 = %.6g, beta = 1, fixed-point mean = %.6g\n", alpha, mean_katz);
    FILE* o = fopen(argv[2], "w");
    if (!o) { perror(argv[2]); return 1; }
    fprintf(o, "# Given constants of %s, computed in FP64 on the GPU (lambda1 after %d power iterations).\n",
            argv[1], sweeps);
    fprintf(o, "# Katz alpha = 0.85 / lambda1, beta = 1; eps = 0.01 x each measure's fixed-point mean.\n");
    fprintf(o, "LAMBDA=%.10f\nALPHA=%.6g\nBETA=1\nEPS_PR=0.01\nEPS_KATZ=%.6g\nEPS_EV=%.6g\n", lam, alpha,
            0.01 * mean_katz, 0.01 * mean_ev);
    fclose(o);
    printf("wrote %s\n", argv[2]);
    return 0;
}
