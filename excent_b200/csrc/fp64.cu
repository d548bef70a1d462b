// fp64.cu -- the FP64 steps that run on the device: the eigenvector lambda1 /
// normalisation power iteration and the Katz fixed-point mean that give a
// graph's "given constants" (the reference computes them in
// tools/excent_params.cu:133-172), and an FP64 Jacobi / power-iteration
// solve of PageRank, Katz and eigenvector centrality for verification of
// large graphs (tools/centrality_reference.cu:31-59, 184-214).
//
// Graphs are device-resident CSR (offsets u64[n+1], lists i32[m]) and
// symmetric, so a pull over out-lists equals the in-neighbour sum.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "common.h"
#include "device.cuh"

namespace excent {

// y[v] = c + s * sum_{u in N(v)} x[u] (/ L(u) if divdeg), c[v] from cv if given;
// one warp per vertex.
// If mx is given: mx[0] = max |y - x|, mx[1] = max |y| (as ordered bit patterns).
__global__ void k_pull64(int n, const ull* idx, const int* adj, const double* x, double* y, double c, double s,
                         int divdeg, ull* mx, const double* cv = nullptr) {
    const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    double acc = 0;
    for (ull e = idx[w] + lane; e < idx[w + 1]; e += 32) {
        const int u = adj[e];
        acc += divdeg ? x[u] / (double)(idx[u + 1] - idx[u]) : x[u];
    }
    acc = warp_sum(acc);
    if (lane == 0) {
        const double nv = (cv ? cv[w] : c) + s * acc;
        y[w] = nv;
        if (mx) {
            atomicMax(&mx[0], (ull)__double_as_longlong(fabs(nv - x[w])));
            atomicMax(&mx[1], (ull)__double_as_longlong(fabs(nv)));
        }
    }
}

// out[0] += sum x^2, out[1] += sum x, out[2] = max |x - y| (bit pattern) if y
__global__ void k_norms64(int n, const double* x, const double* y, double* out, ull* mx) {
    double a = 0, b = 0, d = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        a += x[v] * x[v];
        b += x[v];
        if (y) d = fmax(d, fabs(x[v] - y[v]));
    }
    a = warp_sum(a);
    b = warp_sum(b);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_down_sync(FULL, d, o));
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out[0], a);
        atomicAdd(&out[1], b);
        if (y) atomicMax(mx, (ull)__double_as_longlong(d));
    }
}

__global__ void k_scale64(int n, double* x, double f, double add) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        x[v] = x[v] * f + add;
}

}  // namespace excent

using namespace excent;

namespace {
struct Bufs {
    double* v[2] = {nullptr, nullptr};
    double* red = nullptr;
    ull* mx = nullptr;
    ~Bufs() {
        for (double* p : v) if (p) cudaFree(p);
        if (red) cudaFree(red);
        if (mx) cudaFree(mx);
    }
};

int norms(int n, const double* x, const double* y, Bufs& B, int grid, double* ss, double* sum, double* maxdiff) {
    EX_CUDA(cudaMemset(B.red, 0, 2 * sizeof(double)));
    EX_CUDA(cudaMemset(B.mx, 0, sizeof(ull)));
    k_norms64<<<grid, 256>>>(n, x, y, B.red, B.mx);
    double h[2];
    ull m = 0;
    EX_CUDA(cudaMemcpy(h, B.red, sizeof h, cudaMemcpyDeviceToHost));
    EX_CUDA(cudaMemcpy(&m, B.mx, sizeof m, cudaMemcpyDeviceToHost));
    if (ss) *ss = h[0];
    if (sum) *sum = h[1];
    if (maxdiff) { double d; memcpy(&d, &m, 8); *maxdiff = d; }
    return EXCENT_OK;
}
}  // namespace

__global__ void k_tofloat(int n, const double* x, float* y) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        y[v] = (float)x[v];
}

extern "C" int excent_params_fp64(int device, int n, const unsigned long long* d_idx, const int32_t* d_adj,
                                  double katz_numerator, double* out, float* d_v1) {
    EX_CHECK_ARG(n >= 1 && d_idx && d_adj && out, "bad argument");
    EX_CUDA(cudaSetDevice(device));
    int sms = 0;
    EX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int G = sms * 8;
    const unsigned wb = (unsigned)(((long long)n * 32 + 255) / 256);
    Bufs B;
    for (auto& p : B.v) if (cudaMalloc(&p, (size_t)n * sizeof(double)) != cudaSuccess) { cudaGetLastError(); EX_FAIL(EXCENT_ERR_NOMEM, "params: vectors do not fit"); }
    EX_CUDA(cudaMalloc(&B.red, 2 * sizeof(double)));
    EX_CUDA(cudaMalloc(&B.mx, sizeof(ull)));
    // lambda1: unit all-ones start, y = A x, lam = ||y||, x = y / lam; stop when
    // |lam - lamPrev| / lam < 1e-12 after 10 sweeps (tools/excent_params.cu:133-147)
    k_scale64<<<G, 256>>>(n, B.v[0], 0.0, 1.0 / std::sqrt((double)n));
    double lam = 0, lamPrev = 0, ss = 0, vsum = 0;
    int pit = 0;
    for (; pit < 5000; pit++) {
        k_pull64<<<wb, 256>>>(n, d_idx, d_adj, B.v[0], B.v[1], 0.0, 1.0, 0, nullptr);
        EX_TRY(norms(n, B.v[1], nullptr, B, G, &ss, nullptr, nullptr));
        if (!(ss > 0)) EX_FAIL(EXCENT_ERR_ARG, "params: the graph has no edges (A x = 0), lambda1 is undefined");
        lam = std::sqrt(ss);
        k_scale64<<<G, 256>>>(n, B.v[1], 1.0 / lam, 0.0);
        std::swap(B.v[0], B.v[1]);
        if (pit > 10 && std::fabs(lam - lamPrev) / lam < 1e-12) break;
        lamPrev = lam;
    }
    EX_TRY(norms(n, B.v[0], nullptr, B, G, nullptr, &vsum, nullptr));
    const double meanEV = vsum * vsum / n;
    if (d_v1) k_tofloat<<<G, 256>>>(n, B.v[0], d_v1);  // unit principal eigenvector
    // Katz fixed point x = 1 + alpha A x, alpha = katz_numerator / lambda1, for its mean (:150-162)
    const double alpha = katz_numerator / lam;
    k_scale64<<<G, 256>>>(n, B.v[0], 0.0, 1.0);
    double meanK = 0;
    for (int it = 0; it < 5000; it++) {
        k_pull64<<<wb, 256>>>(n, d_idx, d_adj, B.v[0], B.v[1], 1.0, alpha, 0, nullptr);
        std::swap(B.v[0], B.v[1]);
        double sum = 0;
        EX_TRY(norms(n, B.v[0], nullptr, B, G, nullptr, &sum, nullptr));
        const double nm = sum / n;
        if (std::fabs(nm - meanK) / nm < 1e-12) { meanK = nm; break; }
        meanK = nm;
    }
    EX_CUDA(cudaDeviceSynchronize());
    out[0] = lam; out[1] = alpha; out[2] = meanEV; out[3] = meanK; out[4] = pit;
    return EXCENT_OK;
}

extern "C" int excent_reference_fp64(int device, int n, const unsigned long long* d_idx, const int32_t* d_adj,
                                     int kind, double alpha, double beta, double tol, int maxit, double* x_out,
                                     int* iterations) {
    EX_CHECK_ARG(n >= 1 && d_idx && d_adj && x_out && kind >= 0 && kind <= 2, "bad argument");
    EX_CUDA(cudaSetDevice(device));
    int sms = 0;
    EX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int G = sms * 8;
    const unsigned wb = (unsigned)(((long long)n * 32 + 255) / 256);
    Bufs B;
    for (auto& p : B.v) if (cudaMalloc(&p, (size_t)n * sizeof(double)) != cudaSuccess) { cudaGetLastError(); EX_FAIL(EXCENT_ERR_NOMEM, "reference: vectors do not fit"); }
    EX_CUDA(cudaMalloc(&B.red, 2 * sizeof(double)));
    EX_CUDA(cudaMalloc(&B.mx, 2 * sizeof(ull)));
    double c = 0, s = 1;
    int divdeg = 0;
    if (kind == 0) { c = 0.15; s = 0.85; divdeg = 1; }
    else if (kind == 1) { c = beta; s = alpha; }
    k_scale64<<<G, 256>>>(n, B.v[0], 0.0, kind == 0 ? 0.15 : 1.0);
    int it = 0;
    double rel = 1;
    for (; it < maxit && rel > tol; it++) {
        if (kind == 2) {
            k_pull64<<<wb, 256>>>(n, d_idx, d_adj, B.v[0], B.v[1], 0.0, 1.0, 0, nullptr);
            double ss = 0;
            EX_TRY(norms(n, B.v[1], nullptr, B, G, &ss, nullptr, nullptr));
            k_scale64<<<G, 256>>>(n, B.v[1], 1.0 / std::sqrt(ss), 0.0);
            double md = 0;
            EX_TRY(norms(n, B.v[1], B.v[0], B, G, nullptr, nullptr, &md));
            rel = it == 0 ? 1.0 : md;
        } else {
            EX_CUDA(cudaMemset(B.mx, 0, 2 * sizeof(ull)));
            k_pull64<<<wb, 256>>>(n, d_idx, d_adj, B.v[0], B.v[1], c, s, divdeg, B.mx);
            ull h[2];
            EX_CUDA(cudaMemcpy(h, B.mx, sizeof h, cudaMemcpyDeviceToHost));
            double d, m;
            memcpy(&d, &h[0], 8);
            memcpy(&m, &h[1], 8);
            rel = d / m;
        }
        std::swap(B.v[0], B.v[1]);
    }
    EX_CUDA(cudaMemcpy(x_out, B.v[0], (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    if (kind == 2) {  // unit L2 norm, sign fixed by the sum (tools/centrality_reference.cu:71-76)
        double s2 = 0, t = 0;
        for (int i = 0; i < n; i++) { s2 += x_out[i] * x_out[i]; t += x_out[i]; }
        const double f = (t < 0 ? -1.0 : 1.0) / std::sqrt(s2);
        for (int i = 0; i < n; i++) x_out[i] *= f;
    }
    if (iterations) *iterations = it;
    return EXCENT_OK;
}

__global__ void k_scatter64(int k, const int* vids, const float* vals, double* t) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) t[vids[i]] += (double)vals[i];
}

extern "C" int excent_ppr_fp64(int device, int n, const unsigned long long* d_idx, const int32_t* d_adj, double d,
                               int k, const int32_t* vids, const float* vals, double tol, int maxit, double* x_out,
                               int* iterations) {
    EX_CHECK_ARG(n >= 1 && d_idx && d_adj && x_out && k >= 0 && (k == 0 || (vids && vals)), "bad argument");
    for (int i = 0; i < k; i++) EX_CHECK_ARG(vids[i] >= 0 && vids[i] < n, "seed vertex %d out of range", vids[i]);
    EX_CUDA(cudaSetDevice(device));
    int sms = 0;
    EX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int G = sms * 8;
    const unsigned wb = (unsigned)(((long long)n * 32 + 255) / 256);
    Bufs B;
    double* t = nullptr;
    int* dv = nullptr;
    float* dval = nullptr;
    for (auto& p : B.v) if (cudaMalloc(&p, (size_t)n * sizeof(double)) != cudaSuccess) { cudaGetLastError(); EX_FAIL(EXCENT_ERR_NOMEM, "ppr reference: vectors do not fit"); }
    EX_CUDA(cudaMalloc(&B.red, 2 * sizeof(double)));
    EX_CUDA(cudaMalloc(&B.mx, 2 * sizeof(ull)));
    int rc = EXCENT_OK;
    int it = 0;
    do {
        if (cudaMalloc(&t, (size_t)n * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&dv, std::max(k, 1) * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&dval, std::max(k, 1) * sizeof(float)) != cudaSuccess) {
            cudaGetLastError(); set_error("ppr reference: teleport vector does not fit"); rc = EXCENT_ERR_NOMEM; break;
        }
        cudaMemset(t, 0, (size_t)n * sizeof(double));
        if (k) {
            cudaMemcpy(dv, vids, (size_t)k * sizeof(int), cudaMemcpyHostToDevice);
            cudaMemcpy(dval, vals, (size_t)k * sizeof(float), cudaMemcpyHostToDevice);
            k_scatter64<<<std::min(1024, (k + 255) / 256), 256>>>(k, dv, dval, t);
        }
        cudaMemcpy(B.v[0], t, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice);
        double rel = 1;
        for (; it < maxit && rel > tol; it++) {
            cudaMemset(B.mx, 0, 2 * sizeof(ull));
            k_pull64<<<wb, 256>>>(n, d_idx, d_adj, B.v[0], B.v[1], 0.0, d, 1, B.mx, t);
            ull h[2];
            if (cudaMemcpy(h, B.mx, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) break;
            double dd, mm;
            memcpy(&dd, &h[0], 8);
            memcpy(&mm, &h[1], 8);
            rel = mm > 0 ? dd / mm : 0.0;
            std::swap(B.v[0], B.v[1]);
        }
        const cudaError_t err = cudaMemcpy(x_out, B.v[0], (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) { set_error("ppr reference: %s", cudaGetErrorString(err)); rc = EXCENT_ERR_CUDA; }
    } while (0);
    if (t) cudaFree(t);
    if (dv) cudaFree(dv);
    if (dval) cudaFree(dval);
    if (iterations) *iterations = it;
    return rc;
}
