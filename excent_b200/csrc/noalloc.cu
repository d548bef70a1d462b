// noalloc.cu -- excent_params_fp64_noalloc: the given-constants computation
// (FP64 lambda1 power iteration, eigenvector mean, Katz mean) of
// excent_params_fp64 without any device allocation.
//
// Who needs it: hosts that own all device memory themselves and do not let a
// library call cudaMalloc -- an inference server or framework that reserves
// the GPU's memory up front in its own pool (so a cudaMalloc would fail or
// fragment it), or a latency-sensitive pipeline where the device-wide
// synchronisation that cudaMalloc/cudaFree can cause would stall other
// streams. Those callers pass their own inputs and outputs and get the same
// results as excent_params_fp64.
//
// The two FP64 iteration vectors and the reduction slots live in one
// file-scope device array, g_noalloc_scratch, sized for graphs of at most
// EXCENT_NOALLOC_MAX_N vertices (2 * 2^20 doubles + 64 = 16 MiB + 512 bytes).
// Every GPU that loads the library holds this array until the process exits.
// All calls share it and it keeps the last call's contents, so calls that
// overlap on the GPU (two host threads, or two streams) race on it and must
// be serialised by the caller.
//
// Host code cannot use the array's name as a device address. Every call looks
// the address up with cudaGetSymbolAddress on the device it runs on, with that
// device current (cheap, and it allocates nothing), so a cudaDeviceReset in
// between cannot leave a stale address behind. Every call runs its kernels on
// the legacy default stream, reads reduction results back to the host with
// cudaMemcpy each sweep and ends with cudaDeviceSynchronize: it must not be
// called while any stream on the device is being captured.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "common.h"
#include "device.cuh"

namespace {

using excent::ull;

constexpr int NOALLOC_MAX_N = EXCENT_NOALLOC_MAX_N;
constexpr int NOALLOC_RED = 64;   // reduction slots (doubles) after the two vectors

static __device__ __align__(256) double g_noalloc_scratch[2 * (size_t)NOALLOC_MAX_N + NOALLOC_RED];

// y[v] = sum over the list of v of x[u]; one warp per vertex.
__global__ void k_na_spmv(int n, const ull* idx, const int* adj, const double* x, double* y, double c, double s) {
    const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    double acc = 0;
    for (ull e = idx[w] + lane; e < idx[w + 1]; e += 32) acc += x[adj[e]];
    acc = excent::warp_sum(acc);
    if (lane == 0) y[w] = c + s * acc;
}

// red[0] += sum x^2, red[1] += sum x
__global__ void k_na_norms(int n, const double* x, double* red) {
    double a = 0, b = 0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        a += x[v] * x[v];
        b += x[v];
    }
    a = excent::warp_sum(a);
    b = excent::warp_sum(b);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&red[0], a);
        atomicAdd(&red[1], b);
    }
}

__global__ void k_na_affine(int n, double* x, double f, double add) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        x[v] = x[v] * f + add;
}

__global__ void k_na_tofloat(int n, const double* x, float* y) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        y[v] = (float)x[v];
}

// Device address of the scratch array on the current device, looked up on
// every call (the caller has made the device current).
int scratch_address(double** out) {
    double* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        EX_FAIL(EXCENT_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed (%s)", cudaGetErrorString(e));
    *out = p;
    return EXCENT_OK;
}

// Zero the two reduction sums, launch the norms, read them back.
int sums(int n, const double* x, double* red, int grid, double* ss, double* sum) {
    EX_CUDA(cudaMemsetAsync(red, 0, 2 * sizeof(double), 0));
    k_na_norms<<<grid, 256>>>(n, x, red);
    double h[2];
    EX_CUDA(cudaMemcpy(h, red, sizeof h, cudaMemcpyDeviceToHost));
    if (ss) *ss = h[0];
    if (sum) *sum = h[1];
    return EXCENT_OK;
}

}  // namespace

extern "C" int excent_params_fp64_noalloc(int device, int n, const unsigned long long* d_idx, const int32_t* d_adj,
                                          double katz_numerator, double* out, float* d_v1) {
    EX_CHECK_ARG(d_idx && d_adj && out, "null argument");
    EX_CHECK_ARG(n >= 1, "n must be >= 1");
    EX_CHECK_ARG(n <= NOALLOC_MAX_N,
                 "n = %d exceeds the %d vertices the static scratch of excent_params_fp64_noalloc holds; "
                 "use excent_params_fp64", n, NOALLOC_MAX_N);
    EX_CUDA(cudaSetDevice(device));
    double* base = nullptr;
    EX_TRY(scratch_address(&base));
    double* v0 = base;
    double* v1 = base + NOALLOC_MAX_N;
    double* red = base + 2 * (size_t)NOALLOC_MAX_N;
    int sms = 0;
    EX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int G = sms * 8;
    const unsigned wb = (unsigned)(((long long)n * 32 + 255) / 256);
    // lambda1 from the unit all-ones vector; stop at a relative change < 1e-12 after 10 sweeps
    k_na_affine<<<G, 256>>>(n, v0, 0.0, 1.0 / std::sqrt((double)n));
    double lam = 0, lamPrev = 0, ss = 0, vsum = 0;
    int pit = 0;
    for (; pit < 5000; pit++) {
        k_na_spmv<<<wb, 256>>>(n, d_idx, d_adj, v0, v1, 0.0, 1.0);
        EX_TRY(sums(n, v1, red, G, &ss, nullptr));
        if (!(ss > 0)) EX_FAIL(EXCENT_ERR_ARG, "params: the graph has no edges (A x = 0), lambda1 is undefined");
        lam = std::sqrt(ss);
        k_na_affine<<<G, 256>>>(n, v1, 1.0 / lam, 0.0);
        std::swap(v0, v1);
        if (pit > 10 && std::fabs(lam - lamPrev) / lam < 1e-12) break;
        lamPrev = lam;
    }
    EX_TRY(sums(n, v0, red, G, nullptr, &vsum));
    const double meanEV = vsum * vsum / n;
    if (d_v1) k_na_tofloat<<<G, 256>>>(n, v0, d_v1);
    // Katz fixed point x = 1 + alpha A x for its mean
    const double alpha = katz_numerator / lam;
    k_na_affine<<<G, 256>>>(n, v0, 0.0, 1.0);
    double meanK = 0;
    for (int it = 0; it < 5000; it++) {
        k_na_spmv<<<wb, 256>>>(n, d_idx, d_adj, v0, v1, 1.0, alpha);
        std::swap(v0, v1);
        double sum = 0;
        EX_TRY(sums(n, v0, red, G, nullptr, &sum));
        const double nm = sum / n;
        if (std::fabs(nm - meanK) / nm < 1e-12) { meanK = nm; break; }
        meanK = nm;
    }
    EX_CUDA(cudaGetLastError());
    EX_CUDA(cudaDeviceSynchronize());
    out[0] = lam; out[1] = alpha; out[2] = meanEV; out[3] = meanK; out[4] = pit;
    return EXCENT_OK;
}
