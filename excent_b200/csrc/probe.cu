// probe.cu -- excent_reduction_peak: the measured ceiling of the operation a
// scatter pass is made of, a reduction (red.global.add) of one FP32 value, or
// of a float4 of every measure, to a random vertex of an n-vertex residual
// array. On R-MAT graphs the residual array of one measure fits in L2 and the
// scatter is bound by the L2 reduction units rather than by DRAM, so this is
// the roofline its reductions per second are compared with (the HBM copy
// bandwidth is the other one).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.h"

namespace {

__device__ __forceinline__ unsigned mix32(unsigned x) {
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void k_red_probe1(float* r, unsigned n, unsigned long long ops, unsigned seed) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < ops; i += stride) {
        const unsigned u = mix32((unsigned)i ^ seed) % n;
        asm volatile("red.global.add.f32 [%0], %1;" ::"l"(r + u), "f"(1.0f) : "memory");
    }
}

__global__ void k_red_probe4(float4* r, unsigned n, unsigned long long ops, unsigned seed) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < ops; i += stride) {
        const unsigned u = mix32((unsigned)i ^ seed) % n;
        asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(r + u), "f"(1.0f), "f"(1.0f), "f"(1.0f),
                     "f"(0.0f)
                     : "memory");
    }
}

}  // namespace

extern "C" int excent_reduction_peak(int device, int n, int vec4, unsigned long long ops, double* per_second) {
    EX_CHECK_ARG(n >= 1 && ops >= 1 && per_second, "bad argument");
    EX_CUDA(cudaSetDevice(device));
    int sms = 0;
    EX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const size_t bytes = (size_t)n * (vec4 ? sizeof(float4) : sizeof(float));
    void* r = nullptr;
    if (cudaMalloc(&r, bytes) != cudaSuccess) { cudaGetLastError(); EX_FAIL(EXCENT_ERR_NOMEM, "probe array of %zu bytes", bytes); }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = EXCENT_OK;
    float best = 0.f;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = EXCENT_ERR_CUDA;
    for (int rep = 0; rc == EXCENT_OK && rep < 4; rep++) {   // the first launch warms up; best of the other three
        cudaEventRecord(e0);
        if (vec4) k_red_probe4<<<sms * 8, 256>>>((float4*)r, (unsigned)n, ops, 0x9e3779b9u * (rep + 1));
        else k_red_probe1<<<sms * 8, 256>>>((float*)r, (unsigned)n, ops, 0x9e3779b9u * (rep + 1));
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = EXCENT_ERR_CUDA; break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    const cudaError_t last = cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(r);
    if (rc != EXCENT_OK || last != cudaSuccess)
        EX_FAIL(EXCENT_ERR_CUDA, "reduction probe failed (%s)", cudaGetErrorString(last));
    *per_second = best > 0.f ? (double)ops / (best * 1e-3) : 0.0;
    return EXCENT_OK;
}
