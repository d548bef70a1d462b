// device.cuh -- device-side building blocks shared by the sm_100a kernels:
// residual layouts, the take (exchange) of a vertex's residual, vector
// reductions into residuals, warp scans/shuffles and the warp-cooperative
// scatter of one adjacency list.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace excent {

typedef unsigned long long ull;
static constexpr unsigned FULL = 0xffffffffu;
static constexpr int MAXM = 3;

// Per-run measure constants as the kernels see them (src/excent.cu:29-37).
struct DevMeasures {
    int nm;
    float eps[MAXM];
    float scale[MAXM];
    int divdeg[MAXM];
};

// Residual/value layout: L == 1 stores one measure as float[n]; L == 4 stores
// up to three measures vertex-major as float4[n] = {m0, m1, m2, 0}, so one
// pushed edge updates all measures of its target with one 16-byte reduction.
template <int L> struct Lane;
template <> struct Lane<1> { typedef float T; };
template <> struct Lane<4> { typedef float4 T; };

__device__ __forceinline__ void red_add(float* r, int u, float p) {
    asm volatile("red.global.add.f32 [%0], %1;" ::"l"(r + u), "f"(p) : "memory");
}
__device__ __forceinline__ void red_add(float4* r, int u, float4 p) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(r + u), "f"(p.x), "f"(p.y), "f"(p.z),
                 "f"(p.w)
                 : "memory");
}

__device__ __forceinline__ bool nonzero(float p) { return p != 0.f; }
// measures a push weight carries (nonzero components)
__device__ __forceinline__ unsigned measures_in(float p) { return p != 0.f; }
__device__ __forceinline__ unsigned measures_in(float4 p) {
    return (unsigned)(p.x != 0.f) + (unsigned)(p.y != 0.f) + (unsigned)(p.z != 0.f);
}
__device__ __forceinline__ bool nonzero(float4 p) { return p.x != 0.f || p.y != 0.f || p.z != 0.f || p.w != 0.f; }

__device__ __forceinline__ float shfl(float v, int src) { return __shfl_sync(FULL, v, src); }
__device__ __forceinline__ float4 shfl(float4 v, int src) {
    return make_float4(__shfl_sync(FULL, v.x, src), __shfl_sync(FULL, v.y, src), __shfl_sync(FULL, v.z, src),
                       __shfl_sync(FULL, v.w, src));
}
template <typename T> __device__ __forceinline__ const T* shfl_ptr(const T* p, int src) {
    return (const T*)__shfl_sync(FULL, (unsigned long long)p, src);
}

template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    return v;  // valid in lane 0
}
__device__ __forceinline__ float4 warp_sum(float4 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(FULL, v.x, o);
        v.y += __shfl_down_sync(FULL, v.y, o);
        v.z += __shfl_down_sync(FULL, v.z, o);
        v.w += __shfl_down_sync(FULL, v.w, o);
    }
    return v;  // valid in lane 0
}
__device__ __forceinline__ unsigned warp_incl_scan(unsigned v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned t = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ bool bit_of(const uint32_t* bm, long long v) { return (bm[v >> 5] >> (v & 31)) & 1u; }

// Pending test over every measure (src/excent.cu:58-64).
__device__ __forceinline__ bool pending_of(float r, const DevMeasures& M) { return fabsf(r) > M.eps[0]; }
__device__ __forceinline__ bool pending_of(float4 r, const DevMeasures& M) {
    bool p = fabsf(r.x) > M.eps[0];
    if (M.nm > 1) p |= fabsf(r.y) > M.eps[1];
    if (M.nm > 2) p |= fabsf(r.z) > M.eps[2];
    return p;
}

// Take vertex v's residual for every measure still above its threshold:
// d = exchange(r[v], 0), x[v] += d (one writer per vertex), and return the
// per-edge push weight scale*d/(float)deg (divdeg) or scale*d
// (src/excent.cu:104-115, same evaluation order).
__device__ __forceinline__ float take(float* x, float* r, int v, ull deg, const DevMeasures& M) {
    float d = 0.f;
    if (fabsf(r[v]) > M.eps[0]) {
        d = atomicExch(&r[v], 0.f);
        x[v] += d;
    }
    if (d == 0.f) return 0.f;
    return M.divdeg[0] ? M.scale[0] * d / (float)deg : M.scale[0] * d;
}
__device__ __forceinline__ float take_one(float* rp, float rv, float eps) {
    return fabsf(rv) > eps ? atomicExch(rp, 0.f) : 0.f;
}
__device__ __forceinline__ float weight(float d, ull deg, const DevMeasures& M, int k) {
    if (d == 0.f) return 0.f;
    return M.divdeg[k] ? M.scale[k] * d / (float)deg : M.scale[k] * d;
}
__device__ __forceinline__ float4 take(float4* x, float4* r, int v, ull deg, const DevMeasures& M) {
    float4 rv = r[v];
    float* rp = reinterpret_cast<float*>(r + v);
    float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
    d.x = take_one(rp, rv.x, M.eps[0]);
    if (M.nm > 1) d.y = take_one(rp + 1, rv.y, M.eps[1]);
    if (M.nm > 2) d.z = take_one(rp + 2, rv.z, M.eps[2]);
    if (d.x != 0.f || d.y != 0.f || d.z != 0.f) {
        float4 xv = x[v];
        xv.x += d.x; xv.y += d.y; xv.z += d.z;
        x[v] = xv;
    }
    return make_float4(weight(d.x, deg, M, 0), weight(d.y, deg, M, 1), weight(d.z, deg, M, 2), 0.f);
}

__device__ __forceinline__ int ld_edge(const int* p) { return __ldcs(p); }

// Hub-target aggregation: in an encoded edge cache an entry < 0 names slot
// (entry & HUB_MASK) of a high-degree target; its contributions are summed in
// the CTA's shared accumulators (hacc) and flushed once per CTA.
static constexpr int HUB_MASK = 0x7fffffff;
__device__ __forceinline__ void hacc_add(float* hacc, int slot, float p) { atomicAdd(hacc + slot, p); }
__device__ __forceinline__ void hacc_add(float4* hacc, int slot, float4 p) {
    float* h = reinterpret_cast<float*>(hacc + slot);
    if (p.x != 0.f) atomicAdd(h, p.x);
    if (p.y != 0.f) atomicAdd(h + 1, p.y);
    if (p.z != 0.f) atomicAdd(h + 2, p.z);
}
template <typename P>
__device__ __forceinline__ void scatter_one(P* r, int u, P p, P* hacc) {
    if (u < 0) hacc_add(hacc, u & HUB_MASK, p);
    else red_add(r, u, p);
}
__device__ __forceinline__ int4 ld_edge4(const int4* p) { return __ldcs(p); }

// All 32 lanes scatter one adjacency list nb[0..deg): peel to a 16-byte
// boundary, then 128-bit loads, then the tail.
template <typename P>
__device__ __forceinline__ void warp_scatter(P* r, const int* nb, unsigned deg, P p, int lane, P* hacc) {
    const unsigned mis = (unsigned)(((uintptr_t)nb >> 2) & 3u);
    unsigned head = (4u - mis) & 3u;
    if (head > deg) head = deg;
    if (lane < (int)head) scatter_one(r, ld_edge(nb + lane), p, hacc);
    const int4* body = reinterpret_cast<const int4*>(nb + head);
    const unsigned nbody = (deg - head) >> 2;
    unsigned i = lane;
    for (; i + 96 < nbody; i += 128) {  // four 128-bit loads in flight per lane
        const int4 q0 = ld_edge4(body + i), q1 = ld_edge4(body + i + 32);
        const int4 q2 = ld_edge4(body + i + 64), q3 = ld_edge4(body + i + 96);
        scatter_one(r, q0.x, p, hacc); scatter_one(r, q0.y, p, hacc); scatter_one(r, q0.z, p, hacc); scatter_one(r, q0.w, p, hacc);
        scatter_one(r, q1.x, p, hacc); scatter_one(r, q1.y, p, hacc); scatter_one(r, q1.z, p, hacc); scatter_one(r, q1.w, p, hacc);
        scatter_one(r, q2.x, p, hacc); scatter_one(r, q2.y, p, hacc); scatter_one(r, q2.z, p, hacc); scatter_one(r, q2.w, p, hacc);
        scatter_one(r, q3.x, p, hacc); scatter_one(r, q3.y, p, hacc); scatter_one(r, q3.z, p, hacc); scatter_one(r, q3.w, p, hacc);
    }
    for (; i < nbody; i += 32) {
        const int4 q = ld_edge4(body + i);
        scatter_one(r, q.x, p, hacc); scatter_one(r, q.y, p, hacc); scatter_one(r, q.z, p, hacc); scatter_one(r, q.w, p, hacc);
    }
    const unsigned tail = (deg - head) & 3u;
    if (lane < (int)tail) scatter_one(r, ld_edge(nb + head + nbody * 4 + lane), p, hacc);
}

// ---- bulk-copy staging (cp.async.bulk with an mbarrier, one per warp) ----
// Plain, non-multicast bulk copies from this GPU's own memory into the CTA's
// shared memory: 16-byte aligned source, destination and size.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void bar_init(unsigned long long* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Lane 0: expect `bytes` on the barrier and start the copy global -> shared.
__device__ __forceinline__ void bulk_stage(unsigned long long* bar, void* dst, const void* src, unsigned bytes) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier reads of dst come first
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
// Wait for the phase `parity` of the barrier to complete, at most `limit`
// polls; false if it did not.
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, unsigned parity, unsigned limit) {
    for (unsigned it = 0; it < limit; it++) {
        unsigned done = 0;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace excent
