// ref_kernels.cu -- host entry points that launch the reference's own device
// kernels (src/excent.cu of SPADE-IITJ/ExCent) on caller-provided device
// buffers, so GPU tests can compare the product's integer outputs (pending
// bitmap, per-chunk demand table, compacted lists) bit for bit with the
// reference kernels on identical residuals.
//
// TEST INFRASTRUCTURE ONLY (the checker). Built by oracle/Makefile into
// oracle/_ref/ from the reference source where it lies; the reference's
// main() is renamed so the translation unit links as a library.
#define main excent_reference_main
#include "excent.cu"
#undef main

static Measures make_measures(int nm, float** x, float** r, const float* eps, const float* scale,
                              const int* divdeg) {
    Measures M{};
    M.nm = nm;
    M.pushed = nullptr;
    for (int k = 0; k < nm; k++) {
        M.x[k] = x ? x[k] : nullptr; M.r[k] = r[k]; M.eps[k] = eps[k];
        M.scale[k] = scale ? scale[k] : 0.f; M.divdeg[k] = divdeg ? divdeg[k] : 0;
    }
    return M;
}

extern "C" {

// k_snapshot as launched at src/excent.cu:663 (cnt and hotpend are zeroed here, as :660-661 do).
int ref_snapshot(int n, int nm, float** d_r, const float* eps, const ull* d_idx, const int* d_cv0, int nc,
                 unsigned* d_bitmap, ull* d_cnt, const unsigned* d_hot, ull* d_hotpend, unsigned short* d_trace) {
    Measures M = make_measures(nm, nullptr, d_r, eps, nullptr, nullptr);
    cudaMemset(d_cnt, 0, 2 * (size_t)nc * sizeof(ull));
    cudaMemset(d_hotpend, 0, sizeof(ull));
    k_snapshot<<<(unsigned)(((size_t)n + 255) / 256), 256>>>(n, M, d_idx, d_cv0, nc, d_bitmap, d_cnt, d_hot,
                                                              d_hotpend, d_trace);
    return (int)cudaDeviceSynchronize();
}

// k_compact as launched at src/excent.cu:641-642.
int ref_compact(int v0, int v1, const unsigned* d_bitmap, int* d_out, unsigned* d_count) {
    cudaMemset(d_count, 0, sizeof(unsigned));
    k_compact<<<(unsigned)((v1 - v0 + 255) / 256), 256>>>(v0, v1, d_bitmap, d_out, d_count);
    return (int)cudaDeviceSynchronize();
}

// k_init as launched at src/excent.cu:370-372.
int ref_init(int n, const ull* d_idx, float* d_x, float* d_r, int kind, float beta, float lambda) {
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    k_init<<<sms * 8, 256>>>(n, d_idx, d_x, d_r, kind, beta, lambda);
    return (int)cudaDeviceSynchronize();
}

// k_compact_hot as launched at src/excent.cu:617-618.
int ref_compact_hot(int lo, int hi, const int* d_hids, int nm, float** d_r, const float* eps, int* d_out,
                    unsigned* d_count) {
    Measures M = make_measures(nm, nullptr, d_r, eps, nullptr, nullptr);
    cudaMemset(d_count, 0, sizeof(unsigned));
    k_compact_hot<<<(unsigned)((hi - lo + 255) / 256), 256>>>(lo, hi, d_hids, M, d_out, d_count);
    return (int)cudaDeviceSynchronize();
}

// k_fill_hot as launched at src/excent.cu:704-705.
int ref_fill_hot(int lo, int hi, const int* d_hids, const ull* d_hoff, const ull* d_idx, ull e0, const int* d_src,
                 int* d_hedges) {
    k_fill_hot<<<warp_grid(hi - lo), 256>>>(lo, hi, d_hids, d_hoff, d_idx, e0, d_src, d_hedges);
    return (int)cudaDeviceSynchronize();
}

}
