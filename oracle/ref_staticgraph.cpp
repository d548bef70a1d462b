// ref_staticgraph.cpp -- C entry points around the reference's own header-only
// storage reader (include/StaticGraph.h of SPADE-IITJ/ExCent), so the tests can
// pin the product's chunk planner, EGR parsing and gather page-run counts
// against the reference code itself.
//
// TEST INFRASTRUCTURE ONLY (the checker). Built by oracle/Makefile into
// oracle/_ref/ with the include path pointing at the reference checkout; the
// header is compiled where it lies and is not copied.
#include "StaticGraph.h"

extern "C" {

void* ref_sg_open(const char* path, int io_threads, int offsets_in_ram) {
    return new StaticGraph(path, io_threads, offsets_in_ram != 0);
}
void ref_sg_close(void* h) { delete (StaticGraph*)h; }
int ref_sg_n(void* h) { return ((StaticGraph*)h)->n; }
ull ref_sg_m(void* h) { return ((StaticGraph*)h)->m; }
ull ref_sg_degree(void* h, int v) { return ((StaticGraph*)h)->degree(v); }
ull ref_sg_offset(void* h, ull v) { return ((StaticGraph*)h)->offset((size_t)v); }
void ref_sg_read_offsets(void* h, ull v0, ull cnt, ull* dst) { ((StaticGraph*)h)->read_offsets(v0, cnt, dst); }
void ref_sg_read_edges(void* h, ull e0, ull e1, int* dst) { ((StaticGraph*)h)->read_edges(e0, e1, dst); }
void ref_sg_copy_list(void* h, int v, int* dst) {
    StaticGraph* g = (StaticGraph*)h;
    memcpy(dst, g->edges(v), g->degree(v) * sizeof(int));
}
int ref_sg_plan_chunks(void* h, ull max_edges, ull* out, int cap) {
    std::vector<EdgeChunk> ch = ((StaticGraph*)h)->plan_chunks(max_edges);
    for (int c = 0; c < (int)ch.size() && c < cap; c++) {
        out[4 * c] = (ull)ch[c].v0; out[4 * c + 1] = (ull)ch[c].v1;
        out[4 * c + 2] = ch[c].e0; out[4 * c + 3] = ch[c].e1;
    }
    return (int)ch.size();
}
void ref_sg_prefetch(void* h, const int* vids, int k, ull* pages, ull* runs) {
    ((StaticGraph*)h)->prefetch_lists(vids, k, pages, runs);
}

}
