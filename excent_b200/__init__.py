"""excent_b200 -- B200 (sm_100a) engine for ExCent's delta-push centrality path.

Python is a thin ctypes layer over libexcent_b200.so (include/excent_b200.h);
all computation runs in the library's CUDA kernels. There is no CPU fallback:
the first call into the engine without the built library raises ImportError.

Host-side mirror of the reference's option surface (src/excent.cu:251-316):
``measures("all", alpha=..., lam=..., eps_katz=..., eps_ev=...)`` builds the
measure table; ``Engine`` owns the device state of one run; ``DeviceGraph``
generates seeded R-MAT graphs on the device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi
from ._capi import ExcentError, Measures, PassLog, Stats, call, load

KIND_NAMES = {0: "pr", 1: "katz", 2: "ev"}


def _ptr(a, t=None):
    """Address of a numpy array / torch tensor / int as a void pointer value."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the engine must be contiguous"
    return a.ctypes.data


def _tp(a, t):
    return C.cast(_ptr(a), t) if a is not None else C.cast(0, t)


EV_INIT_FP64 = 1


def measures(measure, alpha=-1.0, beta=1.0, lam=-1.0, eps_pr=0.01, eps_katz=-1.0, eps_ev=-1.0,
             ev_init_fp64=False) -> Measures:
    """--measure pr|katz|ev|all with --alpha/--beta/--lambda/--eps-* (src/excent.cu:292-316, 344-351).
    ev_init_fp64: eigenvector initial residual from the FP64 lambda1 (the reference rounds it to float)."""
    M = Measures()
    call("excent_measures_make", C.byref(M), measure.encode(), float(alpha), float(beta), float(lam),
         float(eps_pr), float(eps_katz), float(eps_ev))
    if ev_init_fp64:
        M.flags |= EV_INIT_FP64
    return M


def plan_chunks(idx, max_edges):
    """Greedy contiguous chunks of <= max_edges edges, >= 1 vertex each
    (include/StaticGraph.h:128-139). Returns (v0[nc] int32, e[nc+1] uint64)."""
    idx = np.asarray(idx, dtype=np.uint64)
    n = len(idx) - 1
    v0s, es = [], [0]
    v = 0
    while v < n:
        limit = int(idx[v]) + int(max_edges)
        v1 = int(np.searchsorted(idx[v + 1:n + 1], limit, side="right")) + v
        if v1 <= v:
            v1 = v + 1
        v0s.append(v)
        es.append(int(idx[v1]))
        v = v1
    return np.array(v0s, dtype=np.int32), np.array(es, dtype=np.uint64)


def chunk_cap(m, chunk_medges=0.0, target_chunks=16.0, min_chunk_medges=4.0):
    """Edge cap per chunk (src/excent.cu:321-326)."""
    if chunk_medges > 0:
        return int(chunk_medges * 1e6)
    import math
    lo, hi = int(min_chunk_medges * 1e6), 64000000
    return min(hi, max(lo, int(math.ceil(m / target_chunks))))


class Engine:
    """Device state of one run: offsets, values/residuals, bitmap, demand
    table, pending lists and the HBM edge cache (include/excent_b200.h)."""

    def __init__(self, n, m, meas: Measures, chunk_v0, chunk_e, device=0):
        self.n, self.m, self.meas = int(n), int(m), meas
        self.chunk_v0 = np.ascontiguousarray(chunk_v0, dtype=np.int32)
        self.chunk_e = np.ascontiguousarray(chunk_e, dtype=np.uint64)
        self.nc = len(self.chunk_v0)
        h = C.c_void_p()
        call("excent_engine_create", int(device), self.n, self.m, C.byref(meas), self.nc,
             _tp(self.chunk_v0, _capi.i32p), _tp(self.chunk_e, _capi.u64p), C.byref(h))
        self.h = h

    def close(self):
        if self.h:
            call("excent_engine_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----- graph upload
    def upload_offsets(self, idx, v0=0, count=None):
        count = (self.n + 1 - v0) if count is None else count
        call("excent_engine_upload_offsets", self.h, _ptr(idx), v0, count)

    def reserve_cache(self, edges):
        call("excent_engine_reserve_cache", self.h, int(edges))

    def load_cache(self, e0, e1, edges):
        call("excent_engine_load_cache", self.h, int(e0), int(e1), _ptr(edges))

    def upload_graph(self, idx, adj):
        """Host CSR -> device offsets and a full edge cache."""
        self.upload_offsets(idx)
        self.reserve_cache(self.m)
        if self.m:
            self.load_cache(0, self.m, adj)

    def upload_device(self, d_idx, d_adj):
        call("excent_engine_upload_device", self.h, _ptr(d_idx), _ptr(d_adj))

    def set_loaded(self, c, loaded=True):
        call("excent_engine_set_loaded", self.h, int(c), int(loaded))

    # ----- passes
    def init(self):
        call("excent_engine_init", self.h)

    def snapshot(self, use_hot=False):
        cnt = np.zeros(2 * self.nc, dtype=np.uint64)
        hp = C.c_uint64()
        rs = np.zeros(3, dtype=np.float64)
        call("excent_engine_snapshot", self.h, int(use_hot), _tp(cnt, _capi.u64p), C.byref(hp), _tp(rs, _capi.f64p))
        return cnt, hp.value, rs[:self.meas.nm].copy()

    def bitmap(self):
        w = np.zeros((self.n + 31) // 32, dtype=np.uint32)
        call("excent_engine_bitmap", self.h, _tp(w, _capi.u32p))
        return w

    def chunk_list(self, c):
        nv = int((self.chunk_v0[c + 1] if c + 1 < self.nc else self.n) - self.chunk_v0[c])
        ids = np.zeros(max(nv, 1), dtype=np.int32)
        k = C.c_uint()
        call("excent_engine_chunk_list", self.h, int(c), _tp(ids, _capi.i32p), C.byref(k))
        return ids[:k.value].copy()

    def push_cached(self, mode, cnt, list_frac=0.5):
        mode = np.ascontiguousarray(mode, dtype=np.uint8)
        cnt = np.ascontiguousarray(cnt, dtype=np.uint64)
        call("excent_engine_push_cached", self.h, _tp(mode, _capi.u8p), _tp(cnt, _capi.u64p), float(list_frac))

    def sync(self):
        call("excent_engine_sync", self.h)

    def solve(self, list_frac=0.5, max_passes=100000, use_graph=True):
        """Device solve of a fully cached graph; returns Stats."""
        call("excent_engine_solve", self.h, float(list_frac), int(max_passes), int(use_graph))
        return self.stats()

    def stats(self, with_log=False):
        st = Stats()
        if with_log:
            cap = 1 << 17
            log = (PassLog * cap)()
            call("excent_engine_stats", self.h, C.byref(st), log, cap)
            return st, [log[i] for i in range(min(st.passes, cap))]
        call("excent_engine_stats", self.h, C.byref(st), None, 0)
        return st

    def read(self, i, residual=False, out=None):
        if out is None:
            out = np.empty(self.n, dtype=np.float32)
        call("excent_engine_read", self.h, int(i), int(residual), _ptr(out), 0, self.n)
        return out

    def write(self, i, x=None, r=None):
        x = None if x is None else np.ascontiguousarray(x, dtype=np.float32)
        r = None if r is None else np.ascontiguousarray(r, dtype=np.float32)
        call("excent_engine_write", self.h, int(i), _ptr(x), _ptr(r))

    def trace(self, enable=True):
        call("excent_engine_trace", self.h, int(enable))

    def read_trace(self):
        out = np.zeros(self.n, dtype=np.uint16)
        call("excent_engine_read_trace", self.h, _tp(out, _capi.u16p))
        return out

    def launches(self):
        v = C.c_uint64()
        call("excent_engine_launches", self.h, C.byref(v))
        return v.value

    def results(self):
        return [self.read(i) for i in range(self.meas.nm)]

    def set_hub_targets(self, k):
        """Shared-memory aggregation of the contributions to the k highest-degree targets (0: off)."""
        call("excent_engine_set_hub_targets", self.h, int(k))

    def set_hub_order(self, order="first"):
        """Device solve: where the lists longer than 256 entries go in each pass
        ("first", "last", or "table": with the rest)."""
        code = {"auto": -1, "table": 0, "first": 1, "last": 2, "launch-first": 3, False: 0, True: 1}[order]
        call("excent_engine_set_hub_order", self.h, code)

    def autotune(self, list_frac=0.5, max_passes=100000):
        """Time the candidate settings (excent_engine_autotune), keep the fastest; returns
        (best, [every candidate]) as dicts."""
        best = _capi.Tune()
        tried = (_capi.Tune * 16)()
        nt = C.c_int()
        call("excent_engine_autotune", self.h, float(list_frac), int(max_passes), C.byref(best), tried, 16,
             C.byref(nt))
        as_dict = lambda t: {"hub_targets": t.hub_targets,  # noqa: E731
                             "hub_order": ["table", "first", "last", "launch-first"][t.hub_order],
                             "chunk_sweep": bool(t.chunk_sweep), "sweep_demand": t.sweep_demand,
                             "ms": round(t.ms, 3)}
        return as_dict(best), [as_dict(tried[i]) for i in range(nt.value)]

    def scatter_peak(self):
        """Entries per second of one reduction per edge-cache entry (excent_engine_scatter_peak)."""
        v = C.c_double()
        call("excent_engine_scatter_peak", self.h, C.byref(v))
        return v.value

    def set_chunk_sweep(self, on=True):
        """Cached pushes one chunk per launch, in chunk order (the reference's launch order);
        "auto": when the graph has more than one chunk."""
        call("excent_engine_set_chunk_sweep", self.h, -1 if on == "auto" else int(bool(on)))

    def set_sweep_demand(self, frac):
        """Sweep (chunk by chunk) only the passes whose pending entries reach frac * m."""
        call("excent_engine_set_sweep_demand", self.h, float(frac))

    def set_claim_tiles(self, tiles=0):
        """Tiles of 32 items a push warp claims at a time (0: by the launch's size)."""
        call("excent_engine_set_claim_tiles", self.h, int(tiles))

    def host_cache(self):
        """Pinned host memory for the entries past the edge cache (excent_engine_host_cache):
        returns (numpy int32 view to fill, first edge index)."""
        p = C.c_void_p()
        first = C.c_uint64()
        call("excent_engine_host_cache", self.h, C.byref(p), C.byref(first))
        cnt = self.m - first.value
        if not cnt:
            return np.empty(0, dtype=np.int32), first.value
        buf = (C.c_int32 * cnt).from_address(p.value)
        return np.ctypeslib.as_array(buf), first.value

    def host_pushed(self):
        v = C.c_uint64()
        call("excent_engine_host_pushed", self.h, C.byref(v))
        return v.value

    def ev_project(self, v1):
        """FP64 eigenvector normalisation step with the unit principal eigenvector v1 (None: off)."""
        call("excent_engine_ev_project", self.h, _ptr(v1))

    def stream(self):
        """The engine's cudaStream_t as an integer handle (torch.cuda.ExternalStream accepts it)."""
        s = C.c_void_p()
        call("excent_engine_stream", self.h, C.byref(s))
        return s.value or 0

    def profile(self, enable=True):
        call("excent_engine_profile", self.h, int(enable))

    def profile_read(self):
        """Summed ms of {snapshot, plan, push, hub} over profiled passes, and the pass count."""
        ms = np.zeros(4, dtype=np.float64)
        p = C.c_uint64()
        call("excent_engine_profile_read", self.h, _tp(ms, _capi.f64p), C.byref(p))
        return dict(zip(("snapshot", "plan", "push", "hub"), ms.tolist())), p.value


def reduction_peak(n, vec4=False, ops=1 << 28, device=0):
    """Random FP32 (or float4) reductions per second into an n-vertex array (excent_reduction_peak)."""
    v = C.c_double()
    call("excent_reduction_peak", int(device), int(n), int(bool(vec4)), int(ops), C.byref(v))
    return v.value


def ppr_fp64(n, d_idx, d_adj, seeds, values, d=0.85, tol=1e-10, maxit=2000, device=0):
    """FP64 personalized PageRank of one seed set on a device graph (excent_ppr_fp64); values is a
    scalar (the same residual at every seed) or one value per seed."""
    seeds = np.ascontiguousarray(seeds, dtype=np.int32)
    vals = np.ascontiguousarray(np.broadcast_to(np.float32(values), seeds.shape), dtype=np.float32)
    x = np.empty(n, dtype=np.float64)
    it = C.c_int()
    call("excent_ppr_fp64", int(device), int(n), _ptr(d_idx), _ptr(d_adj), float(d), len(seeds), _ptr(seeds),
         _ptr(vals), float(tol), int(maxit), _tp(x, _capi.f64p), C.byref(it))
    return x, it.value


def write_egr(path, idx, adj, wide=True):
    """Write a CSR graph as an EGR file (README.md:136-146): int32 n, then int32 -1 and int64 m
    with uint64 offsets (wide), or int32 m with uint32 offsets (narrow); then int32 lists."""
    idx = np.asarray(idx)
    adj = np.asarray(adj)
    n = len(idx) - 1
    with open(path, "wb") as f:
        if wide:
            f.write(np.array([n, -1], dtype="<i4").tobytes())
            f.write(np.array([len(adj)], dtype="<i8").tobytes())
            f.write(np.ascontiguousarray(idx, dtype="<u8").tobytes())
        else:
            if len(adj) >= 2 ** 31:
                raise ValueError("narrow EGR holds fewer than 2^31 entries")
            f.write(np.array([n, len(adj)], dtype="<i4").tobytes())
            f.write(np.ascontiguousarray(idx, dtype="<u4").tobytes())
        f.write(np.ascontiguousarray(adj, dtype="<i4").tobytes())


def params_fp64(n, d_idx, d_adj, katz_numerator=0.85, device=0, v1_out=None):
    """Given constants of a device-resident symmetric graph (tools/excent_params.cu:133-163):
    {lambda, alpha, mean_ev, mean_katz, sweeps}; v1_out (device buffer of n float32) receives
    the unit principal eigenvector."""
    out = np.zeros(5, dtype=np.float64)
    call("excent_params_fp64", int(device), int(n), _ptr(d_idx), _ptr(d_adj), float(katz_numerator),
         _tp(out, _capi.f64p), _ptr(v1_out))
    return {"lambda": out[0], "alpha": out[1], "mean_ev": out[2], "mean_katz": out[3], "sweeps": int(out[4])}


def reference_fp64(n, d_idx, d_adj, measure, alpha=0.0, beta=1.0, tol=1e-9, maxit=20000, device=0):
    """FP64 reference solution on the device (tools/centrality_reference.cu:184-214)."""
    kind = {"pr": 0, "katz": 1, "ev": 2}[measure]
    x = np.empty(n, dtype=np.float64)
    it = C.c_int()
    call("excent_reference_fp64", int(device), int(n), _ptr(d_idx), _ptr(d_adj), kind, float(alpha), float(beta),
         float(tol), int(maxit), _tp(x, _capi.f64p), C.byref(it))
    return x, it.value


def rmat_write_egr(path, scale, edge_factor, seed, a=0.57, b=0.19, c=0.19, max_part_keys=0, device=0):
    """The symmetric R-MAT graph of DeviceGraph, generated in source partitions that fit device
    memory and written as a wide EGR file (excent_rmat_write_egr). Returns (m, partitions)."""
    m = C.c_uint64()
    parts = C.c_int()
    call("excent_rmat_write_egr", int(device), int(scale), int(edge_factor), int(seed), a, b, c,
         int(max_part_keys), os.fsencode(path), C.byref(m), C.byref(parts))
    return m.value, parts.value


class DeviceGraph:
    """Seeded R-MAT graph generated on the device (excent_rmat_generate)."""

    def __init__(self, scale, edge_factor, seed, a=0.57, b=0.19, c=0.19, symmetric=True, weights=False, device=0):
        h = C.c_void_p()
        call("excent_rmat_generate", int(device), int(scale), int(edge_factor), int(seed), a, b, c,
             int(symmetric), int(weights), C.byref(h))
        self.h = h
        n = C.c_int()
        m = C.c_uint64()
        call("excent_dgraph_info", h, C.byref(n), C.byref(m))
        self.n, self.m, self.weighted = n.value, m.value, bool(weights)

    def device_ptrs(self):
        i, a, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
        call("excent_dgraph_device_ptrs", self.h, C.byref(i), C.byref(a), C.byref(w))
        return i.value, a.value, w.value

    def download(self, idx=None, adj=None, w=None):
        """Copy to host arrays (numpy or pinned torch tensors); allocates numpy arrays if None."""
        if idx is None:
            idx = np.empty(self.n + 1, dtype=np.uint64)
        if adj is None:
            adj = np.empty(max(self.m, 1), dtype=np.int32)
        if w is None and self.weighted:
            w = np.empty(max(self.m, 1), dtype=np.float32)
        call("excent_dgraph_download", self.h, _ptr(idx), _ptr(adj), _ptr(w) if self.weighted else None)
        return idx, adj, w

    def close(self):
        if self.h:
            call("excent_dgraph_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """B personalized PageRank (kind "ppr") or Katz ("katz") solves at once on a
    device-resident graph (excent_batch_*), residuals vertex-major [n][B]."""

    def __init__(self, n, m, d_idx, d_adj, B, kind="ppr", d_or_alpha=0.85, device=0):
        h = C.c_void_p()
        k = {"ppr": 0, "katz": 1}[kind]
        call("excent_batch_create", int(device), int(n), int(m), _ptr(d_idx), _ptr(d_adj), int(B), k,
             float(d_or_alpha), C.byref(h))
        self.h, self.n, self.B, self.kind = h, int(n), int(B), kind

    def seed(self, seeds, values, eps):
        """seeds: list of vertex-id arrays (one per lane); values: matching arrays or scalars; eps per lane."""
        nq = len(seeds)
        off = np.zeros(nq + 1, dtype=np.int32)
        off[1:] = np.cumsum([len(s) for s in seeds])
        vids = np.ascontiguousarray(np.concatenate(seeds) if nq else np.zeros(0), dtype=np.int32)
        vals = np.ascontiguousarray(np.concatenate([np.broadcast_to(np.asarray(v, dtype=np.float32), (len(s),))
                                                    for s, v in zip(seeds, values)]) if nq else np.zeros(0),
                                    dtype=np.float32)
        e = np.ascontiguousarray(np.broadcast_to(np.asarray(eps, dtype=np.float32), (nq,)))
        call("excent_batch_seed", self.h, nq, _ptr(off), _ptr(vids) if len(vids) else None,
             _ptr(vals) if len(vals) else None, _ptr(e))

    def set_dense(self, groups=4):
        """Hub segments of rows with more active 16-byte groups than this scatter over the groups."""
        call("excent_batch_set_dense", self.h, int(groups))

    def set_greedy(self, greedy=True):
        call("excent_batch_set_greedy", self.h, int(greedy))

    def solve(self, max_passes=100000, use_graph=True):
        call("excent_batch_solve", self.h, int(max_passes), int(use_graph))
        return self.stats()

    def stats(self):
        p = C.c_int()
        v, e, u, c, hs = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        call("excent_batch_stats", self.h, C.byref(p), C.byref(v), C.byref(e), C.byref(u), C.byref(c), C.byref(hs))
        return {"passes": p.value, "pushed_vertices": v.value, "pushed_edges": e.value, "lane_updates": u.value,
                "rows_checked": c.value, "hub_segments": hs.value}

    def read(self, lane, residual=False, out=None):
        if out is None:
            out = np.empty(self.n, dtype=np.float32)
        call("excent_batch_read", self.h, int(lane), int(residual), _ptr(out))
        return out

    def stream(self):
        s = C.c_void_p()
        call("excent_batch_stream", self.h, C.byref(s))
        return s.value or 0

    def launches(self):
        v = C.c_uint64()
        call("excent_batch_launches", self.h, C.byref(v))
        return v.value

    def close(self):
        if self.h:
            call("excent_batch_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def seed_engine(eng, vids, vals):
    """Zero a single-measure engine and seed residuals (excent_engine_seed)."""
    vids = np.ascontiguousarray(vids, dtype=np.int32)
    vals = np.ascontiguousarray(np.broadcast_to(np.asarray(vals, dtype=np.float32), vids.shape))
    call("excent_engine_seed", eng.h, len(vids), _ptr(vids), _ptr(vals))


def resume(eng, list_frac=0.5, max_passes=100000, use_graph=True):
    call("excent_engine_resume", eng.h, float(list_frac), int(max_passes), int(use_graph))
    return eng.stats()


def _pack_queries(seeds, values, eps):
    nq = len(seeds)
    off = np.zeros(nq + 1, dtype=np.int32)
    off[1:] = np.cumsum([len(s) for s in seeds])
    vids = np.ascontiguousarray(np.concatenate(seeds), dtype=np.int32)
    vals = np.ascontiguousarray(np.concatenate([np.broadcast_to(np.asarray(v, dtype=np.float32), (len(s),))
                                                for s, v in zip(seeds, values)]), dtype=np.float32)
    e = np.ascontiguousarray(np.broadcast_to(np.asarray(eps, dtype=np.float32), (nq,)))
    return off, vids, vals, e


def autotune_batch(n, m, d_idx, d_adj, seeds, values, eps, kind="ppr", d_or_alpha=0.85, device=0, max_passes=100000):
    """Batch width and greedy mode with the lowest time per query on these queries
    (excent_batch_autotune): (B, greedy, {(B, greedy): ms per query})."""
    off, vids, vals, e = _pack_queries(seeds, values, eps)
    best = C.c_int()
    greedy = C.c_int()
    ms = np.zeros(8, dtype=np.float64)
    call("excent_batch_autotune", int(device), int(n), int(m), _ptr(d_idx), _ptr(d_adj), {"ppr": 0, "katz": 1}[kind],
         float(d_or_alpha), len(seeds), _ptr(off), _ptr(vids), _ptr(vals), _ptr(e), int(max_passes), C.byref(best),
         C.byref(greedy), _tp(ms, _capi.f64p))
    table = {(B, g): ms[2 * i + g] for i, B in enumerate((32, 64, 128, 256)) for g in (0, 1)}
    return best.value, bool(greedy.value), table


def shard(count, world, rank):
    """Contiguous share [lo, hi) of `count` independent units (queries, replicas) for `rank` of `world`."""
    lo = count * rank // world
    hi = count * (rank + 1) // world
    return lo, hi
