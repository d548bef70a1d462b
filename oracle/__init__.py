"""CPU oracle for the ExCent delta-push centrality path.

TEST INFRASTRUCTURE ONLY. This package is the checker: only the test suite,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it.
The product (``excent_b200``) never imports it.

It wraps ``oracle/liboracle.so`` (built from ``oracle/oracle.c``) and adds the
numpy pieces: the EGR file format, CSR construction for the synthetic R-MAT
graphs, and the result metrics of the reference's comparison tool.
Reference citations are relative to the SPADE-IITJ/ExCent project.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_u64p = C.POINTER(C.c_uint64)
_i32p = C.POINTER(C.c_int32)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
_u16p = C.POINTER(C.c_uint16)


def reference_root() -> str:
    """Where the reference checkout is: $EXCENT_REFERENCE, else the Makefile's REF default."""
    r = os.environ.get("EXCENT_REFERENCE")
    if r:
        return r
    out = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True)
    return out.stdout.strip()


def build() -> None:
    """Compile liboracle.so (and the reference harnesses when the reference checkout exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    ref = reference_root()
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.or_rmat_key.restype = C.c_uint64
        L.or_rmat_key.argtypes = [C.c_uint64]
        L.or_rmat_pairs.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, _i32p, _i32p]
        L.or_rmat_weights.argtypes = [C.c_uint64, C.c_uint64, _f32p]
        L.or_jacobi.restype = C.c_int
        L.or_jacobi.argtypes = [C.c_int, _u64p, _i32p, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double,
                                C.c_int, _f64p, _f64p]
        L.or_power.restype = C.c_int
        L.or_power.argtypes = [C.c_int, _u64p, _i32p, C.c_double, C.c_int, _f64p, _f64p]
        L.or_unit.argtypes = [C.c_int, _f64p]
        L.or_params.argtypes = [C.c_int, _u64p, _i32p, _f64p]
        L.or_snapshot.argtypes = [C.c_int, C.c_int, _f32p, _f32p, _u64p, _i32p, C.c_int, _u32p, _u32p, _u64p, _u64p,
                                  _u16p]
        L.or_init.argtypes = [C.c_int, C.c_int, _u64p, C.c_double, C.c_double, _f32p, _f32p]
        L.or_delta_push.restype = C.c_int
        L.or_delta_push.argtypes = [C.c_int, C.c_int, _u64p, _i32p, _i32p, C.c_int, _f32p, _f32p, _i32p, C.c_double,
                                    C.c_int, C.c_uint64, C.c_int, _f32p, _f32p, _u64p]
        L.or_plan_chunks.restype = C.c_int
        L.or_plan_chunks.argtypes = [C.c_int, _u64p, C.c_uint64, _u64p]
        L.or_chunk_cap.restype = C.c_uint64
        L.or_chunk_cap.argtypes = [C.c_uint64, C.c_double, C.c_double, C.c_double]
        L.or_fetch_plan.argtypes = [C.c_int, _u64p, _u8p, _u8p, C.c_double, _u64p, C.c_int, C.c_int, _i32p, _i32p,
                                    _u8p, _u64p, _u64p, C.POINTER(C.c_int)]
        L.or_gather_list.restype = C.c_int
        L.or_gather_list.argtypes = [C.c_int, C.c_int, _u32p, _u64p, _i32p, _u64p]
        L.or_prefetch_runs.argtypes = [_i32p, C.c_int, _u64p, C.c_uint64, C.c_uint64, C.c_int, _u64p, _u64p]
        L.or_cache_chunks.restype = C.c_int
        L.or_cache_chunks.argtypes = [C.c_int, _u64p, C.c_uint64, C.c_uint64]
        L.or_hot_select.restype = C.c_int
        L.or_hot_select.argtypes = [C.c_int, _u64p, C.c_uint64, _i32p, _u64p, _u64p]
        L.or_tau.restype = C.c_double
        L.or_tau.argtypes = [C.c_double, _f64p, _f64p]
        L.or_ppr.restype = C.c_int
        L.or_ppr.argtypes = [C.c_int, _u64p, _i32p, C.c_int, C.c_double, _f64p, C.c_double, C.c_int, _f64p]
        L.or_row_normalise.argtypes = [C.c_int, _u64p, _f32p, _f64p]
        L.or_wfwd.restype = C.c_int
        L.or_wfwd.argtypes = [C.c_int, _u64p, _i32p, _f64p, C.c_double, C.c_double, _f64p, C.c_double, C.c_int, _f64p]
        L.or_wadj.restype = C.c_int
        L.or_wadj.argtypes = [C.c_int, _u64p, _i32p, _f64p, C.c_double, _f64p, C.c_double, C.c_int, _f64p]
        L.or_wgrad.argtypes = [C.c_int, _u64p, _i32p, _f32p, _f64p, C.c_double, _f64p, _f64p, _f64p]
        L.or_csr_build.restype = C.c_uint64
        L.or_csr_build.argtypes = [C.c_int, C.c_uint64, _i32p, _i32p, C.c_int, _u64p, _i32p]
        L.or_lambda1.restype = C.c_double
        L.or_lambda1.argtypes = [C.c_int, _u64p, _i32p, C.c_double, C.c_int]
        _lib = L
    return _lib


def P(a, t):
    """ctypes pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return C.cast(0, t)
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


# ------------------------------------------------------------------ EGR format

def read_egr(path):
    """EGR binary CSR (little-endian): int32 n, int32 m or -1, [int64 m], nindex[n+1]
    (int64 iff -1, else int32 read as uint32), int32 nlist[m]. Restates the layout of
    README.md:136-146 and the parse of include/StaticGraph.h:32-56."""
    with open(path, "rb") as f:
        b = f.read()
    n, e32 = np.frombuffer(b[:8], dtype="<i4")
    off = 8
    if e32 == -1:
        m = int(np.frombuffer(b[8:16], dtype="<i8")[0])
        off = 16
        idx = np.frombuffer(b[off:off + 8 * (n + 1)], dtype="<u8").astype(np.uint64)
        off += 8 * (n + 1)
    else:
        m = int(e32)
        idx = np.frombuffer(b[off:off + 4 * (n + 1)], dtype="<u4").astype(np.uint64)
        off += 4 * (n + 1)
    adj = np.frombuffer(b[off:off + 4 * m], dtype="<i4").astype(np.int32)
    if len(adj) != m:
        raise ValueError(f"{path}: truncated nlist ({len(adj)} of {m})")
    return int(n), np.ascontiguousarray(idx), np.ascontiguousarray(adj)


def write_egr(path, idx, adj, wide=True):
    n = len(idx) - 1
    with open(path, "wb") as f:
        if wide:
            f.write(np.array([n, -1], dtype="<i4").tobytes())
            f.write(np.array([len(adj)], dtype="<i8").tobytes())
            f.write(np.asarray(idx, dtype="<u8").tobytes())
        else:
            f.write(np.array([n, len(adj)], dtype="<i4").tobytes())
            f.write(np.asarray(idx, dtype="<u4").tobytes())
        f.write(np.asarray(adj, dtype="<i4").tobytes())


# ------------------------------------------------------------------ R-MAT

def rmat_thresholds(a=0.57, b=0.19, c=0.19):
    """32-bit quadrant thresholds; same arithmetic as the product's generator."""
    return int(a * 4294967296.0), int((a + b) * 4294967296.0), int((a + b + c) * 4294967296.0)


def rmat_pairs(scale, npairs, seed, abc=(0.57, 0.19, 0.19)):
    tA, tAB, tABC = rmat_thresholds(*abc)
    src = np.empty(npairs, dtype=np.int32)
    dst = np.empty(npairs, dtype=np.int32)
    lib().or_rmat_pairs(scale, npairs, seed, tA, tAB, tABC, P(src, _i32p), P(dst, _i32p))
    return src, dst


def csr_from_pairs(n, src, dst, symmetric=True):
    """Add both directions (symmetric), drop self-loops and duplicates, sort each list."""
    s = src.astype(np.int64)
    d = dst.astype(np.int64)
    if symmetric:
        s, d = np.concatenate([s, d]), np.concatenate([d, s])
    keep = s != d
    key = np.unique((s[keep] << 32) | d[keep])
    rows = (key >> 32).astype(np.int64)
    adj = (key & 0xFFFFFFFF).astype(np.int32)
    idx = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(np.bincount(rows, minlength=n), out=idx[1:])
    return idx, np.ascontiguousarray(adj)


def csr_build(n, src, dst, symmetric=True):
    """OpenMP CSR build (oracle.c or_csr_build); same result as csr_from_pairs."""
    idx = np.zeros(n + 1, dtype=np.uint64)
    adj = np.empty(max(1, len(src) * (2 if symmetric else 1)), dtype=np.int32)
    m = lib().or_csr_build(n, len(src), P(src, _i32p), P(dst, _i32p), int(symmetric), P(idx, _u64p), P(adj, _i32p))
    return idx, adj[:m].copy() if m < len(adj) // 2 else np.ascontiguousarray(adj[:m])


def rmat_graph(scale, edge_factor, seed, symmetric=True, fast=False):
    n = 1 << scale
    npairs = n * edge_factor // 2 if symmetric else n * edge_factor
    src, dst = rmat_pairs(scale, npairs, seed)
    idx, adj = (csr_build if fast else csr_from_pairs)(n, src, dst, symmetric)
    return n, idx, adj


def lambda1(n, idx, adj, tol=1e-10, maxit=5000):
    return float(lib().or_lambda1(n, P(idx, _u64p), P(adj, _i32p), tol, maxit))


def rmat_weights(m, seed):
    w = np.empty(m, dtype=np.float32)
    lib().or_rmat_weights(m, seed, P(w, _f32p))
    return w


# ------------------------------------------------------------------ solvers

def jacobi(n, idx, adj, measure, alpha=None, beta=1.0, tol=1e-9, maxit=20000):
    """FP64 reference for pr / katz (tools/centrality_reference.cu:184-214)."""
    x = np.empty(n, dtype=np.float64)
    rel = C.c_double()
    if measure == "pr":
        it = lib().or_jacobi(n, P(idx, _u64p), P(adj, _i32p), 0.15, 0.85, 1, 0.15, tol, maxit, P(x, _f64p),
                             C.byref(rel))
    elif measure == "katz":
        it = lib().or_jacobi(n, P(idx, _u64p), P(adj, _i32p), beta, alpha, 0, 1.0, tol, maxit, P(x, _f64p),
                             C.byref(rel))
    else:
        lam = C.c_double()
        it = lib().or_power(n, P(idx, _u64p), P(adj, _i32p), tol, maxit, P(x, _f64p), C.byref(lam))
        return x, it
    return x, it


def reference_solution(n, idx, adj, measure, alpha=None, beta=1.0):
    return jacobi(n, idx, adj, measure, alpha=alpha, beta=beta)[0]


def params(n, idx, adj):
    """Given constants (tools/excent_params.cu:133-172) as the .env strings it writes."""
    out = np.zeros(5, dtype=np.float64)
    lib().or_params(n, P(idx, _u64p), P(adj, _i32p), P(out, _f64p))
    lam, alpha, mean_ev, mean_k, pit = out
    return {
        "LAMBDA": "%.10f" % lam, "ALPHA": "%.6g" % alpha, "BETA": "1", "EPS_PR": "0.01",
        "EPS_KATZ": "%.6g" % (0.01 * mean_k), "EPS_EV": "%.6g" % (0.01 * mean_ev),
        "_lambda": lam, "_mean_ev": mean_ev, "_mean_k": mean_k, "_pit": int(pit),
    }


def snapshot(n, r_list, eps, idx, cv0, hot=None, trace=None):
    """CPU k_snapshot (src/excent.cu:69-98): bitmap, cnt[2nc], hotpend."""
    nm = len(r_list)
    r = np.ascontiguousarray(np.stack([np.asarray(x, dtype=np.float32) for x in r_list]))
    epsa = np.asarray(eps, dtype=np.float32)
    cv0 = np.ascontiguousarray(cv0, dtype=np.int32)
    nc = len(cv0)
    bitmap = np.zeros((n + 31) // 32, dtype=np.uint32)
    cnt = np.zeros(2 * nc, dtype=np.uint64)
    hp = C.c_uint64()
    lib().or_snapshot(n, nm, P(r, _f32p), P(epsa, _f32p), P(idx, _u64p), P(cv0, _i32p), nc,
                      P(hot, _u32p), P(bitmap, _u32p), P(cnt, _u64p), C.byref(hp), P(trace, _u16p))
    return bitmap, cnt, hp.value


KINDS = {"pr": 0, "katz": 1, "ev": 2}


def engine_constants(kinds, alpha=None, beta=1.0, lam=None, eps_pr=0.01, eps_katz=None, eps_ev=None):
    """eps / scale / divdeg per measure as src/excent.cu:344-351 sets them (float32)."""
    eps, scale, divdeg = [], [], []
    for k in kinds:
        if k == "pr":
            eps.append(eps_pr); scale.append(0.85); divdeg.append(1)
        elif k == "katz":
            eps.append(eps_katz); scale.append(alpha); divdeg.append(0)
        else:
            eps.append(eps_ev); scale.append(1.0 / lam); divdeg.append(0)
    return (np.array(eps, dtype=np.float32), np.array(scale, dtype=np.float32), np.array(divdeg, dtype=np.int32))


def delta_push(n, idx, adj, kinds, cv0=None, alpha=None, beta=1.0, lam=None, eps_pr=0.01, eps_katz=None, eps_ev=None,
               list_frac=0.5, max_passes=100000, max_edges=0, threads=0):
    """CPU port of the engine (init src/excent.cu:41-47, push :100-124, passes :656-760)."""
    nm = len(kinds)
    x = np.zeros((nm, n), dtype=np.float32)
    r = np.zeros((nm, n), dtype=np.float32)
    for i, k in enumerate(kinds):
        lib().or_init(n, KINDS[k], P(idx, _u64p), beta, lam if lam else 1.0, P(x[i], _f32p), P(r[i], _f32p))
    eps, scale, divdeg = engine_constants(kinds, alpha, beta, lam, eps_pr, eps_katz, eps_ev)
    if cv0 is None:
        cv0 = np.zeros(1, dtype=np.int32)
    cv0 = np.ascontiguousarray(cv0, dtype=np.int32)
    pushed = C.c_uint64()
    passes = lib().or_delta_push(n, nm, P(idx, _u64p), P(adj, _i32p), P(cv0, _i32p), len(cv0), P(eps, _f32p),
                                 P(scale, _f32p), P(divdeg, _i32p), list_frac, max_passes, max_edges, threads,
                                 P(x, _f32p), P(r, _f32p), C.byref(pushed))
    return x, r, passes, pushed.value


def plan_chunks(idx, max_edges):
    n = len(idx) - 1
    nc = lib().or_plan_chunks(n, P(idx, _u64p), max_edges, P(None, _u64p))
    out = np.zeros(4 * nc, dtype=np.uint64)
    lib().or_plan_chunks(n, P(idx, _u64p), max_edges, P(out, _u64p))
    return out.reshape(nc, 4)


def chunk_cap(m, chunk_medges=0.0, target_chunks=16.0, min_chunk_medges=4.0):
    return int(lib().or_chunk_cap(m, chunk_medges, target_chunks, min_chunk_medges))


def fetch_plan(cnt, resident, loaded, stream_ratio, chunk_edges, hot_mode, pass_, hlo, hhi):
    nc = len(chunk_edges)
    mode = np.zeros(nc, dtype=np.uint8)
    pv, dm, nb = C.c_uint64(), C.c_uint64(), C.c_int()
    lib().or_fetch_plan(nc, P(np.ascontiguousarray(cnt, dtype=np.uint64), _u64p),
                        P(np.ascontiguousarray(resident, dtype=np.uint8), _u8p),
                        P(np.ascontiguousarray(loaded, dtype=np.uint8), _u8p), stream_ratio,
                        P(np.ascontiguousarray(chunk_edges, dtype=np.uint64), _u64p), int(hot_mode), pass_,
                        P(np.ascontiguousarray(hlo, dtype=np.int32), _i32p),
                        P(np.ascontiguousarray(hhi, dtype=np.int32), _i32p), P(mode, _u8p),
                        C.byref(pv), C.byref(dm), C.byref(nb))
    return mode, pv.value, dm.value, bool(nb.value)


def gather_list(v0, v1, bitmap, idx):
    vids = np.zeros(max(v1 - v0, 1), dtype=np.int32)
    off = np.zeros(max(v1 - v0, 1) + 1, dtype=np.uint64)
    k = lib().or_gather_list(v0, v1, P(bitmap, _u32p), P(idx, _u64p), P(vids, _i32p), P(off, _u64p))
    return vids[:k].copy(), off[:k + 1].copy()


def prefetch_runs(vids, idx, nlist_off, page=4096, io_threads=16):
    vids = np.ascontiguousarray(vids, dtype=np.int32)
    pg, rn = C.c_uint64(), C.c_uint64()
    lib().or_prefetch_runs(P(vids, _i32p), len(vids), P(idx, _u64p), nlist_off, page, io_threads,
                           C.byref(pg), C.byref(rn))
    return pg.value, rn.value


def cache_chunks(chunk_edges, free_bytes, reserve):
    ce = np.ascontiguousarray(chunk_edges, dtype=np.uint64)
    return lib().or_cache_chunks(len(ce), P(ce, _u64p), free_bytes, reserve)


def hot_select(idx, budget):
    n = len(idx) - 1
    ids = np.zeros(max(n, 1), dtype=np.int32)
    T, E = C.c_uint64(), C.c_uint64()
    nh = lib().or_hot_select(n, P(idx, _u64p), budget, P(ids, _i32p), C.byref(T), C.byref(E))
    return ids[:nh].copy(), T.value, E.value


def tau(t_stream, t_g, f):
    tg = np.ascontiguousarray(t_g, dtype=np.float64)
    ff = np.ascontiguousarray(f, dtype=np.float64)
    return lib().or_tau(t_stream, P(tg, _f64p), P(ff, _f64p))


def ppr(n, idx, adj, teleport, kind=0, d=0.85, tol=1e-12, maxit=100000):
    """FP64 personalized PageRank (kind 0) or Katz with a beta vector (kind 1)."""
    t = np.ascontiguousarray(teleport, dtype=np.float64)
    x = np.empty(n, dtype=np.float64)
    lib().or_ppr(n, P(idx, _u64p), P(adj, _i32p), kind, d, P(t, _f64p), tol, maxit, P(x, _f64p))
    return x


def row_normalise(idx, w):
    n = len(idx) - 1
    wn = np.empty(len(w), dtype=np.float64)
    lib().or_row_normalise(n, P(idx, _u64p), P(np.ascontiguousarray(w, dtype=np.float32), _f32p), P(wn, _f64p))
    return wn


def weighted_forward(idx, adj, wn, c, s, t, tol=1e-13, maxit=100000):
    n = len(idx) - 1
    x = np.empty(n, dtype=np.float64)
    lib().or_wfwd(n, P(idx, _u64p), P(adj, _i32p), P(np.ascontiguousarray(wn), _f64p), c, s,
                  P(np.ascontiguousarray(t, dtype=np.float64), _f64p), tol, maxit, P(x, _f64p))
    return x


def weighted_adjoint(idx, adj, wn, s, g, tol=1e-13, maxit=100000):
    n = len(idx) - 1
    lam = np.empty(n, dtype=np.float64)
    lib().or_wadj(n, P(idx, _u64p), P(adj, _i32p), P(np.ascontiguousarray(wn), _f64p), s,
                  P(np.ascontiguousarray(g, dtype=np.float64), _f64p), tol, maxit, P(lam, _f64p))
    return lam


def weighted_grad(idx, adj, w, wn, s, x, lam):
    n = len(idx) - 1
    gw = np.empty(len(adj), dtype=np.float64)
    lib().or_wgrad(n, P(idx, _u64p), P(adj, _i32p), P(np.ascontiguousarray(w, dtype=np.float32), _f32p),
                   P(np.ascontiguousarray(wn), _f64p), s, P(np.ascontiguousarray(x, dtype=np.float64), _f64p),
                   P(np.ascontiguousarray(lam, dtype=np.float64), _f64p), P(gw, _f64p))
    return gw


# ------------------------------------------------------------------ metrics

def unit(v):
    """tools/centrality_reference.cu:71-76: unit L2 norm, sign fixed by the sum."""
    v = np.asarray(v, dtype=np.float64)
    s = float(np.dot(v, v))
    t = float(v.sum())
    return v * ((-1.0 if t < 0 else 1.0) / np.sqrt(s))


def compare(measure, ref, x, K=100):
    """tools/centrality_reference.cu:78-106 (L1 rel, L2, top-K overlap) plus the
    max per-vertex error and the top-1000 overlap; ev compares unit vectors."""
    r = np.asarray(ref, dtype=np.float64)
    xx = np.asarray(x, dtype=np.float32).astype(np.float64)
    if measure == "ev":
        r, xx = unit(r), unit(xx)
    d = np.abs(xx - r)
    out = {"l1_rel": float(d.sum() / np.abs(r).sum()), "l1": float(d.sum()), "l2": float(np.sqrt((d * d).sum())),
           "max_abs": float(d.max()) if len(d) else 0.0}
    for k in (K, 1000):
        k = min(k, len(r))
        a = np.argsort(-r, kind="stable")[:k]
        b = np.argsort(-xx, kind="stable")[:k]
        out[f"top{k}"] = int(len(np.intersect1d(a, b)))
    return out


def rank_quality(measure, ref, x):
    """tools/centrality_reference.cu:109-139: P@k for k in 10..100000, Kendall tau@1000."""
    r = np.asarray(ref, dtype=np.float64)
    xx = np.asarray(x, dtype=np.float32).astype(np.float64)
    if measure == "ev":
        r, xx = unit(r), unit(xx)
    n = len(r)
    ir = np.lexsort((np.arange(n), -r))
    ix = np.lexsort((np.arange(n), -xx))
    out = {}
    for k in (10, 100, 1000, 10000, 100000):
        if k > n:
            break
        out[f"P@{k}"] = len(np.intersect1d(ir[:k], ix[:k])) / k
    T = min(1000, n)
    top = ir[:T]
    dr = r[top][:, None] - r[top][None, :]
    dx = xx[top][:, None] - xx[top][None, :]
    iu = np.triu_indices(T, 1)
    prod = (dr * dx)[iu]
    out["tau@1000"] = float(((prod > 0).sum() - (prod < 0).sum()) / (T * (T - 1) / 2))
    return out
