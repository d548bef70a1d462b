"""Parity of the CUDA engine with the oracle and with the reference's own kernels.

Integer work (pending bitmap, per-chunk demand table, hot pending count,
compacted pending lists) must be bit-exact; FP32 results are compared with the
FP64 oracle as L1 relative error, max per-vertex error and top-k overlap.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import excent_b200 as X  # noqa: E402


def chunks_for(idx, cap):
    v0, e = X.plan_chunks(idx, cap)
    return v0, e


def make_engine(n, idx, adj, meas, cap=None, upload_edges=True):
    m = len(adj)
    v0, e = chunks_for(idx, cap or max(m, 1))
    eng = X.Engine(n, m, meas, v0, e)
    if upload_edges:
        eng.upload_graph(idx, adj)
    else:
        eng.upload_offsets(idx)
    return eng


def meas_for(kinds, env=None, **kw):
    if env is not None:
        kw = dict(alpha=float(env["ALPHA"]), lam=float(env["LAMBDA"]), eps_katz=float(env["EPS_KATZ"]),
                  eps_ev=float(env["EPS_EV"]))
    return X.measures(kinds, **kw)


def bits_of(bm, n):
    v = np.arange(n)
    return ((bm[v >> 5] >> (v & 31)) & 1).astype(bool)


# ------------------------------------------------------------------ reference kernels

def ref_kernels():
    p = os.path.join(O.REF_DIR, "libexcent_ref.so")
    if not os.path.exists(p):
        pytest.skip("reference kernel harness not built (make -C oracle ref)")
    L = C.CDLL(p)
    L.ref_snapshot.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ref_compact.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.ref_init.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_float]
    return L


def snapshot_case(nm, seed, n, idx, cap, hot_frac):
    rng = np.random.default_rng(seed)
    eps = np.array([0.01, 0.05, 0.003][:nm], dtype=np.float32)
    r = [rng.normal(0, eps[k] * 1.2, n).astype(np.float32) for k in range(nm)]
    # some exact-threshold values: |r| == eps is not pending
    r[0][::97] = eps[0]
    v0, e = chunks_for(idx, cap)
    hot_ids = np.sort(rng.choice(n, max(1, int(hot_frac * n)), replace=False)).astype(np.int32)
    hot = np.zeros((n + 31) // 32, dtype=np.uint32)
    for v in hot_ids:
        hot[v >> 5] |= np.uint32(1 << int(v & 31))
    return eps, r, v0, e, hot_ids, hot


@pytest.mark.parametrize("nm", [1, 2, 3])
@pytest.mark.parametrize("cap", [37, 1000, 10 ** 9])
@pytest.mark.parametrize("use_hot", [False, True])
def test_snapshot_bitexact_vs_oracle_and_reference(rmat12, nm, cap, use_hot):
    n, idx, adj = rmat12
    eps, r, v0, e, hot_ids, hot = snapshot_case(nm, 11 + nm, n, idx, cap, 0.05)
    kinds = ["pr", "katz", "ev"][:nm]
    meas = X.measures("all" if nm == 3 else "pr", alpha=0.1, lam=10.0, eps_katz=1.0, eps_ev=1.0)
    meas.nm = nm
    for k in range(nm):
        meas.eps[k] = float(eps[k])
    eng = X.Engine(n, len(adj), meas, v0, e)
    eng.upload_offsets(idx)
    if use_hot:
        deg = np.diff(idx.astype(np.int64))[hot_ids]
        off = np.zeros(len(hot_ids) + 1, dtype=np.uint64)
        off[1:] = np.cumsum(deg)
        import excent_b200._capi as K
        K.call("excent_engine_hot_setup", eng.h, len(hot_ids), hot_ids.ctypes.data_as(K.i32p),
               off.ctypes.data_as(K.u64p), hot.ctypes.data_as(K.u32p))
    eng.init()
    eng.trace(True)
    for k in range(nm):
        eng.write(k, r=r[k])
    cnt, hp, rsum = eng.snapshot(use_hot=use_hot)
    bm = eng.bitmap()
    tr = eng.read_trace()
    bm_o, cnt_o, hp_o = O.snapshot(n, r, eps, idx, v0, hot if use_hot else None)
    assert np.array_equal(bm, bm_o)
    assert np.array_equal(cnt, cnt_o)
    assert hp == hp_o
    pend_any = np.zeros(n, bool)
    for k in range(nm):
        pend_any |= np.abs(r[k]) > eps[k]
        assert abs(rsum[k] - np.abs(r[k].astype(np.float64)).sum()) <= 1e-9 * max(1.0, rsum[k])
    assert np.array_equal(tr, pend_any.astype(np.uint16))
    bits = bits_of(bm, n)
    bounds = list(v0) + [n]
    for c in range(len(v0)):
        lst = np.sort(eng.chunk_list(c))
        want = np.nonzero(bits[bounds[c]:bounds[c + 1]])[0] + bounds[c]
        assert np.array_equal(lst, want), c
    # the reference's own k_snapshot on identical inputs
    L = ref_kernels()
    dev = torch.device("cuda")
    d_r = [torch.from_numpy(r[k]).to(dev) for k in range(nm)]
    d_idx = torch.from_numpy(idx.view(np.int64)).to(dev)
    d_cv0 = torch.from_numpy(v0).to(dev)
    d_bm = torch.zeros((n + 31) // 32, dtype=torch.int32, device=dev)
    d_cnt = torch.zeros(2 * len(v0), dtype=torch.int64, device=dev)
    d_hot = torch.from_numpy(hot.view(np.int32)).to(dev)
    d_hp = torch.zeros(1, dtype=torch.int64, device=dev)
    rp = (C.c_void_p * 3)(*[t.data_ptr() for t in d_r], *([0] * (3 - nm)))
    ep = (C.c_float * 3)(*[float(x) for x in eps], *([0.0] * (3 - nm)))
    assert L.ref_snapshot(n, nm, rp, ep, d_idx.data_ptr(), d_cv0.data_ptr(), len(v0), d_bm.data_ptr(),
                          d_cnt.data_ptr(), d_hot.data_ptr() if use_hot else None, d_hp.data_ptr(), None) == 0
    assert np.array_equal(d_bm.cpu().numpy().view(np.uint32), bm)
    assert np.array_equal(d_cnt.cpu().numpy().view(np.uint64), cnt)
    assert int(d_hp.item()) == hp
    # and the reference's k_compact per chunk, as sorted sets
    out = torch.zeros(n, dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    for c in range(len(v0)):
        assert L.ref_compact(int(bounds[c]), int(bounds[c + 1]), d_bm.data_ptr(), out.data_ptr(), count.data_ptr()) == 0
        k = int(count.item())
        assert np.array_equal(np.sort(out[:k].cpu().numpy()), np.sort(eng.chunk_list(c)))
    eng.close()


@pytest.mark.parametrize("nm", [1, 3])
@pytest.mark.parametrize("cap", [1000, 10 ** 9])
def test_hot_compact_and_fill_bitexact_vs_reference(rmat12, nm, cap):
    """The degree cache's integer work on identical inputs: the pending hot
    list of each chunk's hot range (as a sorted set) against the reference's
    k_compact_hot, and the pass-0 fill of the hot lists out of streamed chunks
    against the reference's k_fill_hot and the CSR itself (src/excent.cu:178-182,
    211-220, 617-618, 704-705)."""
    import excent_b200._capi as K
    n, idx, adj = rmat12
    eps, r, v0, e, _, _ = snapshot_case(nm, 29 + nm, n, idx, cap, 0.05)
    deg = np.diff(idx.astype(np.int64))
    # the highest-degree vertices (ties by id), as the degree cache holds them
    hot_ids = np.sort(np.argsort(-deg, kind="stable")[:max(1, n // 20)]).astype(np.int32)
    hot_ids = hot_ids[deg[hot_ids] > 0]
    hot = np.zeros((n + 31) // 32, dtype=np.uint32)
    for v in hot_ids:
        hot[v >> 5] |= np.uint32(1 << int(v & 31))
    hoff = np.zeros(len(hot_ids) + 1, dtype=np.uint64)
    hoff[1:] = np.cumsum(deg[hot_ids])
    meas = X.measures("all" if nm == 3 else "pr", alpha=0.1, lam=10.0, eps_katz=1.0, eps_ev=1.0)
    meas.nm = nm
    for k in range(nm):
        meas.eps[k] = float(eps[k])
    eng = X.Engine(n, len(adj), meas, v0, e)
    eng.upload_offsets(idx)
    K.call("excent_engine_hot_setup", eng.h, len(hot_ids), hot_ids.ctypes.data_as(K.i32p),
           hoff.ctypes.data_as(K.u64p), hot.ctypes.data_as(K.u32p))
    eng.init()
    for k in range(nm):
        eng.write(k, r=r[k])
    L = ref_kernels()
    L.ref_compact_hot.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p]
    L.ref_fill_hot.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p,
                               C.c_void_p]
    dev = torch.device("cuda")
    d_r = [torch.from_numpy(r[k]).to(dev) for k in range(nm)]
    d_hids = torch.from_numpy(hot_ids).to(dev)
    d_hoff = torch.from_numpy(hoff.view(np.int64)).to(dev)
    d_idx = torch.from_numpy(idx.view(np.int64)).to(dev)
    rp = (C.c_void_p * 3)(*[t.data_ptr() for t in d_r], *([0] * (3 - nm)))
    ep = (C.c_float * 3)(*[float(x) for x in eps], *([0.0] * (3 - nm)))
    out = torch.zeros(max(len(hot_ids), 1), dtype=torch.int32, device=dev)
    count = torch.zeros(1, dtype=torch.int32, device=dev)
    bounds = list(v0) + [n]
    ranges = [(int(np.searchsorted(hot_ids, bounds[c])), int(np.searchsorted(hot_ids, bounds[c + 1])))
              for c in range(len(v0))] + [(0, len(hot_ids))]
    pend = np.zeros(n, bool)
    for k in range(nm):
        pend |= np.abs(r[k]) > eps[k]
    mine = np.zeros(max(len(hot_ids), 1), dtype=np.int32)
    for lo, hi in ranges:
        kk = C.c_uint()
        K.call("excent_engine_hot_pending", eng.h, lo, hi, mine.ctypes.data_as(K.i32p), C.byref(kk))
        got = np.sort(mine[:kk.value])
        assert np.array_equal(got, lo + np.nonzero(pend[hot_ids[lo:hi]])[0]), (lo, hi)
        assert L.ref_compact_hot(lo, hi, d_hids.data_ptr(), nm, rp, ep, out.data_ptr(), count.data_ptr()) == 0
        assert np.array_equal(got, np.sort(out[:int(count.item())].cpu().numpy())), (lo, hi)
    # pass-0 fill: stream every chunk through slot 0 with an empty demand table (no push)
    K.call("excent_engine_slots_create", eng.h, int(max(np.diff(np.asarray(e, dtype=np.int64)).max(), 1)),
           int(np.diff(bounds).max()), 0)
    ed = C.POINTER(C.c_int32)()
    K.call("excent_engine_slot_buffers", eng.h, 0, C.byref(ed), None, None)
    zero = np.zeros(2 * len(v0), dtype=np.uint64)
    d_hedges = torch.zeros(max(int(hoff[-1]), 1), dtype=torch.int32, device=dev)
    e_all = [int(x) for x in e]   # nc + 1 edge bounds
    for c in range(len(v0)):
        lo, hi = ranges[c]
        ne = int(e_all[c + 1] - e_all[c])
        K.call("excent_engine_slot_wait", eng.h, 0)
        np.ctypeslib.as_array(ed, shape=(max(ne, 1),))[:ne] = adj[e_all[c]:e_all[c + 1]]
        K.call("excent_engine_push_stream", eng.h, 0, c, zero.ctypes.data_as(K.u64p), 0.5, 0, lo, hi)
        if hi > lo:
            src = torch.from_numpy(np.ascontiguousarray(adj[e_all[c]:e_all[c + 1]])).to(dev)
            assert L.ref_fill_hot(lo, hi, d_hids.data_ptr(), d_hoff.data_ptr(), d_idx.data_ptr(), int(e_all[c]),
                                  src.data_ptr(), d_hedges.data_ptr()) == 0
    eng.sync()
    hedges = np.zeros(max(int(hoff[-1]), 1), dtype=np.int32)
    K.call("excent_engine_hot_edges", eng.h, hedges.ctypes.data_as(K.i32p))
    want = np.concatenate([adj[idx[v]:idx[v + 1]] for v in hot_ids]) if len(hot_ids) else np.zeros(0, np.int32)
    assert np.array_equal(hedges[:len(want)], want)
    assert np.array_equal(d_hedges.cpu().numpy()[:len(want)], want)
    eng.close()


@pytest.mark.parametrize("measure", ["pr", "katz", "ev", "all"])
def test_init_matches_reference_k_init(sample, measure):
    n, idx, adj, env = sample
    meas = meas_for(measure, env)
    eng = make_engine(n, idx, adj, meas)
    eng.init()
    kinds = [int(meas.kind[i]) for i in range(meas.nm)]
    L = ref_kernels()
    dev = torch.device("cuda")
    d_idx = torch.from_numpy(idx.view(np.int64)).to(dev)
    for i, k in enumerate(kinds):
        x = torch.zeros(n, dtype=torch.float32, device=dev)
        r = torch.zeros(n, dtype=torch.float32, device=dev)
        assert L.ref_init(n, d_idx.data_ptr(), x.data_ptr(), r.data_ptr(), k, float(env["BETA"]),
                          float(np.float32(float(env["LAMBDA"])))) == 0
        assert np.array_equal(eng.read(i), x.cpu().numpy())
        assert np.array_equal(eng.read(i, residual=True), r.cpu().numpy())
    eng.close()


def solve_and_compare(n, idx, adj, measure, env=None, cap=None, use_graph=True, list_frac=0.5, **kw):
    meas = meas_for(measure, env, **kw)
    eng = make_engine(n, idx, adj, meas, cap)
    st = eng.solve(list_frac=list_frac, use_graph=use_graph)
    xs = eng.results()
    res = []
    names = ["pr", "katz", "ev"] if measure == "all" else [measure]
    alpha = float(env["ALPHA"]) if env else kw.get("alpha")
    for i, k in enumerate(names):
        # converged: no residual above its threshold
        r = eng.read(i, residual=True)
        assert np.all(np.abs(r) <= np.float32(meas.eps[i])), k
        ref = O.reference_solution(n, idx, adj, k, alpha=alpha)
        res.append(O.compare(k, ref, xs[i]))
    eng.close()
    return st, res


@pytest.mark.parametrize("measure", ["pr", "katz", "ev", "all"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_solve_sample_vs_fp64_oracle(sample, measure, use_graph):
    n, idx, adj, env = sample
    st, res = solve_and_compare(n, idx, adj, measure, env, use_graph=use_graph)
    assert st.passes > 0 and st.pushed > 0
    # CPU port of the reference engine on the same graph: same algorithm, so comparable error
    kinds = ["pr", "katz", "ev"] if measure == "all" else [measure]
    xs, _, _, _ = O.delta_push(n, idx, adj, kinds, alpha=float(env["ALPHA"]), lam=float(env["LAMBDA"]),
                               eps_katz=float(env["EPS_KATZ"]), eps_ev=float(env["EPS_EV"]))
    for i, k in enumerate(kinds):
        ref = O.reference_solution(n, idx, adj, k, alpha=float(env["ALPHA"]))
        port = O.compare(k, ref, xs[i])
        assert res[i]["l1_rel"] <= 1.5 * port["l1_rel"] + 1e-6, (k, res[i], port)
        assert res[i]["top100"] >= 95


def test_solve_rmat16_pagerank(rmat16):
    n, idx, adj = rmat16
    st, res = solve_and_compare(n, idx, adj, "pr")
    assert res[0]["l1_rel"] < 0.04 and res[0]["top1000"] >= 980, res
    assert st.pushed > 5 * len(adj)


def test_solve_multi_chunk_host_driven_push(rmat12):
    """The host-driven pass of the CLI: snapshot, host fetch plan, push of
    every resident chunk in one launch, until nothing is pending."""
    n, idx, adj = rmat12
    meas = X.measures("pr")
    eng = make_engine(n, idx, adj, meas, cap=5000)
    eng.init()
    passes = 0
    while True:
        cnt, hp, rs = eng.snapshot()
        if cnt[0::2].sum() == 0:
            break
        mode = (cnt[0::2] > 0).astype(np.uint8)
        eng.push_cached(mode, cnt, 0.5)
        eng.sync()
        passes += 1
        assert passes < 500
    x = eng.read(0)
    ref = O.reference_solution(n, idx, adj, "pr")
    c = O.compare("pr", ref, x)
    assert c["l1_rel"] < 0.05 and c["top100"] >= 95
    eng.close()


def test_rmat_generator_bitexact_vs_oracle():
    for scale, ef, seed, sym in [(10, 16, 1, True), (12, 8, 3, True), (11, 16, 4, False)]:
        g = X.DeviceGraph(scale, ef, seed, symmetric=sym, weights=not sym)
        idx, adj, w = g.download()
        n, idx_o, adj_o = O.rmat_graph(scale, ef, seed, symmetric=sym)
        assert g.n == n and g.m == len(adj_o)
        assert np.array_equal(idx, idx_o) and np.array_equal(adj[:g.m], adj_o)
        if not sym:
            assert np.array_equal(w[:g.m], O.rmat_weights(g.m, seed))
        g.close()


@pytest.mark.parametrize("scale,ef,seed,part_keys", [(10, 16, 1, 0), (12, 8, 3, 9000), (14, 16, 5, 40000),
                                                     (13, 32, 2, 1 << 40)])
def test_partitioned_egr_writer_bitexact(tmp_path, scale, ef, seed, part_keys):
    """The out-of-core generator writes the same graph as the one-shot device
    generator and the oracle's CPU generator, whatever the partition size."""
    p = str(tmp_path / "g.egr")
    m, parts = X.rmat_write_egr(p, scale, ef, seed, max_part_keys=part_keys)
    if part_keys and part_keys < 1 << 20:
        assert parts > 1
    n, idx, adj = O.read_egr(p)
    n_o, idx_o, adj_o = O.rmat_graph(scale, ef, seed)
    assert n == n_o and m == len(adj_o) == len(adj)
    assert np.array_equal(idx, idx_o) and np.array_equal(adj, adj_o)
    g = X.DeviceGraph(scale, ef, seed)
    i2, a2, _ = g.download()
    assert np.array_equal(i2, idx) and np.array_equal(a2[:g.m], adj)
    g.close()


def test_partitioned_egr_writer_rejects_tiny_partitions(tmp_path):
    with pytest.raises(X.ExcentError, match="source bucket"):
        X.rmat_write_egr(str(tmp_path / "g.egr"), 12, 16, 1, max_part_keys=10)


@pytest.mark.parametrize("sweep", [False, True])
@pytest.mark.parametrize("measure", ["pr", "katz", "ev", "all"])
def test_error_no_looser_than_reference_engine(sample, measure, sweep):
    """The reference engine's own result dumps on the sample (built from its
    source and run on a B200, committed under tests/golden/) against the
    reference's FP64 oracle vectors: our errors must not be looser.

    Both engines add FP32 residuals with atomics in a run-dependent order, so
    one solve is one draw: the reference binary's Katz L1 error moved by 9 %
    between two runs on R-MAT scale 16, ours moves by a few percent. The median
    of five of our solves is held to the reference's single run with 5 % on
    the L1 and 10 % on the max error."""
    from conftest import GOLDEN
    n, idx, adj, env = sample
    names = ["pr", "katz", "ev"] if measure == "all" else [measure]
    meas = meas_for(measure, env)
    eng = make_engine(n, idx, adj, meas)
    eng.set_chunk_sweep(sweep)
    eng.set_hub_order("table" if sweep else "first")
    runs = {k: [] for k in names}
    for _ in range(5):
        eng.solve()
        for i, k in enumerate(names):
            ref = np.fromfile(os.path.join(GOLDEN, f"sample_ref_{k}.f64"))
            runs[k].append(O.compare(k, ref, eng.read(i)))
    for k in names:
        ref = np.fromfile(os.path.join(GOLDEN, f"sample_ref_{k}.f64"))
        theirs = O.compare(k, ref, np.fromfile(os.path.join(GOLDEN, f"sample_excent_{measure}_{k}.f32"),
                                               dtype=np.float32))
        med = {q: float(np.median([r[q] for r in runs[k]])) for q in ("l1_rel", "max_abs", "top100", "top1000")}
        print(measure, k, "ours (median of 5)", med, "reference engine", theirs)
        assert med["l1_rel"] <= theirs["l1_rel"] * 1.05, (k, med, theirs)
        assert med["max_abs"] <= theirs["max_abs"] * 1.10, (k, med, theirs)
        # on 2000 vertices the 1000th value sits in a dense band (94 vertices within 1 % of it)
        # while eps 0.01 leaves per-vertex errors of about 3 %, so membership of the top half
        # flips with the FP32 summation order: an allowance of 1 % of the set
        assert med["top1000"] >= theirs["top1000"] - 10, (k, med, theirs)
        assert med["top100"] >= theirs["top100"] - 1, (k, med, theirs)
    eng.close()


def test_ev_normalisation_step_keeps_the_unit_eigenvector(rmat16):
    """EV with the FP64 normalisation step converges to the same unit vector
    (checked against the FP64 oracle) at a tight eps."""
    n, idx, adj = rmat16
    dev = torch.device("cuda")
    d_idx = torch.from_numpy(idx.view(np.int64)).to(dev)
    d_adj = torch.from_numpy(adj).to(dev)
    v1 = torch.empty(n, dtype=torch.float32, device=dev)
    par = X.params_fp64(n, d_idx.data_ptr(), d_adj.data_ptr(), v1_out=v1)
    ref = O.reference_solution(n, idx, adj, "ev")
    assert np.abs(O.unit(v1.cpu().numpy()) - O.unit(ref)).max() < 1e-5
    for proj in (False, True):
        meas = X.measures("ev", lam=par["lambda"], eps_ev=1e-6)
        eng = make_engine(n, idx, adj, meas)
        if proj:
            eng.ev_project(v1)
        st = eng.solve(max_passes=5000)
        c = O.compare("ev", ref, eng.read(0))
        print("projection", proj, "passes", st.passes, c)
        assert st.passes < 5000
        assert c["l1_rel"] < 2e-3 and c["top1000"] >= 990
        eng.close()


@pytest.mark.parametrize("measure", ["pr", "all"])
@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("order", ["table", "first"])
def test_chunk_sweep_matches_one_launch(rmat16, measure, use_graph, order):
    """Chunk by chunk (one launch per chunk, in chunk order; with a CUDA graph,
    chunks with nothing to push are skipped by IF nodes) reaches the fixed
    point of the one-launch pass, on a graph cut into several chunks."""
    n, idx, adj = rmat16
    par = O.params(n, idx, adj)
    kw = dict(alpha=0.9 / par["_lambda"], lam=par["_lambda"], eps_katz=1e-5, eps_ev=1e-5) if measure == "all" else {}
    names = ["pr", "katz", "ev"] if measure == "all" else ["pr"]
    res = {}
    for sweep in (False, True):
        meas = X.measures(measure, **kw)
        eng = make_engine(n, idx, adj, meas, cap=len(adj) // 7 + 1)
        assert eng.nc >= 7
        eng.set_hub_order(order)
        eng.set_chunk_sweep(sweep)
        l0 = eng.launches()
        st = eng.solve(use_graph=use_graph)
        res[(sweep, "launches")] = eng.launches() - l0
        for i, k in enumerate(names):
            r = eng.read(i, residual=True)
            assert np.all(np.abs(r) <= np.float32(meas.eps[i]))
            ref = O.reference_solution(n, idx, adj, k, alpha=kw.get("alpha"))
            res[(sweep, k)] = O.compare(k, ref, eng.read(i))
        res[(sweep, "pushed")] = st.pushed
        eng.close()
    print(res)
    for k in names:
        assert res[(True, k)]["l1_rel"] <= 1.25 * res[(False, k)]["l1_rel"] + 3e-5, (k, res)
        assert res[(True, k)]["top1000"] >= res[(False, k)]["top1000"] - 5
    assert res[(True, "launches")] > res[(False, "launches")]


@pytest.mark.parametrize("measure", ["pr", "all"])
def test_engine_autotune_keeps_the_fastest_and_solves(rmat16, measure):
    """excent_engine_autotune times every candidate (swept with three demand thresholds and
    three slot counts, or high-degree lists first), leaves the engine on the fastest, and the
    solve with those settings reaches every threshold."""
    n, idx, adj = rmat16
    par = O.params(n, idx, adj)
    kw = dict(alpha=0.9 / par["_lambda"], lam=par["_lambda"], eps_katz=1e-5, eps_ev=1e-5) if measure == "all" else {}
    meas = X.measures(measure, **kw)
    eng = make_engine(n, idx, adj, meas, cap=len(adj) // 7 + 1)
    best, tried = eng.autotune()
    assert len(tried) == 8
    assert best["ms"] == min(t["ms"] for t in tried) and all(t["ms"] > 0 for t in tried)
    assert {t["sweep_demand"] for t in tried if t["chunk_sweep"]} == {0.25, 0.5, 1.0}
    eng.solve()
    for i in range(meas.nm):
        assert np.all(np.abs(eng.read(i, residual=True)) <= np.float32(meas.eps[i]))
    eng.close()


@pytest.mark.parametrize("measure", ["pr", "all"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_sweep_demand_threshold(rmat16, measure, use_graph):
    """A sweeping engine with a demand threshold sweeps only the passes whose
    pending entries reach frac * m and pushes the others in one launch: the
    same fixed point, and a launch count between the one-launch solve's and the
    every-pass sweep's. A threshold above any demand launches like no sweep."""
    n, idx, adj = rmat16
    m = len(adj)
    par = O.params(n, idx, adj)
    kw = dict(alpha=0.9 / par["_lambda"], lam=par["_lambda"], eps_katz=1e-5, eps_ev=1e-5) if measure == "all" else {}
    names = ["pr", "katz", "ev"] if measure == "all" else ["pr"]
    res = {}
    for tag, sweep, frac in [("one", False, 0.0), ("all", True, 0.0), ("some", True, 0.3), ("none", True, 1e6)]:
        meas = X.measures(measure, **kw)
        eng = make_engine(n, idx, adj, meas, cap=m // 7 + 1)
        eng.set_hub_order("table")
        eng.set_chunk_sweep(sweep)
        eng.set_sweep_demand(frac)
        l0 = eng.launches()
        st = eng.solve(use_graph=use_graph)
        res[(tag, "launches")] = eng.launches() - l0
        res[(tag, "per_pass")] = res[(tag, "launches")] / (st.passes + 1)
        _, plog = eng.stats(with_log=True)
        res[(tag, "demand")] = [int(p.demand) for p in plog]
        for i, k in enumerate(names):
            r = eng.read(i, residual=True)
            assert np.all(np.abs(r) <= np.float32(meas.eps[i])), (tag, k)
            ref = O.reference_solution(n, idx, adj, k, alpha=kw.get("alpha"))
            res[(tag, k)] = O.compare(k, ref, eng.read(i))
        eng.close()
    print(res)
    d = res[("some", "demand")]
    assert max(d) >= 0.3 * m > min(d)   # both kinds of pass occur
    for k in names:
        for tag in ("some", "none"):
            assert res[(tag, k)]["l1_rel"] <= 1.25 * res[("one", k)]["l1_rel"] + 3e-5, (tag, k, res)
    # launches per pass (the orders differ, so do the pass counts): a threshold above every
    # pass's demand launches like one launch per pass, a threshold inside the range in between
    assert abs(res[("none", "per_pass")] - res[("one", "per_pass")]) <= 1.0, res
    assert res[("none", "per_pass")] <= res[("some", "per_pass")] + 0.5 < res[("all", "per_pass")], res


@pytest.mark.parametrize("measure", ["pr", "all"])
@pytest.mark.parametrize("k", [1, 64, 2048])
@pytest.mark.parametrize("sweep", [False, True])
def test_hub_targets_match_plain_push(rmat16, measure, k, sweep):
    """Shared-memory aggregation of the top-k targets reaches the same fixed
    point, leaves the cache decodable (set to 0 restores the plain ids), in one
    launch per pass or chunk by chunk."""
    n, idx, adj = rmat16
    par = O.params(n, idx, adj)
    kw = dict(alpha=0.9 / par["_lambda"], lam=par["_lambda"], eps_katz=1e-5, eps_ev=1e-5) if measure == "all" else {}
    names = ["pr", "katz", "ev"] if measure == "all" else ["pr"]
    res = {}
    for hk in (0, k):
        meas = X.measures(measure, **kw)
        eng = make_engine(n, idx, adj, meas)
        eng.set_chunk_sweep(sweep)
        eng.set_hub_targets(hk)
        eng.solve()
        for i, name in enumerate(names):
            r = eng.read(i, residual=True)
            assert np.all(np.abs(r) <= np.float32(meas.eps[i]))
            ref = O.reference_solution(n, idx, adj, name, alpha=kw.get("alpha"))
            res[(hk, name)] = O.compare(name, ref, eng.read(i))
        if hk:   # back to plain ids: a second solve from scratch still matches
            eng.set_hub_targets(0)
            eng.solve()
            c = O.compare(names[0], O.reference_solution(n, idx, adj, names[0], alpha=kw.get("alpha")), eng.read(0))
            assert c["l1_rel"] <= 1.25 * res[(0, names[0])]["l1_rel"] + 1e-5
        eng.close()
    for name in names:
        assert res[(k, name)]["l1_rel"] <= 1.25 * res[(0, name)]["l1_rel"] + 1e-5, (name, res)
        assert res[(k, name)]["top100"] >= 95


@pytest.mark.parametrize("measure", ["pr", "all"])
@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("sweep", [False, True])
def test_high_degree_first_order(rmat16, measure, use_graph, sweep):
    """Pushing the high-degree lists first in each pass reaches the same fixed
    point, also with hub targets and with the cache reloaded from host memory
    (the reload re-encodes the hub-target slots)."""
    n, idx, adj = rmat16
    par = O.params(n, idx, adj)
    kw = dict(alpha=0.9 / par["_lambda"], lam=par["_lambda"], eps_katz=1e-5, eps_ev=1e-5) if measure == "all" else {}
    names = ["pr", "katz", "ev"] if measure == "all" else ["pr"]
    assert int((np.diff(idx) > 256).sum()) > 0
    res = {}
    for mode in ("plain", "first", "last", "first+targets"):
        meas = X.measures(measure, **kw)
        eng = make_engine(n, idx, adj, meas)
        eng.set_chunk_sweep(sweep)
        eng.set_hub_order({"plain": "table", "first": "first", "last": "last", "first+targets": "first"}[mode])
        if mode == "first+targets":
            eng.set_hub_targets(512)
            eng.load_cache(0, len(adj), np.ascontiguousarray(adj, dtype=np.int32))
        st = eng.solve(use_graph=use_graph)
        for i, name in enumerate(names):
            r = eng.read(i, residual=True)
            assert np.all(np.abs(r) <= np.float32(meas.eps[i]))
            ref = O.reference_solution(n, idx, adj, name, alpha=kw.get("alpha"))
            res[(mode, name)] = O.compare(name, ref, eng.read(i))
        res[(mode, "pushed")] = st.pushed
        eng.close()
    print(res)
    for mode in ("first", "last", "first+targets"):
        for name in names:
            # eps-level slack: the eps of Katz and EV here is 1e-5
            assert res[(mode, name)]["l1_rel"] <= 1.25 * res[("plain", name)]["l1_rel"] + 3e-5, (mode, name, res)


@pytest.mark.parametrize("measure", ["pr", "all"])
@pytest.mark.parametrize("use_graph", [True, False])
@pytest.mark.parametrize("resident", [0, 2])
def test_host_cache_zero_copy_solve(rmat16, measure, use_graph, resident):
    """Chunks past the HBM cache read in place from pinned host memory: the
    device solve reaches the fixed point of the fully cached solve, and the
    entries it pushed from host memory are counted."""
    n, idx, adj = rmat16
    par = O.params(n, idx, adj)
    kw = dict(alpha=0.9 / par["_lambda"], lam=par["_lambda"], eps_katz=1e-5, eps_ev=1e-5) if measure == "all" else {}
    names = ["pr", "katz", "ev"] if measure == "all" else ["pr"]
    m = len(adj)
    cap = m // 5 + 1
    v0, e = chunks_for(idx, cap)
    assert len(v0) >= 4
    res = {}
    for mode in ("device", "host"):
        meas = X.measures(measure, **kw)
        eng = X.Engine(n, m, meas, v0, e)
        eng.set_hub_order("first")    # the same pass order in both modes: this test is about where
        eng.set_chunk_sweep(False)    # the lists are read from
        eng.upload_offsets(idx)
        if mode == "device":
            eng.reserve_cache(m)
            eng.load_cache(0, m, np.ascontiguousarray(adj, dtype=np.int32))
        else:
            ce = int(e[resident])
            eng.reserve_cache(ce)
            if ce:
                eng.load_cache(0, ce, np.ascontiguousarray(adj[:ce], dtype=np.int32))
            buf, first = eng.host_cache()
            assert first == ce and len(buf) == m - ce
            buf[:] = adj[ce:]
        st = eng.solve(use_graph=use_graph)
        for i, name in enumerate(names):
            r = eng.read(i, residual=True)
            assert np.all(np.abs(r) <= np.float32(meas.eps[i]))
            ref = O.reference_solution(n, idx, adj, name, alpha=kw.get("alpha"))
            res[(mode, name)] = O.compare(name, ref, eng.read(i))
        hp = eng.host_pushed()
        if mode == "host":
            assert 0 < hp <= st.pushed
        else:
            assert hp == 0
        eng.close()
    for name in names:
        assert res[("host", name)]["l1_rel"] <= 1.25 * res[("device", name)]["l1_rel"] + 1e-5, (name, res)
