"""Host runtime parity (no GPU): EGR reader, planner decisions, gather list,
page-run dedup and the command-line surface, against the oracle and against
the reference's own code (include/StaticGraph.h through oracle/_ref/libsg_ref.so,
and the reference binary oracle/_ref/excent, whose option parse and `graph:`
line run before it touches the GPU)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN

import excent_b200 as X  # noqa: E402
import excent_b200._capi as K  # noqa: E402

SAMPLE = os.path.join(GOLDEN, "sample.egr")


def egr_open(path, threads=16, in_ram=0):
    h = C.c_void_p()
    K.call("excent_egr_open", path.encode(), threads, in_ram, C.byref(h))
    return h


def egr_info(h):
    n, m, w = C.c_int(), C.c_uint64(), C.c_int()
    K.call("excent_egr_info", h, C.byref(n), C.byref(m), C.byref(w))
    return n.value, m.value, bool(w.value)


@pytest.fixture(scope="module")
def rmat14_files(tmp_path_factory):
    d = tmp_path_factory.mktemp("egr")
    n, idx, adj = O.rmat_graph(14, 16, 3)
    wide = str(d / "w.egr")
    narrow = str(d / "n.egr")
    O.write_egr(wide, idx, adj, wide=True)
    O.write_egr(narrow, idx, adj, wide=False)
    return n, idx, adj, wide, narrow, d


@pytest.mark.parametrize("kind", ["wide", "narrow"])
@pytest.mark.parametrize("in_ram", [0, 1])
def test_egr_reader_roundtrip(rmat14_files, kind, in_ram):
    n, idx, adj, wide, narrow, _ = rmat14_files
    h = egr_open(wide if kind == "wide" else narrow, 16, in_ram)
    assert egr_info(h) == (n, len(adj), kind == "wide")
    off = np.zeros(n + 1, dtype=np.uint64)
    K.call("excent_egr_read_offsets", h, 0, n + 1, off.ctypes.data)
    assert np.array_equal(off, idx)
    for e0, e1 in [(0, len(adj)), (5, 5), (17, len(adj) // 3)]:
        buf = np.zeros(max(e1 - e0, 1), dtype=np.int32)
        K.call("excent_egr_read_edges", h, e0, e1, buf.ctypes.data)
        assert np.array_equal(buf[:e1 - e0], adj[e0:e1])
    K.call("excent_egr_close", h)


def test_egr_reader_errors(rmat14_files):
    n, idx, adj, wide, narrow, d = rmat14_files
    raw = open(wide, "rb").read()
    bad = {
        "trunc.egr": raw[:-4],
        "short.egr": raw[:6],
        "n0.egr": np.array([0, 0], dtype="<i4").tobytes(),
        "neg.egr": np.array([5, -7], dtype="<i4").tobytes() + b"\0" * 64,
    }
    dec = bytearray(raw)
    # offsets decreasing at vertex 3: idx[4] := idx[3] - 1 (wide header is 16 bytes)
    v = int(idx[3])
    dec[16 + 8 * 4:16 + 8 * 5] = np.array([max(v - 1, 0)], dtype="<u8").tobytes()
    if v > 0:
        bad["dec.egr"] = bytes(dec)
    for name, data in bad.items():
        p = str(d / name)
        open(p, "wb").write(data)
        h = C.c_void_p()
        rc = K.load().excent_egr_open(p.encode(), 4, 0, C.byref(h))
        assert rc == 3, (name, rc)   # EXCENT_ERR_IO
        assert K.load().excent_last_error()
    h = C.c_void_p()
    assert K.load().excent_egr_open(str(d / "missing.egr").encode(), 4, 0, C.byref(h)) == 3


def _ref_sg():
    p = os.path.join(O.REF_DIR, "libsg_ref.so")
    if not os.path.exists(p):
        pytest.skip("reference StaticGraph harness not built")
    L = C.CDLL(p)
    L.ref_sg_open.restype = C.c_void_p
    L.ref_sg_open.argtypes = [C.c_char_p, C.c_int, C.c_int]
    L.ref_sg_close.argtypes = [C.c_void_p]
    L.ref_sg_plan_chunks.restype = C.c_int
    L.ref_sg_plan_chunks.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p, C.c_int]
    L.ref_sg_prefetch.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    return L


@pytest.mark.parametrize("cap", [1, 7, 999, 4 * 10 ** 4, 10 ** 9])
def test_plan_chunks_vs_reference(rmat14_files, cap):
    n, idx, adj, wide, narrow, _ = rmat14_files
    L = _ref_sg()
    h = L.ref_sg_open(wide.encode(), 4, 0)
    ref = np.zeros(4 * (n + 1), dtype=np.uint64)
    nc_r = L.ref_sg_plan_chunks(h, cap, ref.ctypes.data, n + 1)
    L.ref_sg_close(h)
    nc = C.c_int()
    K.call("excent_plan_chunks", n, idx.ctypes.data, cap, C.byref(nc), None, 0)
    out = np.zeros(4 * nc.value, dtype=np.uint64)
    K.call("excent_plan_chunks", n, idx.ctypes.data, cap, C.byref(nc), out.ctypes.data, nc.value)
    assert nc.value == nc_r and np.array_equal(out, ref[:4 * nc_r])


@pytest.mark.parametrize("m", [0, 10, 3999999, 4 * 10 ** 6 + 1, 268435456, 8 * 10 ** 9])
@pytest.mark.parametrize("cm,tc,mc", [(0, 16, 4), (2.5, 16, 4), (0, 7, 1), (0, 1000, 0.5)])
def test_chunk_cap_vs_oracle(m, cm, tc, mc):
    assert K.load().excent_chunk_cap(m, cm, tc, mc) == O.chunk_cap(m, cm, tc, mc)


@pytest.mark.parametrize("k", [0, 1, 7, 1023, 1024, 4100, 16383, 16384, 40000])
def test_prefetch_pages_and_runs_vs_reference(rmat14_files, k):
    n, idx, adj, wide, narrow, _ = rmat14_files
    rng = np.random.default_rng(k)
    vids = np.sort(rng.choice(n, min(k, n), replace=False)).astype(np.int32)
    k = len(vids)
    h = egr_open(wide, 16, 0)
    pg, rn = C.c_uint64(), C.c_uint64()
    K.call("excent_egr_prefetch", h, vids.ctypes.data, k, C.byref(pg), C.byref(rn))
    K.call("excent_egr_close", h)
    assert (pg.value, rn.value) == O.prefetch_runs(vids, idx, 16 + 8 * (n + 1), os.sysconf("SC_PAGESIZE"), 16)
    L = _ref_sg()
    hr = L.ref_sg_open(wide.encode(), 16, 0)
    p2, r2 = C.c_uint64(), C.c_uint64()
    L.ref_sg_prefetch(hr, vids.ctypes.data, k, C.byref(p2), C.byref(r2))
    L.ref_sg_close(hr)
    assert (pg.value, rn.value) == (p2.value, r2.value)


def test_fetch_plan_vs_oracle():
    rng = np.random.default_rng(3)
    for trial in range(300):
        nc = int(rng.integers(1, 40))
        edges = rng.integers(0, 10 ** 6, nc).astype(np.uint64)
        cnt = np.zeros(2 * nc, dtype=np.uint64)
        cnt[0::2] = rng.integers(0, 3, nc) * rng.integers(0, 1000, nc)
        cnt[1::2] = (rng.random(nc) * edges * 1.2).astype(np.uint64)
        resident = (rng.random(nc) < 0.4).astype(np.uint8)
        loaded = (resident & (rng.random(nc) < 0.5)).astype(np.uint8)
        tau = float(rng.choice([0.0, 0.005, 0.3, 1.0, 2.0]))
        hot = int(rng.integers(0, 2))
        p = int(rng.integers(0, 3))
        hlo = rng.integers(0, 50, nc).astype(np.int32)
        hhi = (hlo + rng.integers(0, 2, nc)).astype(np.int32)
        mode = np.zeros(nc, dtype=np.uint8)
        pv, dm, nb = C.c_uint64(), C.c_uint64(), C.c_int()
        K.call("excent_fetch_plan", nc, edges.ctypes.data, cnt.ctypes.data, resident.ctypes.data, loaded.ctypes.data,
               tau, hot, p, hlo.ctypes.data, hhi.ctypes.data, mode.ctypes.data, C.byref(pv), C.byref(dm), C.byref(nb))
        mo, pvo, dmo, nbo = O.fetch_plan(cnt, resident, loaded, tau, edges, hot, p, hlo, hhi)
        assert np.array_equal(mode, mo) and (pv.value, dm.value, bool(nb.value)) == (pvo, dmo, nbo), trial


def test_gather_list_vs_oracle(rmat12):
    n, idx, adj = rmat12
    rng = np.random.default_rng(9)
    for dens in (0.0, 0.01, 0.3, 1.0):
        bits = rng.random(n) < dens
        bm = np.zeros((n + 31) // 32, dtype=np.uint64)
        np.add.at(bm, np.arange(n) >> 5, bits.astype(np.uint64) << (np.arange(n) & 31).astype(np.uint64))
        bm = bm.astype(np.uint32)
        for v0, v1 in [(0, n), (5, 37), (31, 33), (1000, 1000), (n - 40, n)]:
            vids = np.zeros(max(v1 - v0, 1), dtype=np.int32)
            off = np.zeros(max(v1 - v0, 1) + 1, dtype=np.uint64)
            k = C.c_int()
            K.call("excent_gather_list", v0, v1, bm.ctypes.data, idx.ctypes.data, vids.ctypes.data, off.ctypes.data,
                   C.byref(k))
            vo, oo = O.gather_list(v0, v1, bm, idx)
            assert np.array_equal(vids[:k.value], vo) and np.array_equal(off[:k.value + 1], oo)


def test_cache_sizing_vs_oracle():
    rng = np.random.default_rng(4)
    for _ in range(200):
        nc = int(rng.integers(1, 30))
        ce = rng.integers(0, 10 ** 7, nc).astype(np.uint64)
        free = int(rng.integers(0, 4 * 10 ** 8))
        res = int(rng.choice([0, 256 << 20, 10 ** 9]))
        r = C.c_int()
        K.call("excent_cache_chunks", nc, ce.ctypes.data, free, res, C.byref(r))
        assert r.value == O.cache_chunks(ce, free, res)


@pytest.mark.parametrize("budget", [0, 1000, 10 ** 5, 10 ** 6, 3 * 10 ** 6, 10 ** 12])
def test_hot_select_vs_oracle(rmat14_files, budget):
    n, idx, adj, *_ = rmat14_files
    nh = C.c_int()
    ids = np.zeros(n, dtype=np.int32)
    hoff = np.zeros(n + 1, dtype=np.uint64)
    bits = np.zeros((n + 31) // 32, dtype=np.uint32)
    T = C.c_uint64()
    K.call("excent_hot_select", n, idx.ctypes.data, budget, None, C.byref(nh), ids.ctypes.data, hoff.ctypes.data,
           bits.ctypes.data, C.byref(T))
    ido, To, Eo = O.hot_select(idx, budget)
    assert np.array_equal(ids[:nh.value], ido) and T.value == To and hoff[nh.value] == Eo
    deg = np.diff(idx.astype(np.int64))
    assert np.array_equal(np.diff(hoff[:nh.value + 1].astype(np.int64)), deg[ido])
    cost = (deg[ido] * 4 + 16).sum()
    assert cost <= budget
    v = np.arange(n)
    inbits = ((bits[v >> 5] >> (v & 31)) & 1).astype(bool)
    assert np.array_equal(np.nonzero(inbits)[0], ido)


def test_hot_select_big_degrees_and_ties_vs_oracle():
    """Degree values of 2^20 and more are admitted whole or not at all, smaller
    ones partly (the first in id order); synthetic offsets with repeated big and
    small degrees, budgets at and around every admission boundary."""
    rng = np.random.default_rng(9)
    n = 3000
    deg = rng.integers(0, 40, n).astype(np.uint64)
    deg[rng.choice(n, 30, replace=False)] = rng.choice([300, 301, 5000], 30)
    big = rng.choice(n, 9, replace=False)
    deg[big] = np.array([1 << 20, 1 << 20, (1 << 20) + 7, 3 << 20, 3 << 20, 3 << 20, (1 << 21) - 1, 1 << 21, 5 << 21],
                        dtype=np.uint64)
    idx = np.zeros(n + 1, dtype=np.uint64)
    idx[1:] = np.cumsum(deg)
    cost = np.sort(deg[deg > 0] * 4 + 16)[::-1].astype(np.int64)
    marks = np.cumsum(cost)
    budgets = {0, 15, 16, 17, int(marks[-1]), int(marks[-1]) + 1, 10 ** 13}
    for i in list(range(0, 12)) + list(range(12, len(marks), 97)):
        budgets |= {int(marks[i]) - 1, int(marks[i]), int(marks[i]) + 1, int(marks[i]) + 8 * 4 + 16}
    for budget in sorted(budgets):
        nh = C.c_int()
        ids = np.zeros(n, dtype=np.int32)
        hoff = np.zeros(n + 1, dtype=np.uint64)
        T = C.c_uint64()
        K.call("excent_hot_select", n, idx.ctypes.data, budget, None, C.byref(nh), ids.ctypes.data,
               hoff.ctypes.data, None, C.byref(T))
        ido, To, Eo = O.hot_select(idx, budget)
        assert np.array_equal(ids[:nh.value], ido), budget
        assert T.value == To and hoff[nh.value] == Eo, (budget, T.value, To)


def test_hot_select_by_score(rmat14_files):
    """--hot-rank: uint16 scores (the --trace-pending format), boundary score partly taken."""
    n, idx, adj, *_ = rmat14_files
    rng = np.random.default_rng(2)
    score = rng.integers(0, 6, n).astype(np.uint16)
    deg = np.diff(idx.astype(np.int64))
    for budget in (0, 10 ** 4, 2 * 10 ** 5, 10 ** 9):
        nh = C.c_int()
        ids = np.zeros(n, dtype=np.int32)
        K.call("excent_hot_select", n, idx.ctypes.data, budget, score.ctypes.data, C.byref(nh), ids.ctypes.data,
               None, None, None)
        sel = ids[:nh.value]
        # restatement of src/excent.cu:459-490
        cost = deg * 4 + 16
        cs = np.zeros(65536)
        np.add.at(cs, score[(deg > 0) & (score > 0)], cost[(deg > 0) & (score > 0)])
        u, S, left = 0.0, 0, 0
        for s in range(65535, 0, -1):
            if u + cs[s] <= budget:
                u += cs[s]
                continue
            S, left = s, budget - int(u)
            break
        want = []
        for v in range(n):
            if deg[v] == 0 or score[v] == 0 or score[v] < S:
                continue
            if score[v] == S:
                if cost[v] > left:
                    continue
                left -= cost[v]
            want.append(v)
        assert np.array_equal(sel, np.array(want, dtype=np.int32)), budget


def test_tau_vs_oracle():
    rng = np.random.default_rng(1)
    for _ in range(500):
        ts = float(rng.random() * 2)
        tg = np.sort(rng.random(3) * 3).astype(np.float64)
        f = np.sort(rng.random(3)).astype(np.float64)
        assert K.load().excent_tau(ts, tg.ctypes.data, f.ctypes.data) == O.tau(ts, tg, f)


# ------------------------------------------------------------------ command line

CLI = K.CLI_PATH
REF_CLI = os.path.join(O.REF_DIR, "excent")

ARG_CASES = [
    [],
    [SAMPLE, "--measure", "katz"],
    [SAMPLE, "--measure", "ev", "--lambda", "3"],
    [SAMPLE, "--measure", "bogus"],
    [SAMPLE, "--measure", "pr", "--bogus"],
    [SAMPLE, "--measure", "pr", "--dedup", "maybe"],
    [SAMPLE, "--measure", "pr", "--cache", "everything"],
    [SAMPLE, "--measure", "pr", "--eps-pr"],
]


@pytest.mark.parametrize("args", ARG_CASES)
def test_cli_argument_errors_match_reference(args):
    ours = subprocess.run([CLI, *args], capture_output=True, text=True)
    assert ours.returncode == 1
    if not os.path.exists(REF_CLI):
        pytest.skip("reference binary not built")
    ref = subprocess.run([REF_CLI, *args], capture_output=True, text=True)
    assert ref.returncode == 1
    norm = lambda s: s.replace(CLI, "X").replace(REF_CLI, "X")  # noqa: E731
    assert norm(ours.stderr) == norm(ref.stderr)


@pytest.mark.parametrize("extra", [[], ["--chunk-medges", "0.001"], ["--target-chunks", "5", "--min-chunk-medges", "0"],
                                   ["--chunk-medges", "0.0000001"]])
def test_cli_graph_line_matches_reference(extra, rmat14_files):
    """The chunk table line printed before any GPU work (src/excent.cu:332)."""
    if not os.path.exists(REF_CLI):
        pytest.skip("reference binary not built")
    for path in (SAMPLE, rmat14_files[3], rmat14_files[4]):
        args = [path, "--measure", "pr", *extra]
        ours = subprocess.run([CLI, *args], capture_output=True, text=True)
        ref = subprocess.run([REF_CLI, *args], capture_output=True, text=True)
        g1 = re.sub(r"open [0-9.]+s", "", ours.stdout.splitlines()[0])
        g2 = re.sub(r"open [0-9.]+s", "", ref.stdout.splitlines()[0])
        assert g1 == g2


@pytest.mark.parametrize("args,msg", [
    (["--ev-init", "fp32"], "--ev-init must be fp64 or reference"),
    (["--chunk-sweep", "maybe"], "--chunk-sweep must be on, off or auto"),
    (["--sweep-demand", "-1"], "--sweep-demand must be a fraction >= 0"),
    (["--host-cache", "mapped"], "--host-cache must be pinned or off"),
])
def test_cli_own_option_errors(args, msg):
    """This CLI's own options (beside the reference's) reject bad values before any work."""
    r = subprocess.run([CLI, SAMPLE, "--measure", "pr", *args], capture_output=True, text=True)
    assert r.returncode == 1 and msg in r.stderr, r.stderr


def test_cli_bad_file_is_an_error(tmp_path):
    p = tmp_path / "t.egr"
    p.write_bytes(np.array([100, 50], dtype="<i4").tobytes())
    r = subprocess.run([CLI, str(p), "--measure", "pr"], capture_output=True, text=True)
    assert r.returncode == 1 and "truncated" in r.stderr


PARAMS = os.path.join(os.path.dirname(K.CLI_PATH), "excent_params")
REF_PARAMS = os.path.join(O.REF_DIR, "excent_params")


def test_params_tool_usage_matches_reference():
    ours = subprocess.run([PARAMS], capture_output=True, text=True)
    assert ours.returncode == 1 and "usage:" in ours.stderr
    if not os.path.exists(REF_PARAMS):
        pytest.skip("reference tool not built")
    ref = subprocess.run([REF_PARAMS], capture_output=True, text=True)
    assert ref.returncode == 1
    assert ours.stderr.replace(PARAMS, "X") == ref.stderr.replace(REF_PARAMS, "X")


def test_params_tool_symmetry_check_before_any_gpu_work(tmp_path):
    """An asymmetric graph is rejected by the sampled symmetry check, with the
    reference tool's message, before the device is touched."""
    n, idx, adj = O.rmat_graph(10, 8, 3, symmetric=False)
    p = str(tmp_path / "d.egr")
    O.write_egr(p, idx, adj)
    ours = subprocess.run([PARAMS, p, str(tmp_path / "d.env")], capture_output=True, text=True)
    assert ours.returncode == 1 and "graph is not symmetric" in ours.stderr
    assert ours.stdout.startswith(f"graph: n={n} m={len(adj)}")


REFTOOL = os.path.join(os.path.dirname(K.CLI_PATH), "excent_reference")
REF_REFTOOL = os.path.join(O.REF_DIR, "centrality_reference")


@pytest.mark.parametrize("mode", ["--compare", "--rank"])
@pytest.mark.parametrize("measure,dump", [("pr", "sample_excent_pr_pr.f32"), ("katz", "sample_excent_katz_katz.f32"),
                                          ("ev", "sample_excent_ev_ev.f32"), ("ev", "sample_excent_all_ev.f32")])
def test_reference_tool_comparison_matches_reference(mode, measure, dump):
    """--compare / --rank of the reference engine's golden dumps against the
    golden FP64 solution: the same line as the reference's own tool (CPU only)."""
    args = [mode, measure, os.path.join(GOLDEN, f"sample_ref_{measure}.f64"), os.path.join(GOLDEN, dump)]
    ours = subprocess.run([REFTOOL, *args], capture_output=True, text=True)
    assert ours.returncode == 0, ours.stderr
    assert ours.stdout.startswith(f"{measure}:")
    if not os.path.exists(REF_REFTOOL):
        pytest.skip("reference tool not built")
    ref = subprocess.run([REF_REFTOOL, *args], capture_output=True, text=True)
    assert ref.returncode == 0
    assert ours.stdout == ref.stdout


def test_reference_tool_usage_matches_reference():
    ours = subprocess.run([REFTOOL], capture_output=True, text=True)
    assert ours.returncode == 1
    if not os.path.exists(REF_REFTOOL):
        pytest.skip("reference tool not built")
    ref = subprocess.run([REF_REFTOOL], capture_output=True, text=True)
    assert ours.stderr.replace(REFTOOL, "X") == ref.stderr.replace(REF_REFTOOL, "X")
