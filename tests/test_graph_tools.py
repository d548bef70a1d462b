"""EGR file tools (no GPU): the .mtx converter against the reference converter's
own outputs (tools/efficient_converter.py, run by tests/golden/make_golden.py on
the sample's .mtx and on an edge-case file), its --sort / --dedup /
--no-self-loops / --symmetric modes against a numpy restatement, the info line
against the reference's egr_info, and the page-cache tool."""
import ctypes as C
import hashlib
import json
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN

import excent_b200._capi as K  # noqa: E402

BIN = os.path.dirname(K.CLI_PATH)
META = json.load(open(os.path.join(GOLDEN, "golden.json")))


def sha(p):
    return hashlib.sha256(open(p, "rb").read()).hexdigest()


def convert(src, dst, flags=0):
    st = np.zeros(5, dtype=np.uint64)
    K.call("excent_mtx_to_egr", src.encode(), dst.encode(), flags, st.ctypes.data_as(K.u64p))
    return st


def parse_mtx(text):
    """(n, [(u, v)]) the way the reference converter reads a file: n = max(rows, cols) of the
    first non-comment line, then every line with two or more fields, 1-based, skipping sources
    past n."""
    lines = [l for l in text.splitlines() if l.strip() and not l.lstrip().startswith("%")]
    r, c = lines[0].split()[:2]
    n = max(int(r), int(c))
    out = []
    for l in lines[1:]:
        p = l.split()
        if len(p) >= 2 and int(p[0]) <= n:
            out.append((int(p[0]) - 1, int(p[1]) - 1))
    return n, out


def csr(n, pairs, sort=False, dedup=False, no_self=False, sym=False):
    lists = [[] for _ in range(n)]
    for u, v in pairs:
        if no_self and u == v:
            continue
        lists[u].append(v)
        if sym and u != v:
            lists[v].append(u)
    if sort or dedup:
        lists = [sorted(set(l)) if dedup else sorted(l) for l in lists]
    idx = np.zeros(n + 1, dtype=np.uint64)
    idx[1:] = np.cumsum([len(l) for l in lists])
    adj = np.array([v for l in lists for v in l], dtype=np.int32)
    return idx, adj


def test_sample_mtx_converts_to_the_reference_converters_output(tmp_path):
    out = str(tmp_path / "s.egr")
    st = convert(os.path.join(GOLDEN, "sample.mtx"), out)
    assert sha(out) == META["efficient_converter sample.mtx"]   # the reference converter's output
    assert sha(out) == sha(os.path.join(GOLDEN, "sample.egr"))   # which is the sample graph itself
    assert list(st) == [2000, 16000, 0, 0, 16000]


def test_edge_cases_convert_to_the_reference_converters_output(tmp_path):
    src = os.path.join(GOLDEN, "edge_cases.mtx")
    assert sha(src) == META["edge_cases.mtx"]
    out = str(tmp_path / "e.egr")
    st = convert(src, out)
    assert sha(out) == META["efficient_converter edge_cases.mtx"]
    assert open(out, "rb").read() == open(os.path.join(GOLDEN, "edge_cases_converted.egr"), "rb").read()
    n, pairs = parse_mtx(open(src).read())
    assert int(st[0]) == n and int(st[2]) == 1 and int(st[3]) == 2   # one source past n, two self-loops


@pytest.mark.parametrize("flags", [1, 2, 3, 4, 6, 8, 10, 14])
def test_converter_modes_vs_restatement(tmp_path, flags):
    src = os.path.join(GOLDEN, "edge_cases.mtx")
    out = str(tmp_path / "e.egr")
    convert(src, out, flags)
    n, pairs = parse_mtx(open(src).read())
    idx, adj = csr(n, pairs, sort=bool(flags & 1), dedup=bool(flags & 2), no_self=bool(flags & 4), sym=bool(flags & 8))
    n2, idx2, adj2 = O.read_egr(out)
    assert n2 == n and np.array_equal(idx2, idx) and np.array_equal(adj2, adj)
    assert os.path.getsize(out) == 16 + 8 * (n + 1) + 4 * len(adj)


@pytest.mark.parametrize("flags", [0, 2, 14])
def test_converter_large_file_threaded(tmp_path, flags):
    """A file of a few MB: parsed by several threads (newline-aligned slices)."""
    rng = np.random.default_rng(3)
    n = 5000
    u = rng.integers(1, n + 1, 300000)
    v = rng.integers(1, n + 1, 300000)
    v[::50] = u[::50]
    src = str(tmp_path / "big.mtx")
    with open(src, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern general\n%% a comment\n")
        f.write(f"{n} {n} {len(u)}\n")
        f.write("".join(f"{a} {b}\n" for a, b in zip(u, v)))
    assert os.path.getsize(src) > 2 << 20
    out = str(tmp_path / "big.egr")
    convert(src, out, flags)
    pairs = list(zip((u - 1).tolist(), (v - 1).tolist()))
    idx, adj = csr(n, pairs, sort=bool(flags & 1), dedup=bool(flags & 2), no_self=bool(flags & 4),
                   sym=bool(flags & 8))
    n2, idx2, adj2 = O.read_egr(out)
    assert n2 == n and np.array_equal(idx2, idx) and np.array_equal(adj2, adj)


@pytest.mark.parametrize("body,what", [("3 3 2\n0 1\n", "1-based"), ("3 3 2\n1 4\n", "1-based"),
                                       ("% only a comment\n", "size line")])
def test_converter_rejects_bad_input(tmp_path, body, what):
    src = str(tmp_path / "bad.mtx")
    open(src, "w").write(body)
    rc = K.load().excent_mtx_to_egr(src.encode(), str(tmp_path / "o.egr").encode(), 0, None)
    assert rc == 3
    assert what.encode() in K.load().excent_last_error()


def test_converter_cli(tmp_path):
    out = str(tmp_path / "s.egr")
    r = subprocess.run([os.path.join(BIN, "excent_convert"), os.path.join(GOLDEN, "sample.mtx"), out, "--dedup"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "16000 written" in r.stdout
    assert sha(out) == sha(os.path.join(GOLDEN, "sample.egr"))   # its lists are sorted and distinct already
    r = subprocess.run([os.path.join(BIN, "excent_convert"), "a.mtx", out, "--frobnicate"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "unknown option --frobnicate" in r.stderr


def test_info_line_matches_the_reference_tool(tmp_path):
    r = subprocess.run([os.path.join(BIN, "excent_info"), os.path.join(GOLDEN, "sample.egr")], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == META["egr_info sample.egr"]
    # an asymmetric graph with self-loops, against the reference binary when it was built here
    ref = os.path.join(O.REF_DIR, "egr_info")
    n, idx, adj = O.rmat_graph(12, 8, 3, symmetric=False)
    adj = adj.copy()
    adj[::37] = np.repeat(np.arange(n), np.diff(idx.astype(np.int64)))[::37]   # some self-loops
    p = str(tmp_path / "d.egr")
    O.write_egr(p, idx, adj)
    ours = subprocess.run([os.path.join(BIN, "excent_info"), p], capture_output=True, text=True).stdout
    assert re.match(r"n=4096 m=\d+ .* reverse-edge missing [1-9]\d*/20000 .* self-loops [1-9]", ours), ours
    if os.path.exists(ref):
        assert ours == subprocess.run([ref, p], capture_output=True, text=True).stdout


def test_evict_tool(tmp_path):
    p = str(tmp_path / "f.bin")
    open(p, "wb").write(os.urandom(1 << 20))
    tool = os.path.join(BIN, "excent_evict")
    r = subprocess.run([tool, p], capture_output=True, text=True)
    assert re.match(r".*f\.bin: [0-9.]+% -> [0-9.]+% resident", r.stdout), r.stdout
    r = subprocess.run([tool, "--report", p], capture_output=True, text=True)
    assert r.returncode == 0 and float(r.stdout) >= 0.0
    r = subprocess.run([tool, str(tmp_path / "missing")], capture_output=True, text=True)
    assert r.returncode == 1
