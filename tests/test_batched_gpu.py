"""Batched personalized PageRank / Katz against the FP64 oracle and against
one-at-a-time seeded solves of the plain engine."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import excent_b200 as X  # noqa: E402


def queries(n, nq, seed, max_size=64):
    rng = np.random.default_rng(seed)
    sizes = np.clip(np.floor(np.exp(rng.uniform(0, np.log(max_size), nq))).astype(int), 1, max_size)
    return [np.sort(rng.choice(n, s, replace=False)).astype(np.int32) for s in sizes]


@pytest.fixture(scope="module")
def dgraph():
    g = X.DeviceGraph(12, 16, 7)
    idx, adj, _ = g.download()
    yield g, idx, adj[:g.m]
    g.close()


@pytest.mark.parametrize("B", [32, 64, 128, 256])
@pytest.mark.parametrize("use_graph", [True, False])
def test_batched_ppr_vs_oracle(dgraph, B, use_graph):
    g, idx, adj = dgraph
    n = g.n
    nq = B - 3  # some idle lanes
    qs = queries(n, nq, B)
    d = 0.85
    eps = 1e-4 * (1 - d)
    di, da, _ = g.device_ptrs()
    b = X.Batch(n, g.m, di, da, B, "ppr", d)
    b.seed(qs, [(1 - d) / len(s) for s in qs], eps)
    st = b.solve(use_graph=use_graph)
    assert st["passes"] > 0 and st["pushed_edges"] > 0
    for q in range(0, nq, 7):
        r = b.read(q, residual=True)
        assert np.all(np.abs(r) <= np.float32(eps))
        x = b.read(q)
        t = np.zeros(n)
        t[qs[q]] = 1.0 / len(qs[q])
        ref = O.ppr(n, idx, adj, t, kind=0, d=d)
        err = np.abs(x - ref).sum()
        # the push conserves mass, so the L1 error is at most |r|_1 / (1 - d); 10% + 1e-5 slack for FP32
        assert err <= 1.1 * np.abs(r.astype(np.float64)).sum() / (1 - d) + 1e-5, (q, err)
    assert np.all(b.read(nq) == 0)  # idle lane untouched
    b.close()


def test_batched_matches_sequential_plain_solves(dgraph):
    g, idx, adj = dgraph
    n = g.n
    qs = queries(n, 32, 3)
    d = 0.85
    eps = 1e-4 * (1 - d)
    di, da, _ = g.device_ptrs()
    b = X.Batch(n, g.m, di, da, 32, "ppr", d)
    b.seed(qs, [(1 - d) / len(s) for s in qs], eps)
    b.solve()
    meas = X.measures("pr", eps_pr=eps)
    v0, e = X.plan_chunks(idx, len(adj))
    eng = X.Engine(n, g.m, meas, v0, e)
    eng.upload_device(di, da)
    for q in (0, 5, 31):
        X.seed_engine(eng, qs[q], (1 - d) / len(qs[q]))
        X.resume(eng)
        xs = eng.read(0)
        xb = b.read(q)
        t = np.zeros(n)
        t[qs[q]] = 1.0 / len(qs[q])
        ref = O.ppr(n, idx, adj, t, kind=0, d=d)
        e_seq = np.abs(xs - ref).sum()
        e_bat = np.abs(xb - ref).sum()
        assert e_bat <= 2 * e_seq + 1e-5, (q, e_bat, e_seq)
    eng.close()
    b.close()


def test_batched_katz_beta_vector(dgraph):
    g, idx, adj = dgraph
    n = g.n
    di, da, _ = g.device_ptrs()
    lam = X.params_fp64(n, di, da)["lambda"]
    alpha = 0.5 / lam
    rng = np.random.default_rng(1)
    B = 32
    seeds = [np.sort(rng.choice(n, 50, replace=False)).astype(np.int32) for _ in range(B)]
    vals = [rng.uniform(0.5, 1.5, 50).astype(np.float32) for _ in range(B)]
    b = X.Batch(n, g.m, di, da, B, "katz", alpha)
    b.seed(seeds, vals, 1e-6)
    b.solve()
    for q in (0, 17):
        beta = np.zeros(n)
        beta[seeds[q]] = vals[q]
        ref = O.ppr(n, idx, adj, beta, kind=1, d=alpha)
        x = b.read(q)
        assert np.abs(x - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max())
    b.close()


def test_autotuner_picks_a_width_and_mode(rmat16):
    n, idx, adj = rmat16
    d_idx = torch.from_numpy(idx.astype(np.int64)).cuda()
    d_adj = torch.from_numpy(adj).cuda()
    rng = np.random.default_rng(3)
    seeds = [np.sort(rng.choice(n, int(k), replace=False)).astype(np.int32) for k in rng.integers(1, 64, 40)]
    vals = [0.15 / len(q) for q in seeds]
    B, greedy, table = X.autotune_batch(n, len(adj), d_idx.data_ptr(), d_adj.data_ptr(), seeds, vals, 1e-4 * 0.15)
    assert B in (32, 64, 128, 256) and greedy in (False, True)
    assert len(table) == 8 and all(v > 0 for v in table.values())
    assert table[(B, int(greedy))] == min(table.values())


def test_device_fp64_ppr_matches_cpu_oracle(dgraph):
    g, idx, adj = dgraph
    n = g.n
    d = 0.85
    di, da, _ = g.device_ptrs()
    for q in queries(n, 3, 11, max_size=200):
        x, it = X.ppr_fp64(n, di, da, q, (1 - d) / len(q), d=d, tol=1e-13)
        t = np.zeros(n)
        t[q] = float(np.float32((1 - d) / len(q))) / (1 - d)   # the seed value as float32, like the device's
        ref = O.ppr(n, idx, adj, t, kind=0, d=d)
        assert it > 10
        assert np.abs(x - ref).max() <= 1e-10 * max(ref.max(), 1e-30) + 1e-14


@pytest.mark.parametrize("B,greedy", [(32, False), (128, True), (256, False)])
def test_batched_ppr_with_hub_segments(B, greedy):
    """Seeds on the highest-degree vertices push lists longer than 512 entries
    (queued as segments): the results still match the device FP64 oracle."""
    g = X.DeviceGraph(16, 16, 3)
    n = g.n
    idx, adj, _ = g.download()
    deg = np.diff(idx.astype(np.int64))
    assert deg.max() > 512
    top = np.argsort(-deg)[:8].astype(np.int32)
    d = 0.85
    eps = 1e-4 * (1 - d)
    qs = [np.array([v], dtype=np.int32) for v in top] + queries(n, B - 8, 5)
    di, da, _ = g.device_ptrs()
    b = X.Batch(n, g.m, di, da, B, "ppr", d)
    b.set_greedy(greedy)
    b.seed(qs, [(1 - d) / len(q) for q in qs], eps)
    b.solve()
    st = b.stats()
    assert st["hub_segments"] > 0
    for q in list(range(8)) + [B - 1]:
        r = b.read(q, residual=True)
        assert np.all(np.abs(r) <= np.float32(eps))
        ref, _ = X.ppr_fp64(n, di, da, qs[q], (1 - d) / len(qs[q]), d=d, tol=1e-12)
        err = np.abs(b.read(q) - ref).sum()
        assert err <= 1.1 * np.abs(r.astype(np.float64)).sum() / (1 - d) + 1e-5, (q, err)
    b.close()
    g.close()
