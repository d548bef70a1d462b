"""Weighted forward solve, adjoint (VJP) and the torch.autograd binding,
against the CPU FP64 oracle, the device FP64 tools and FP64 central finite
differences."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import excent_b200 as X  # noqa: E402
from excent_b200.autograd import WeightedGraph, centrality  # noqa: E402


@pytest.fixture(scope="module")
def wg():
    """Directed weighted R-MAT, scale 12, edge factor 16, seed 4."""
    g = X.DeviceGraph(12, 16, 4, symmetric=False, weights=True)
    idx, adj, w = g.download()
    m = g.m
    dev = torch.device("cuda")
    t_idx = torch.from_numpy(idx.view(np.int64)).to(dev)
    t_adj = torch.from_numpy(adj[:m].copy()).to(dev)
    t_w = torch.from_numpy(w[:m].copy()).to(dev)
    G = WeightedGraph(g.n, t_idx, t_adj, t_w)
    yield g.n, idx, adj[:m].copy(), w[:m].copy(), t_w, G
    G.close()
    g.close()


def targets(n, k=100, seed=4):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, k, replace=False))


@pytest.mark.parametrize("kind,s", [("pr", 0.85), ("katz", 0.6)])
def test_forward_and_vjp_vs_cpu_oracle(wg, kind, s):
    n, idx, adj, w, t_w, G = wg
    G.set_weights(t_w)
    wn = O.row_normalise(idx, w)
    c0 = 1 - s if kind == "pr" else 1.0
    ones = np.ones(n)
    x_ref = O.weighted_forward(idx, adj, wn, c0, s, ones)
    x, passes, pushed = G.forward(kind, s, None, 1e-7)
    xs = x.cpu().numpy()
    assert passes > 0
    assert np.abs(xs - x_ref).max() <= 1e-4 * max(1.0, np.abs(x_ref).max())
    tg = targets(n)
    c = np.zeros(n)
    c[tg] = 1
    lam_ref = O.weighted_adjoint(idx, adj, wn, s, c)
    gw_ref = O.weighted_grad(idx, adj, w, wn, s, x_ref, lam_ref)
    gt, gw = G.vjp(torch.from_numpy(c.astype(np.float32)).cuda(), 1e-7)
    gt = gt.cpu().numpy()
    gw = gw.cpu().numpy()
    assert np.linalg.norm(gt - c0 * lam_ref) <= 1e-4 * np.linalg.norm(c0 * lam_ref)
    assert np.linalg.norm(gw - gw_ref) <= 1e-3 * np.linalg.norm(gw_ref)


def test_fp64_tools_vs_cpu_oracle(wg):
    n, idx, adj, w, t_w, G = wg
    G.set_weights(t_w)
    tg = targets(n)
    c = torch.zeros(n, device="cuda")
    c[torch.from_numpy(tg).cuda()] = 1
    import ctypes as C
    from excent_b200._capi import call
    loss = C.c_double()
    call("excent_wgraph_loss_fp64", G.h, 0, 0.85, None, c.data_ptr(), -1, 0.0, 1e-14, C.byref(loss))
    wn = O.row_normalise(idx, w)
    x_ref = O.weighted_forward(idx, adj, wn, 0.15, 0.85, np.ones(n))
    assert abs(loss.value - x_ref[tg].sum()) <= 1e-10 * abs(loss.value)
    gw64 = np.zeros(len(adj))
    gt64 = np.zeros(n)
    call("excent_wgraph_grad_fp64", G.h, 0, 0.85, None, c.data_ptr(), 1e-14, gt64.ctypes.data, gw64.ctypes.data)
    cc = np.zeros(n)
    cc[tg] = 1
    lam = O.weighted_adjoint(idx, adj, wn, 0.85, cc)
    gw_ref = O.weighted_grad(idx, adj, w, wn, 0.85, x_ref, lam)
    assert np.abs(gw64 - gw_ref).max() <= 1e-9 * np.abs(gw_ref).max()
    assert np.abs(gt64 - 0.15 * lam).max() <= 1e-9 * np.abs(lam).max()


def test_autograd_vs_fp64_central_differences(wg):
    n, idx, adj, w, t_w, G = wg
    tg = targets(n)
    w_t = t_w.clone().requires_grad_(True)
    t_t = torch.ones(n, device="cuda", requires_grad=True)
    x = centrality(G, w_t, t_t, "pr", 0.85, eps=1e-8)
    L = x[torch.from_numpy(tg).cuda()].sum()
    L.backward()
    gw = w_t.grad.cpu().numpy()
    gt = t_t.grad.cpu().numpy()
    import ctypes as C
    from excent_b200._capi import call
    G.set_weights(t_w)
    c = torch.zeros(n, device="cuda")
    c[torch.from_numpy(tg).cuda()] = 1
    rng = np.random.default_rng(4)
    edges = rng.choice(len(adj), 64, replace=False)
    fd = []
    h = 1e-4
    for e in edges:
        lp, lm = C.c_double(), C.c_double()
        call("excent_wgraph_loss_fp64", G.h, 0, 0.85, None, c.data_ptr(), int(e), h, 1e-15, C.byref(lp))
        call("excent_wgraph_loss_fp64", G.h, 0, 0.85, None, c.data_ptr(), int(e), -h, 1e-15, C.byref(lm))
        fd.append((lp.value - lm.value) / (2 * h))
    fd = np.array(fd)
    ad = gw[edges]
    assert np.linalg.norm(ad - fd) <= 1e-3 * np.linalg.norm(fd), (ad[:5], fd[:5])
    # teleport gradient: L is linear in t, dL/dt = (1 - d) lambda
    gt64 = np.zeros(n)
    call("excent_wgraph_grad_fp64", G.h, 0, 0.85, None, c.data_ptr(), 1e-14, gt64.ctypes.data, None)
    assert np.linalg.norm(gt - gt64) <= 1e-3 * np.linalg.norm(gt64)


def test_katz_beta_gradient(wg):
    n, idx, adj, w, t_w, G = wg
    tg = targets(n, 50, 7)
    beta = torch.rand(n, device="cuda") + 0.5
    beta.requires_grad_(True)
    x = centrality(G, t_w.clone(), beta, "katz", 0.7, eps=1e-8)
    x[torch.from_numpy(tg).cuda()].sum().backward()
    wn = O.row_normalise(idx, w)
    c = np.zeros(n)
    c[tg] = 1
    lam = O.weighted_adjoint(idx, adj, wn, 0.7, c)
    g = beta.grad.cpu().numpy()
    assert np.linalg.norm(g - lam) <= 1e-4 * np.linalg.norm(lam)


def test_vjp_with_the_transposed_graph_in_host_memory():
    """The adjoint reads the transposed lists in place from pinned host memory
    and gives the gradients of the device-resident run (and of the oracle)."""
    g = X.DeviceGraph(12, 16, 4, symmetric=False, weights=True)
    idx, adj, w = g.download()
    m = g.m
    dev = torch.device("cuda")
    t_idx = torch.from_numpy(idx.view(np.int64)).to(dev)
    t_adj = torch.from_numpy(adj[:m].copy()).to(dev)
    t_w = torch.from_numpy(w[:m].copy()).to(dev)
    n = g.n
    c = np.zeros(n, dtype=np.float32)
    c[targets(n)] = 1
    res = []
    for host in (False, True):
        G = WeightedGraph(n, t_idx, t_adj, t_w)
        if host:
            G.host_transposed()
        G.forward("pr", 0.85, None, 1e-7)
        gt, gw = G.vjp(torch.from_numpy(c).cuda(), 1e-7)
        res.append((gt.cpu().numpy(), gw.cpu().numpy()))
        G.close()
    (gt0, gw0), (gt1, gw1) = res
    assert np.linalg.norm(gt1 - gt0) <= 1e-4 * np.linalg.norm(gt0)
    assert np.linalg.norm(gw1 - gw0) <= 1e-4 * np.linalg.norm(gw0)
    wn = O.row_normalise(idx, w[:m])
    x_ref = O.weighted_forward(idx, adj[:m], wn, 0.15, 0.85, np.ones(n))
    lam_ref = O.weighted_adjoint(idx, adj[:m], wn, 0.85, c.astype(np.float64))
    gw_ref = O.weighted_grad(idx, adj[:m], w[:m], wn, 0.85, x_ref, lam_ref)
    assert np.linalg.norm(gw1 - gw_ref) <= 1e-3 * np.linalg.norm(gw_ref)
    g.close()
