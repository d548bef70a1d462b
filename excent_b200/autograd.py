"""torch.autograd binding of the weighted delta-push and its adjoint.

    g = WeightedGraph(n, d_idx, d_adj, w)          # device CSR (torch tensors or pointers)
    x = centrality(g, w, t, kind="pr", s=0.85)     # differentiable in w and t
    x[targets].sum().backward()                    # w.grad, t.grad from one adjoint solve

Forward and backward both run in libexcent_b200.so (excent_wgraph_forward /
excent_wgraph_vjp); torch only holds the device buffers. This is the thin
Python test binding of the VJP entry point.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._capi import call

KINDS = {"pr": 0, "katz": 1}


class WeightedGraph:
    """excent_wgraph: forward CSR + row-normalised weights + transpose on one device."""

    def __init__(self, n, idx: torch.Tensor, adj: torch.Tensor, w: torch.Tensor):
        assert idx.is_cuda and adj.is_cuda and w.is_cuda
        self.n, self.m = int(n), int(adj.numel())
        self.idx, self.adj = idx, adj      # kept alive: the library reads them
        self._w = w.detach().contiguous().float()
        h = C.c_void_p()
        call("excent_wgraph_create", idx.device.index or 0, self.n, self.m, idx.data_ptr(), adj.data_ptr(),
             self._w.data_ptr(), C.byref(h))
        self.h = h

    def set_weights(self, w: torch.Tensor):
        self._w = w.detach().contiguous().float()
        call("excent_wgraph_set_weights", self.h, self._w.data_ptr())

    def host_transposed(self):
        """Keep the transposed graph in pinned host memory, read in place by the adjoint push."""
        call("excent_wgraph_host_transposed", self.h)

    def close(self):
        if self.h:
            call("excent_wgraph_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, kind, s, t, eps, max_passes=1000000):
        x = torch.empty(self.n, dtype=torch.float32, device=self.idx.device)
        p, e = C.c_int(), C.c_uint64()
        torch.cuda.synchronize()
        call("excent_wgraph_forward", self.h, KINDS[kind], float(s), t.data_ptr() if t is not None else None,
             float(eps), int(max_passes), x.data_ptr(), C.byref(p), C.byref(e))
        return x, p.value, e.value

    def vjp(self, c, eps, max_passes=1000000):
        gt = torch.empty(self.n, dtype=torch.float32, device=self.idx.device)
        gw = torch.empty(max(self.m, 1), dtype=torch.float32, device=self.idx.device)
        p, e = C.c_int(), C.c_uint64()
        c = c.detach().contiguous().float()
        torch.cuda.synchronize()
        call("excent_wgraph_vjp", self.h, c.data_ptr(), float(eps), int(max_passes), gt.data_ptr(), gw.data_ptr(),
             C.byref(p), C.byref(e))
        return gt, gw[:self.m]


class _Centrality(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, t, g, kind, s, eps, eps_adj):
        g.set_weights(w)
        x, _, _ = g.forward(kind, s, t if t is not None else None, eps)
        ctx.g, ctx.eps_adj = g, eps_adj
        ctx.has_t = t is not None
        return x

    @staticmethod
    def backward(ctx, gx):
        gt, gw = ctx.g.vjp(gx, ctx.eps_adj)
        return gw, (gt if ctx.has_t else None), None, None, None, None, None


def centrality(g: WeightedGraph, w: torch.Tensor, t: torch.Tensor | None = None, kind="pr", s=0.85, eps=1e-7,
               eps_adj=None):
    """Weighted PageRank (x = (1-s) t + s W^T x) or Katz (x = t + s W^T x) with
    gradients for the raw edge weights w and the teleport / beta vector t."""
    return _Centrality.apply(w, t, g, kind, s, eps, eps if eps_adj is None else eps_adj)
