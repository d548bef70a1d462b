"""excent_params_fp64_noalloc: the allocation-free variant of the given-constants
computation, for hosts that own all device memory and do not allow a library
to call cudaMalloc (a framework's or server's own memory pool, or a pipeline
that cannot take the device synchronisation cudaMalloc/cudaFree may cause).

It must give the same lambda1, Katz alpha, eigenvector and Katz means and unit
principal eigenvector as excent_params_fp64, on two calls in a row (the
static scratch array keeps the previous call's contents), and reject graphs
larger than its scratch. This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a GPU", allow_module_level=True)

import excent_b200 as X  # noqa: E402
from excent_b200._capi import call, load  # noqa: E402


def params(fn, n, d_idx, d_adj):
    out = np.zeros(5, dtype=np.float64)
    v1 = torch.empty(n, dtype=torch.float32, device="cuda")
    call(fn, 0, n, d_idx, d_adj, 0.85, out.ctypes.data_as(C.POINTER(C.c_double)), v1.data_ptr())
    return out, v1.cpu().numpy()


@pytest.mark.parametrize("scale,seed", [(10, 1), (14, 2)])
def test_noalloc_matches_allocating_entry_point_twice(scale, seed):
    g = X.DeviceGraph(scale, 16, seed)
    di, da, _ = g.device_ptrs()
    ref, v_ref = params("excent_params_fp64", g.n, di, da)
    for call_no in range(2):
        got, v = params("excent_params_fp64_noalloc", g.n, di, da)
        assert abs(got[0] - ref[0]) <= 1e-10 * ref[0], (call_no, got[0], ref[0])      # lambda1
        assert abs(got[1] - ref[1]) <= 1e-10 * ref[1]                                 # Katz alpha
        assert abs(got[2] - ref[2]) <= 1e-8 * abs(ref[2])                             # eigenvector mean
        assert abs(got[3] - ref[3]) <= 1e-8 * abs(ref[3])                             # Katz mean
        assert np.abs(v - v_ref).max() < 1e-5                                         # unit eigenvector
    g.close()


def test_noalloc_call_leaves_free_device_memory_unchanged():
    """The property the entry point exists for: after a warm-up call (module
    load, lazy context state), a further call takes no device memory at all."""
    g = X.DeviceGraph(12, 16, 3)
    di, da, _ = g.device_ptrs()
    out = np.zeros(5, dtype=np.float64)
    v1 = torch.empty(g.n, dtype=torch.float32, device="cuda")
    call("excent_params_fp64_noalloc", 0, g.n, di, da, 0.85, out.ctypes.data_as(C.POINTER(C.c_double)), v1.data_ptr())
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call("excent_params_fp64_noalloc", 0, g.n, di, da, 0.85, out.ctypes.data_as(C.POINTER(C.c_double)),
             v1.data_ptr())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    g.close()


def test_noalloc_rejects_an_edgeless_graph():
    L = load()
    n = 64
    idx = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    adj = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = np.zeros(5, dtype=np.float64)
    for fn in ("excent_params_fp64_noalloc", "excent_params_fp64"):
        rc = getattr(L, fn)(0, n, C.c_void_p(idx.data_ptr()), C.c_void_p(adj.data_ptr()), C.c_double(0.85),
                            out.ctypes.data_as(C.POINTER(C.c_double)), None)
        assert rc == 1, fn
        assert b"no edges" in L.excent_last_error()


def test_noalloc_rejects_graphs_beyond_its_scratch():
    L = load()
    out = np.zeros(5, dtype=np.float64)
    n = (1 << 20) + 1
    rc = L.excent_params_fp64_noalloc(0, n, 1, 1, 0.85, out.ctypes.data_as(C.POINTER(C.c_double)), None)
    assert rc == 1
    assert b"exceeds" in L.excent_last_error()
