"""C-ABI boundary checks that need no GPU: the library loads, exports every
function include/*.h declares, and validates arguments with status codes."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(excent_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    import excent_b200._capi as K
    L = K.load()
    out = subprocess.run(["nm", "-D", "--defined-only", K.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    decl = declared_functions()
    assert len(decl) > 20
    missing = decl - exported
    assert not missing, missing
    # and the Python binding binds all of them
    bound = {p[0] for p in K.PROTOS}
    assert decl <= bound, decl - bound


def test_measures_validation():
    import excent_b200 as X
    M = X.measures("all", alpha=0.0929536, lam=9.1443499824, eps_katz=0.058337, eps_ev=0.0084467)
    assert M.nm == 3 and list(M.kind) == [0, 1, 2] and list(M.divdeg) == [1, 0, 0]
    assert np.float32(M.scale[0]) == np.float32(0.85)
    assert np.float32(M.scale[2]) == np.float32(1.0 / 9.1443499824)
    assert np.float32(M.eps[0]) == np.float32(0.01)
    for bad in [dict(measure="katz"), dict(measure="ev", lam=3.0), dict(measure="xx")]:
        with pytest.raises(X.ExcentError) as ei:
            X.measures(**bad)
        assert ei.value.code == 1


def test_python_planner_matches_oracle(sample, rmat12):
    import excent_b200 as X
    import oracle as O
    for n, idx, adj in [sample[:3], rmat12]:
        for cap in (1, 50, 1000, 10 ** 6):
            v0, e = X.plan_chunks(idx, cap)
            ref = O.plan_chunks(idx, cap)
            assert np.array_equal(v0, ref[:, 0]) and np.array_equal(e[1:], ref[:, 3])
    for m in (10, 4 * 10 ** 6, 10 ** 9, 5 * 10 ** 9):
        for cm in (0.0, 2.5):
            assert X.chunk_cap(m, cm) == O.chunk_cap(m, cm)


def test_engine_create_fails_with_status_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import excent_b200 as X
    M = X.measures("pr")
    with pytest.raises(X.ExcentError) as ei:
        X.Engine(10, 0, M, [0], [0, 0])
    assert ei.value.code == 2


@pytest.mark.parametrize("name,args", [
    ("excent_engine_set_sweep_demand", [None, 0.5]),
    ("excent_engine_set_claim_tiles", [None, 4]),
    ("excent_engine_set_chunk_sweep", [None, -1]),
    ("excent_engine_set_hub_order", [None, 3]),
    ("excent_engine_host_cache_pin", [None, 0]),
    ("excent_engine_host_cache_begin", [None, None, None, None]),
    ("excent_engine_autotune", [None, 0.5, 100, None, None, 0, None]),
])
def test_engine_entries_reject_a_null_engine(name, args):
    """The pass-order, tuning and host-cache entries check their arguments before any CUDA call."""
    import excent_b200._capi as K
    L = K.load()
    assert getattr(L, name)(*args) == 1
    assert L.excent_last_error()
