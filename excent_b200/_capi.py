"""ctypes prototypes of libexcent_b200.so (include/excent_b200.h).

The library is built in-tree (``python -m excent_b200.build``) and loaded from
the package directory. There is no fallback: a missing or unloadable library
raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libexcent_b200.so")
CLI_PATH = os.path.join(PKG, "bin", "excent")

u64 = C.c_uint64
u64p = C.POINTER(C.c_uint64)
i32p = C.POINTER(C.c_int32)
u32p = C.POINTER(C.c_uint32)
u16p = C.POINTER(C.c_uint16)
u8p = C.POINTER(C.c_uint8)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
vp = C.c_void_p


class Measures(C.Structure):
    _fields_ = [("nm", C.c_int), ("kind", C.c_int * 3), ("eps", C.c_float * 3), ("scale", C.c_float * 3),
                ("divdeg", C.c_int * 3), ("beta", C.c_double), ("lambda_", C.c_double), ("flags", C.c_int)]


class PassLog(C.Structure):
    _fields_ = [("pending", u64), ("demand", u64), ("hot_pending", u64), ("pushed", u64),
                ("rsum", C.c_double * 3), ("n_list", C.c_int), ("n_range", C.c_int), ("lanes", u64),
                ("taken", u64)]


class Tune(C.Structure):
    _fields_ = [("hub_targets", C.c_int), ("hub_order", C.c_int), ("chunk_sweep", C.c_int), ("ms", C.c_double),
                ("sweep_demand", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("passes", C.c_int), ("pushed", u64), ("n_list", u64), ("n_range", u64), ("rsum", C.c_double * 3)]


# (name, restype, argtypes); every function returns an int status unless stated
PROTOS = [
    ("excent_last_error", C.c_char_p, []),
    ("excent_version", C.c_int, []),
    ("excent_measures_make", C.c_int, [C.POINTER(Measures), C.c_char_p, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.c_double, C.c_double]),
    ("excent_engine_create", C.c_int, [C.c_int, C.c_int, u64, C.POINTER(Measures), C.c_int, i32p, u64p,
                                       C.POINTER(vp)]),
    ("excent_engine_destroy", C.c_int, [vp]),
    ("excent_engine_upload_offsets", C.c_int, [vp, vp, u64, u64]),
    ("excent_engine_upload_device", C.c_int, [vp, vp, vp]),
    ("excent_engine_reserve_cache", C.c_int, [vp, u64]),
    ("excent_engine_load_cache", C.c_int, [vp, u64, u64, vp]),
    ("excent_engine_set_loaded", C.c_int, [vp, C.c_int, C.c_int]),
    ("excent_engine_init", C.c_int, [vp]),
    ("excent_engine_snapshot", C.c_int, [vp, C.c_int, u64p, u64p, f64p]),
    ("excent_engine_bitmap", C.c_int, [vp, u32p]),
    ("excent_engine_chunk_list", C.c_int, [vp, C.c_int, i32p, C.POINTER(C.c_uint)]),
    ("excent_engine_push_cached", C.c_int, [vp, u8p, u64p, C.c_double]),
    ("excent_engine_slots_create", C.c_int, [vp, u64, C.c_int, C.c_int]),
    ("excent_engine_slot_buffers", C.c_int, [vp, C.c_int, C.POINTER(i32p), C.POINTER(i32p), C.POINTER(u64p)]),
    ("excent_engine_slot_wait", C.c_int, [vp, C.c_int]),
    ("excent_engine_push_stream", C.c_int, [vp, C.c_int, C.c_int, u64p, C.c_double, C.c_int, C.c_int, C.c_int]),
    ("excent_engine_push_gather", C.c_int, [vp, C.c_int, C.c_int, u64]),
    ("excent_engine_hot_setup", C.c_int, [vp, C.c_int, i32p, u64p, u32p]),
    ("excent_engine_push_hot", C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
    ("excent_engine_hot_pending", C.c_int, [vp, C.c_int, C.c_int, i32p, C.POINTER(C.c_uint)]),
    ("excent_engine_hot_edges", C.c_int, [vp, i32p]),
    ("excent_mtx_to_egr", C.c_int, [C.c_char_p, C.c_char_p, C.c_int, u64p]),
    ("excent_engine_set_chunk_sweep", C.c_int, [vp, C.c_int]),
    ("excent_engine_set_claim_tiles", C.c_int, [vp, C.c_int]),
    ("excent_engine_set_sweep_demand", C.c_int, [vp, C.c_double]),
    ("excent_reduction_peak", C.c_int, [C.c_int, C.c_int, C.c_int, u64, f64p]),
    ("excent_engine_scatter_peak", C.c_int, [vp, f64p]),
    ("excent_engine_autotune", C.c_int, [vp, C.c_double, C.c_int, C.POINTER(Tune), C.POINTER(Tune), C.c_int,
                                         C.POINTER(C.c_int)]),
    ("excent_egr_report", C.c_int, [C.c_char_p, C.c_char_p, C.c_int]),
    ("excent_engine_sync", C.c_int, [vp]),
    ("excent_engine_solve", C.c_int, [vp, C.c_double, C.c_int, C.c_int]),
    ("excent_engine_resume", C.c_int, [vp, C.c_double, C.c_int, C.c_int]),
    ("excent_engine_seed", C.c_int, [vp, C.c_int, vp, vp]),
    ("excent_batch_create", C.c_int, [C.c_int, C.c_int, u64, vp, vp, C.c_int, C.c_int, C.c_double, C.POINTER(vp)]),
    ("excent_batch_destroy", C.c_int, [vp]),
    ("excent_batch_seed", C.c_int, [vp, C.c_int, vp, vp, vp, vp]),
    ("excent_batch_solve", C.c_int, [vp, C.c_int, C.c_int]),
    ("excent_batch_stats", C.c_int, [vp, C.POINTER(C.c_int), u64p, u64p, u64p, u64p, u64p]),
    ("excent_batch_read", C.c_int, [vp, C.c_int, C.c_int, vp]),
    ("excent_batch_stream", C.c_int, [vp, C.POINTER(vp)]),
    ("excent_batch_launches", C.c_int, [vp, u64p]),
    ("excent_batch_set_greedy", C.c_int, [vp, C.c_int]),
    ("excent_batch_set_dense", C.c_int, [vp, C.c_int]),
    ("excent_batch_autotune", C.c_int, [C.c_int, C.c_int, u64, vp, vp, C.c_int, C.c_double, C.c_int, vp, vp, vp, vp,
                                        C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), f64p]),
    ("excent_engine_stats", C.c_int, [vp, C.POINTER(Stats), C.POINTER(PassLog), C.c_int]),
    ("excent_engine_read", C.c_int, [vp, C.c_int, C.c_int, vp, u64, u64]),
    ("excent_engine_write", C.c_int, [vp, C.c_int, vp, vp]),
    ("excent_engine_trace", C.c_int, [vp, C.c_int]),
    ("excent_engine_read_trace", C.c_int, [vp, u16p]),
    ("excent_engine_launches", C.c_int, [vp, u64p]),
    ("excent_engine_stream", C.c_int, [vp, C.POINTER(vp)]),
    ("excent_engine_profile", C.c_int, [vp, C.c_int]),
    ("excent_engine_profile_read", C.c_int, [vp, f64p, u64p]),
    ("excent_wgraph_create", C.c_int, [C.c_int, C.c_int, u64, vp, vp, vp, C.POINTER(vp)]),
    ("excent_wgraph_destroy", C.c_int, [vp]),
    ("excent_wgraph_set_weights", C.c_int, [vp, vp]),
    ("excent_wgraph_forward", C.c_int, [vp, C.c_int, C.c_double, vp, C.c_float, C.c_int, vp, C.POINTER(C.c_int),
                                        u64p]),
    ("excent_wgraph_vjp", C.c_int, [vp, vp, C.c_float, C.c_int, vp, vp, C.POINTER(C.c_int), u64p]),
    ("excent_wgraph_lambda", C.c_int, [vp, vp]),
    ("excent_wgraph_loss_fp64", C.c_int, [vp, C.c_int, C.c_double, vp, vp, C.c_longlong, C.c_double, C.c_double,
                                          f64p]),
    ("excent_wgraph_grad_fp64", C.c_int, [vp, C.c_int, C.c_double, vp, vp, C.c_double, vp, vp]),
    ("excent_wgraph_stream", C.c_int, [vp, C.POINTER(vp)]),
    ("excent_wgraph_host_transposed", C.c_int, [vp]),
    ("excent_params_fp64", C.c_int, [C.c_int, C.c_int, vp, vp, C.c_double, f64p, vp]),
    ("excent_engine_ev_project", C.c_int, [vp, vp]),
    ("excent_engine_set_hub_targets", C.c_int, [vp, C.c_int]),
    ("excent_engine_set_hub_order", C.c_int, [vp, C.c_int]),
    ("excent_engine_host_cache", C.c_int, [vp, C.POINTER(vp), u64p]),
    ("excent_engine_host_cache_begin", C.c_int, [vp, C.POINTER(vp), u64p, C.POINTER(C.c_int)]),
    ("excent_engine_host_cache_pin", C.c_int, [vp, u64]),
    ("excent_engine_host_pushed", C.c_int, [vp, u64p]),
    ("excent_params_fp64_noalloc", C.c_int, [C.c_int, C.c_int, vp, vp, C.c_double, f64p, vp]),
    ("excent_reference_fp64", C.c_int, [C.c_int, C.c_int, vp, vp, C.c_int, C.c_double, C.c_double, C.c_double,
                                        C.c_int, f64p, C.POINTER(C.c_int)]),
    ("excent_device_info", C.c_int, [C.c_int, vp]),
    ("excent_egr_open", C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(vp)]),
    ("excent_egr_close", C.c_int, [vp]),
    ("excent_egr_info", C.c_int, [vp, C.POINTER(C.c_int), u64p, C.POINTER(C.c_int)]),
    ("excent_egr_read_offsets", C.c_int, [vp, u64, u64, vp]),
    ("excent_egr_read_edges", C.c_int, [vp, u64, u64, vp]),
    ("excent_egr_prefetch", C.c_int, [vp, vp, C.c_int, u64p, u64p]),
    ("excent_egr_drop_cache", C.c_int, [vp, u64, u64, u64, u64]),
    ("excent_chunk_cap", C.c_uint64, [u64, C.c_double, C.c_double, C.c_double]),
    ("excent_plan_chunks", C.c_int, [C.c_int, vp, u64, C.POINTER(C.c_int), vp, C.c_int]),
    ("excent_cache_chunks", C.c_int, [C.c_int, vp, u64, u64, C.POINTER(C.c_int)]),
    ("excent_hot_select", C.c_int, [C.c_int, vp, u64, vp, C.POINTER(C.c_int), vp, vp, vp, u64p]),
    ("excent_fetch_plan", C.c_int, [C.c_int, vp, vp, vp, vp, C.c_double, C.c_int, C.c_int, vp, vp, vp, u64p, u64p,
                                    C.POINTER(C.c_int)]),
    ("excent_gather_list", C.c_int, [C.c_int, C.c_int, vp, vp, vp, vp, C.POINTER(C.c_int)]),
    ("excent_tau", C.c_double, [C.c_double, vp, vp]),
    ("excent_cli_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    ("excent_params_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    ("excent_reference_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    ("excent_convert_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    ("excent_info_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    ("excent_evict_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p)]),
    ("excent_rmat_generate", C.c_int, [C.c_int, C.c_int, C.c_int, u64, C.c_double, C.c_double, C.c_double,
                                       C.c_int, C.c_int, C.POINTER(vp)]),
    ("excent_ppr_fp64", C.c_int, [C.c_int, C.c_int, vp, vp, C.c_double, C.c_int, vp, vp, C.c_double, C.c_int, vp,
                                  C.POINTER(C.c_int)]),
    ("excent_rmat_write_egr", C.c_int, [C.c_int, C.c_int, C.c_int, u64, C.c_double, C.c_double, C.c_double, u64,
                                        C.c_char_p, u64p, C.POINTER(C.c_int)]),
    ("excent_dgraph_info", C.c_int, [vp, C.POINTER(C.c_int), u64p]),
    ("excent_dgraph_device_ptrs", C.c_int, [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
    ("excent_dgraph_download", C.c_int, [vp, vp, vp, vp]),
    ("excent_dgraph_destroy", C.c_int, [vp]),
]


class ExcentError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed with status {code}: {msg}")
        self.code = code


_lib = None


def load():
    """Load libexcent_b200.so; raise ImportError if it is missing (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m excent_b200.build` "
                          "(the engine has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, res, args in PROTOS:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def call(name, *args):
    """Call a status-returning entry point; raise ExcentError on failure."""
    L = load()
    rc = getattr(L, name)(*args)
    if rc != 0:
        raise ExcentError(name, rc, L.excent_last_error().decode(errors="replace"))
    return rc
