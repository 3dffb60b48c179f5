"""ctypes binding of libgat (include/gat.h).

The library is loaded from this package directory (built in-tree by
graphautotune_b200.build).  A missing library raises ImportError-like
GatLibraryMissing: there is no Python fallback for any computation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libgat.so"


class GatLibraryMissing(RuntimeError):
    pass


class GatError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{STATUS_NAMES.get(status, status)}] {message}")
        self.status = status
        self.message = message


STATUS_NAMES = {
    0: "GAT_OK", 1: "GAT_ERR_ARGUMENT", 2: "GAT_ERR_PATTERN", 3: "GAT_ERR_IO",
    4: "GAT_ERR_CUDA", 5: "GAT_ERR_MEMORY", 6: "GAT_ERR_UNDEFINED",
    7: "GAT_ERR_DEVICE", 8: "GAT_ERR_STATE", 9: "GAT_ERR_CONFIG",
}
GAT_OK = 0
GAT_ERR_UNDEFINED = 6
MODE_EXACT = 0
MODE_REF_COMPAT = 1
UPLOAD_DEGREE_ORDER = 1


class gat_config(C.Structure):
    _fields_ = [
        ("set_search_type", C.c_int32),
        ("set_intersection_type", C.c_int32),
        ("vertex_store_type", C.c_int32),
        ("graph_backend_type", C.c_int32),
        ("num_blocks", C.c_int32),
        ("threads_per_block", C.c_int32),
        ("threads_per_warp", C.c_int32),
        ("max_regs", C.c_int32),
        ("chunk", C.c_int32),
        ("hub_bitmaps", C.c_int32),
        ("memory_budget", C.c_int64),
        ("special_kernels", C.c_int32),
        ("reserved1", C.c_int32),
        ("reserved", C.c_int64 * 3),
    ]


class gat_stats(C.Structure):
    _fields_ = [
        ("kernel_ms", C.c_double),
        ("total_ms", C.c_double),
        ("raw_sum", C.c_int64),
        ("divisor", C.c_int64),
        ("tasks", C.c_uint64),
        ("balg_bytes", C.c_uint64),
        ("grid", C.c_int32),
        ("block", C.c_int32),
        ("tile", C.c_int32),
        ("launches", C.c_int32),
        ("scratch_bytes", C.c_int64),
    ]


P = C.c_void_p
_SIGS = {
    "gat_last_error": (C.c_char_p, []),
    "gat_version": (C.c_char_p, []),
    "gat_pattern_from_adj": (C.c_int, [C.c_char_p, C.POINTER(P)]),
    "gat_pattern_vertices": (C.c_int, [P]),
    "gat_pattern_automorphisms": (C.c_int, [P, C.POINTER(C.c_int64)]),
    "gat_pattern_adjacency": (C.c_int, [P, C.c_char_p, C.c_size_t]),
    "gat_pattern_free": (None, [P]),
    "gat_enumerate_patterns": (C.c_int, [C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "gat_schedule_build": (C.c_int, [P, C.c_int, P, C.POINTER(P)]),
    "gat_schedule_variants": (C.c_int, [P, C.c_int, P, C.POINTER(C.c_int32)]),
    "gat_schedule_build_variant": (C.c_int, [P, C.c_int, P, C.c_int32, C.POINTER(P)]),
    "gat_schedule_mode": (C.c_int, [P]),
    "gat_schedule_dump": (C.c_int, [P, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "gat_schedule_plan": (C.c_int, [P, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "gat_schedule_free": (None, [P]),
    "gat_config_default": (None, [C.POINTER(gat_config)]),
    "gat_config_engine_default": (None, [C.POINTER(gat_config)]),
    "gat_config_parse": (C.c_int, [C.c_char_p, C.POINTER(gat_config)]),
    "gat_config_format": (C.c_int, [C.POINTER(gat_config), C.c_char_p, C.c_size_t]),
    "gat_graph_load": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(P)]),
    "gat_graph_from_csr": (C.c_int, [C.c_int32, C.c_int64, P, P, C.POINTER(P)]),
    "gat_graph_generate": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_uint64, C.POINTER(P)]),
    "gat_graph_generate_device": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double,
                                            C.c_double, C.c_double, C.c_uint64, P,
                                            C.POINTER(P)]),
    "gat_graph_from_csr_device": (C.c_int, [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, P,
                                            C.POINTER(P)]),
    "gat_graph_validate": (C.c_int, [P, C.c_int]),
    "gat_graph_save": (C.c_int, [P, C.c_char_p]),
    "gat_graph_info": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int32)]),
    "gat_graph_csr": (C.c_int, [P, C.POINTER(P), C.POINTER(P)]),
    "gat_graph_upload": (C.c_int, [P, C.c_int, P]),
    "gat_graph_upload_ex": (C.c_int, [P, C.c_int, C.c_int64, C.c_int64, P]),
    "gat_graph_hubs": (C.c_int, [P, C.c_int, C.POINTER(C.c_int32)]),
    "gat_graph_ordered_csr": (C.c_int, [P, P, P]),
    "gat_graph_free": (None, [P]),
    "gat_executor_create": (C.c_int, [C.POINTER(gat_config), C.POINTER(P)]),
    "gat_executor_free": (None, [P]),
    "gat_executor_count": (C.c_int, [P, P, P, P, C.POINTER(C.c_uint64), C.POINTER(gat_stats)]),
    "gat_executor_count_balg": (C.c_int, [P, P, P, P, C.POINTER(C.c_uint64),
                                          C.POINTER(gat_stats)]),
    "gat_executor_count_range": (C.c_int, [P, P, P, P, C.c_int32, C.c_int32,
                                           C.POINTER(C.c_int64), C.POINTER(gat_stats)]),
    "gat_executor_count_shard": (C.c_int, [P, P, P, P, C.c_int32, C.c_int32,
                                           C.POINTER(C.c_int64), C.POINTER(gat_stats)]),
    "gat_executor_count_shard_balg": (C.c_int, [P, P, P, P, C.c_int32, C.c_int32,
                                                C.POINTER(C.c_int64), C.POINTER(gat_stats)]),
    "gat_batch_create": (C.c_int, [C.POINTER(P)]),
    "gat_batch_add": (C.c_int, [P, P, P, C.POINTER(C.c_int32)]),
    "gat_batch_add_shard": (C.c_int, [P, P, P, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "gat_batch_prepare": (C.c_int, [P, C.POINTER(gat_config), C.c_int]),
    "gat_batch_run": (C.c_int, [P, C.POINTER(gat_stats)]),
    "gat_batch_counts": (C.c_int, [P, C.POINTER(C.c_uint64), C.c_size_t]),
    "gat_batch_size": (C.c_int, [P]),
    "gat_batch_free": (None, [P]),
    "gat_count_noalloc": (C.c_int, [P, P, C.c_int32, C.c_int64, C.c_int32, P,
                                    C.POINTER(gat_config), P, P]),
    "gat_count": (C.c_int, [P, P, C.POINTER(gat_config), C.POINTER(C.c_uint64),
                            C.POINTER(gat_stats)]),
}

_lib = None


def exported_names() -> list[str]:
    return sorted(_SIGS)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise GatLibraryMissing(
                f"{LIB_PATH} is not built; run `python -m graphautotune_b200.build`")
        l = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(status: int) -> None:
    if status != GAT_OK:
        msg = lib().gat_last_error().decode(errors="replace")
        raise GatError(status, msg)


def read_string(fn, *args) -> str:
    need = C.c_size_t(0)
    check(fn(*args, None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    check(fn(*args, buf, need.value, C.byref(need)))
    return buf.value.decode()


def loaded_path() -> str:
    return str(LIB_PATH) if _lib is not None else ""


def version() -> str:
    return lib().gat_version().decode()


os.environ.setdefault("CUDA_MODULE_LOADING", "LAZY")
