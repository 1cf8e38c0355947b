"""ctypes binding of the C ABI in include/gz_b200.h (libgz_b200.so, built in-tree).

There is no CPU fallback: if the shared library cannot be loaded (or built with nvcc) every
entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libgz_b200.so")

GZ_OK = 0
GZ_ERR_INVALID = 1
GZ_ERR_CUDA = 2
GZ_ERR_OUT_OF_SAMPLES = 3
GZ_ERR_LOCKED = 4
GZ_ERR_BAD_VERTEX = 5
GZ_ERR_NOMEM = 6
GZ_ERR_IO = 7
GZ_ERR_TIMEOUT = 8
GZ_ERR_BAD_SAMPLE = 9
GZ_ERR_NO_DEVICE = 10
GZ_ERR_BUDGET = 11
GZ_CAMEO_SKETCH = 0
GZ_CUBE_SKETCH = 1


class gz_params_t(ctypes.Structure):
    _fields_ = [("num_vertices", ctypes.c_uint32), ("num_columns", ctypes.c_uint32),
                ("bkt_per_col", ctypes.c_uint32), ("num_buckets", ctypes.c_uint32),
                ("seed", ctypes.c_uint64), ("sketch_bytes", ctypes.c_uint64),
                ("desired_updates_per_batch", ctypes.c_uint64), ("max_rounds", ctypes.c_uint64),
                ("sketches_factor", ctypes.c_double), ("batch_factor", ctypes.c_double),
                ("vertices_per_tile", ctypes.c_uint32), ("num_tiles", ctypes.c_uint32),
                ("vertices_per_bin", ctypes.c_uint32), ("num_bins", ctypes.c_uint32),
                ("cols_per_sample", ctypes.c_uint32), ("sketch_algorithm", ctypes.c_uint32),
                ("in_place", ctypes.c_uint32), ("entry_form", ctypes.c_uint32)]


class gz_trace_rec_t(ctypes.Structure):
    _fields_ = [("round", ctypes.c_uint32), ("key", ctypes.c_uint32), ("result", ctypes.c_uint32),
                ("pad", ctypes.c_uint32), ("idx", ctypes.c_uint64)]


class gz_profile_t(ctypes.Structure):
    _fields_ = [("gutter_ms", ctypes.c_double), ("sketch_update_ms", ctypes.c_double),
                ("query_ms", ctypes.c_double), ("gutter_launches", ctypes.c_uint64),
                ("sketch_update_launches", ctypes.c_uint64), ("query_rounds", ctypes.c_uint64),
                ("entries_applied", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64)]


# (name, restype, argtypes) for every symbol of include/gz_b200.h
_H = ctypes.c_void_p
_P = ctypes.c_void_p
_u32, _u64, _sz, _i, _d = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_int, ctypes.c_double
SIGNATURES = [
    ("gz_version", ctypes.c_char_p, []),
    ("gz_status_string", ctypes.c_char_p, [_i]),
    ("gz_last_error", ctypes.c_char_p, []),
    ("gz_create", _i, [_u32, _u64, _d, _d, ctypes.POINTER(_H)]),
    ("gz_create_from_serialized", _i, [ctypes.c_char_p, _d, ctypes.POINTER(_H)]),
    ("gz_create_ex", _i, [_u32, _u64, _d, _d, _i, ctypes.POINTER(_H)]),
    ("gz_create_from_serialized_ex", _i, [ctypes.c_char_p, _d, _i, ctypes.POINTER(_H)]),
    ("gz_destroy", _i, [_H]),
    ("gz_get_params", _i, [_H, ctypes.POINTER(gz_params_t)]),
    ("gz_set_gutter_capacity", _i, [_H, _u64]),
    ("gz_allocate_worker_memory", _i, [_H, _sz]),
    ("gz_pre_insert", _i, [_H, _u32, _u32, _i, _i]),
    ("gz_apply_update_batch", _i, [_H, _i, _u32, _P, _sz]),
    ("gz_apply_raw_buckets_update", _i, [_H, _u32, _P]),
    ("gz_update", _i, [_H, _u32, _u32, _i]),
    ("gz_ingest_records", _i, [_H, _P, _sz]),
    ("gz_ingest_records_device", _i, [_H, _P, _sz]),
    ("gz_flush", _i, [_H]),
    ("gz_has_cached_query", _i, [_H, _i, ctypes.POINTER(_i)]),
    ("gz_query_submit", _i, [_H, ctypes.POINTER(_u64)]),
    ("gz_query_wait", _i, [_H, _u64, _P, ctypes.POINTER(_u32), ctypes.POINTER(_sz)]),
    ("gz_connected_components", _i, [_H, _P, ctypes.POINTER(_u32)]),
    ("gz_point_query", _i, [_H, _u32, _u32, ctypes.POINTER(_i)]),
    ("gz_last_query_rounds", _i, [_H, ctypes.POINTER(_sz)]),
    ("gz_spanning_forest", _i, [_H, _P, _sz, ctypes.POINTER(_sz)]),
    ("gz_write_binary", _i, [_H, ctypes.c_char_p]),
    ("gz_dump_sketches", _i, [_H, _P, _sz]),
    ("gz_clear", _i, [_H]),
    ("gz_measure_hash_rate", _i, [_i, ctypes.POINTER(_d)]),
    ("gz_measure_update_rate", _i, [_i, ctypes.POINTER(_d)]),
    ("gz_set_trace", _i, [_H, _i]),
    ("gz_get_trace", _i, [_H, _P, _sz, ctypes.POINTER(_sz)]),
    ("gz_set_profiling", _i, [_H, _i]),
    ("gz_get_profile", _i, [_H, ctypes.POINTER(gz_profile_t)]),
    ("gz_get_stream", _i, [_H, ctypes.POINTER(ctypes.c_void_p)]),
    ("gz_set_tuning", _i, [_H, _u32, _u32, _u32, _u32]),
    ("gz_set_direct_factor", _i, [_H, ctypes.c_double]),
    ("gz_set_query_graph", _i, [_H, _i]),
    ("gz_set_pipeline", _i, [_H, _i]),
    ("gz_set_eager_dsu", _i, [_H, _i]),
    ("gz_ingest_records_noalloc", _i, [_P, _u32, _u64, _d, _P, _sz, _P]),
    ("gz_batch_create", _i, [_u32, _P, _P, _d, _P, ctypes.POINTER(_H)]),
    ("gz_batch_destroy", _i, [_H]),
    ("gz_batch_get_params", _i, [_H, _u32, ctypes.POINTER(gz_params_t)]),
    ("gz_batch_ingest_device", _i, [_H, _P, _P]),
    ("gz_batch_ingest", _i, [_H, _P, _P]),
    ("gz_batch_clear", _i, [_H]),
    ("gz_batch_connected_components", _i, [_H, _P, _P, _P, _P]),
    ("gz_batch_dump_sketches", _i, [_H, _u32, _P, _sz]),
    ("gz_batch_load_sketches", _i, [_H, _u32, _P, _sz]),
    ("gz_batch_set_tuning", _i, [_H, _u32, _u32, _P]),
    ("gz_batch_set_route", _i, [_H, _d]),
    ("gz_batch_autotune", _i, [_H, _u32, _P]),
    ("gz_batch_set_profiling", _i, [_H, _i]),
    ("gz_server_tenant_bytes", _i, [_u32, _d, ctypes.POINTER(_u64)]),
    ("gz_server_create", _i, [_u64, _u64, _d, ctypes.POINTER(_H)]),
    ("gz_server_destroy", _i, [_H]),
    ("gz_server_admit", _i, [_H, _u32, _u64, ctypes.POINTER(_u32)]),
    ("gz_server_evict", _i, [_H, _u32]),
    ("gz_server_usage", _i, [_H, ctypes.POINTER(_u64), ctypes.POINTER(_u64), ctypes.POINTER(_u32)]),
    ("gz_server_set_route", _i, [_H, _d]),
    ("gz_server_get_params", _i, [_H, _u32, ctypes.POINTER(gz_params_t)]),
    ("gz_server_ingest", _i, [_H, _u32, _P, _P, _P]),
    ("gz_server_ingest_segments", _i, [_H, _u32, _P, _P, _P]),
    ("gz_host_register", _i, [_P, _u64]),
    ("gz_host_unregister", _i, [_P]),
    ("gz_server_set_query_snapshot", _i, [_H, _i]),
    ("gz_server_query_submit", _i, [_H, _u32, _P, ctypes.POINTER(_u64)]),
    ("gz_server_query_wait", _i, [_H, _u64, _P, _P, _P, _P]),
    ("gz_server_query_ready", _i, [_H, _u64, ctypes.POINTER(_i)]),
    ("gz_server_dump_sketches", _i, [_H, _u32, _P, _sz]),
    ("gz_server_write_binary", _i, [_H, _u32, ctypes.c_char_p]),
    ("gz_server_admit_serialized", _i, [_H, ctypes.c_char_p, ctypes.POINTER(_u32)]),
    ("gz_batch_get_profile", _i, [_H, ctypes.POINTER(gz_profile_t)]),
]

_lib = None
_lock = threading.Lock()


def load(build_if_missing: bool = True):
    """Load libgz_b200.so (building it with nvcc first if it is absent or stale)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing:
            from . import build as _build
            try:
                _build.build()
            except Exception as e:  # nvcc missing and no prebuilt library
                if not os.path.exists(LIB_PATH):
                    raise RuntimeError(f"libgz_b200.so is not built and cannot be built: {e}")
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; run python -m graphzeppelin_b200.build")
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error() -> str:
    return load().gz_last_error().decode()


def status_string(rc: int) -> str:
    return load().gz_status_string(rc).decode()
