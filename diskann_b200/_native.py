"""ctypes binding of ``libdiskann_b200.so`` (the C ABI declared in include/diskann_b200.h).

The library is built in-tree (``diskann_b200/_lib``) by ``diskann_b200.build``.  There is no
fallback: if the library is missing, importing the search API raises.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
# DISKANN_B200_LIB selects another build of the same library (for example a profiling build).
LIB_PATH = os.environ.get("DISKANN_B200_LIB") or os.path.join(_HERE, "_lib", "libdiskann_b200.so")

# Every symbol include/diskann_b200.h declares (checked by the ABI test).
EXPORTED_SYMBOLS = (
    "dk_abi_version",
    "dk_last_error",
    "dk_knn_validate",
    "dk_index_create",
    "dk_index_destroy",
    "dk_index_get_info",
    "dk_search",
    "dk_search_device",
    "dk_search_device_noalloc",
    "dk_score_candidates",
    "dk_range_search",
    "dk_range_search_device",
    "dk_paged_search_create",
    "dk_paged_search_next",
    "dk_paged_search_destroy",
    "dk_inmem_index_create",
    "dk_inmem_set_tags",
    "dk_inmem_search",
    "dk_server_create",
    "dk_server_submit",
    "dk_server_poll",
    "dk_server_cancel",
    "dk_server_replay",
    "dk_server_get_info",
    "dk_server_destroy",
    "dk_distance",
    "dk_compute_medoid",
    "dk_build_vamana",
    "dk_build_vamana_device",
    "dk_pq_train",
    "dk_pq_encode",
)


class IndexDesc(ctypes.Structure):
    _fields_ = [
        ("num_points", ctypes.c_uint32),
        ("num_frozen", ctypes.c_uint32),
        ("dim", ctypes.c_uint32),
        ("metric", ctypes.c_int32),
        ("vectors", ctypes.c_void_p),
        ("vector_stride", ctypes.c_uint64),
        ("adjacency", ctypes.c_void_p),
        ("adjacency_stride", ctypes.c_uint64),
        ("degrees", ctypes.c_void_p),
        ("max_degree", ctypes.c_uint32),
        ("pq_chunks", ctypes.c_uint32),
        ("pq_offsets", ctypes.c_void_p),
        ("pq_pivots", ctypes.c_void_p),
        ("pq_codes", ctypes.c_void_p),
        ("pq_code_stride", ctypes.c_uint64),
        ("flags", ctypes.c_uint32),
    ]


INDEX_BF16 = 1
INDEX_FP8 = 2


class InmemDesc(ctypes.Structure):
    _fields_ = [
        ("capacity", ctypes.c_uint32),
        ("num_frozen", ctypes.c_uint32),
        ("dim", ctypes.c_uint32),
        ("metric", ctypes.c_int32),
        ("elem", ctypes.c_int32),
        ("rows", ctypes.c_void_p),
        ("row_stride", ctypes.c_uint64),
        ("adjacency", ctypes.c_void_p),
        ("adjacency_stride", ctypes.c_uint64),
        ("degrees", ctypes.c_void_p),
        ("max_degree", ctypes.c_uint32),
        ("external_ids", ctypes.c_void_p),
    ]


class IndexInfo(ctypes.Structure):
    _fields_ = [
        ("num_points", ctypes.c_uint32),
        ("num_frozen", ctypes.c_uint32),
        ("dim", ctypes.c_uint32),
        ("max_degree", ctypes.c_uint32),
        ("pq_chunks", ctypes.c_uint32),
        ("metric", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("device_bytes", ctypes.c_uint64),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("strategy", ctypes.c_int32),
        ("max_k", ctypes.c_uint32),
        ("max_l", ctypes.c_uint32),
        ("beam_width", ctypes.c_uint32),
        ("queue_depth", ctypes.c_uint32),
        ("max_slots", ctypes.c_uint32),
        ("streams", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("memory_bytes", ctypes.c_uint64),
    ]


class ServerInfo(ctypes.Structure):
    _fields_ = [
        ("slots", ctypes.c_uint32),
        ("queue_depth", ctypes.c_uint32),
        ("streams", ctypes.c_uint32),
        ("pad", ctypes.c_uint32),
        ("device_bytes", ctypes.c_uint64),
        ("launches", ctypes.c_uint64),
        ("memory_bytes", ctypes.c_uint64),
        ("reserved_bytes", ctypes.c_uint64),
    ]


_lock = threading.Lock()
_lib = None


def load():
    """Load the shared library (raises ``RuntimeError`` if it was not built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA library first "
                "(python -c 'import diskann_b200.build as b; b.build()')"
            )
        L = ctypes.CDLL(LIB_PATH)
        u32, u64, i32, vp = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p
        L.dk_abi_version.restype = i32
        L.dk_abi_version.argtypes = []
        L.dk_last_error.restype = i32
        L.dk_last_error.argtypes = [ctypes.c_char_p, u64]
        L.dk_knn_validate.restype = i32
        L.dk_knn_validate.argtypes = [u32, u32, u32]
        L.dk_index_create.restype = i32
        L.dk_index_create.argtypes = [ctypes.POINTER(IndexDesc), i32, ctypes.POINTER(vp)]
        L.dk_index_destroy.restype = i32
        L.dk_index_destroy.argtypes = [vp]
        L.dk_index_get_info.restype = i32
        L.dk_index_get_info.argtypes = [vp, ctypes.POINTER(IndexInfo)]
        L.dk_search.restype = i32
        L.dk_search.argtypes = [vp, i32, vp, u64, u32, u32, u32, u32, vp, vp, vp]
        L.dk_search_device.restype = i32
        L.dk_search_device.argtypes = [vp, i32, vp, u64, u32, u32, u32, u32, vp, vp, vp, vp]
        f32 = ctypes.c_float
        L.dk_range_search.restype = i32
        L.dk_range_search.argtypes = [vp, vp, u64, u32, u32, u32, f32, f32, f32, f32, u32, u32,
                                      vp, vp, vp]
        L.dk_range_search_device.restype = i32
        L.dk_range_search_device.argtypes = [vp, vp, u64, u32, u32, u32, f32, f32, f32, f32, u32,
                                             u32, vp, vp, vp, vp]
        L.dk_paged_search_create.restype = i32
        L.dk_paged_search_create.argtypes = [vp, vp, u64, u32, u32, vp, u32, u32,
                                             ctypes.POINTER(vp)]
        L.dk_paged_search_next.restype = i32
        L.dk_paged_search_next.argtypes = [vp, u32, vp, vp, vp]
        L.dk_paged_search_destroy.restype = i32
        L.dk_paged_search_destroy.argtypes = [vp]
        L.dk_inmem_index_create.restype = i32
        L.dk_inmem_index_create.argtypes = [ctypes.POINTER(InmemDesc), i32, ctypes.POINTER(vp)]
        L.dk_inmem_set_tags.restype = i32
        L.dk_inmem_set_tags.argtypes = [vp, u32, u32, vp]
        L.dk_inmem_search.restype = i32
        L.dk_inmem_search.argtypes = [vp, vp, u64, u32, u32, u32, u32, vp, vp, vp]
        L.dk_search_device_noalloc.restype = i32
        L.dk_search_device_noalloc.argtypes = [vp, i32, vp, u64, u32, u32, u32, u32, vp, vp, vp, vp]
        L.dk_score_candidates.restype = i32
        L.dk_score_candidates.argtypes = [vp, i32, vp, u64, u32, vp, u32, vp, vp]
        L.dk_server_create.restype = i32
        L.dk_server_create.argtypes = [vp, ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
        L.dk_server_submit.restype = i32
        L.dk_server_submit.argtypes = [vp, vp, u32, u32, ctypes.POINTER(u64)]
        L.dk_server_poll.restype = i32
        L.dk_server_poll.argtypes = [vp, u64, vp, vp, vp]
        L.dk_server_replay.restype = i32
        L.dk_server_cancel.restype = i32
        L.dk_server_cancel.argtypes = [vp, u64]
        L.dk_server_replay.argtypes = [vp, vp, u64, u32, vp, vp, vp, u32, vp, vp, vp]
        L.dk_server_get_info.restype = i32
        L.dk_server_get_info.argtypes = [vp, ctypes.POINTER(ServerInfo)]
        L.dk_server_destroy.restype = i32
        L.dk_server_destroy.argtypes = [vp]
        _lib = L
        return L


def last_error() -> tuple[int, str]:
    buf = ctypes.create_string_buffer(1024)
    status = load().dk_last_error(buf, len(buf))
    return int(status), buf.value.decode(errors="replace")
