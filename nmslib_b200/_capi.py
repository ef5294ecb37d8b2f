"""ctypes binding of the engine's C ABI (include/nmslib_b200.h).

The shared library is built in-tree (nmslib_b200/libnmslib_b200.so, see build.py). There is no
fallback: if the library is missing or cannot load, every search raises.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnmslib_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "nmslib_b200.h")

OK = 0
ERR_BAD_FILE, ERR_UNSUPPORTED, ERR_BAD_ARG, ERR_OOM = -1, -2, -3, -4
ERR_DEVICE, ERR_TIMEOUT, ERR_CORRUPT_GRAPH, ERR_CAPACITY = -5, -6, -7, -8

SPACE_L2, SPACE_COSINE, SPACE_NEGDOT, SPACE_L1, SPACE_LINF, SPACE_L2SQR_SIFT = 0, 1, 2, 3, 4, 5
ALGO_HYBRID, ALGO_OLD, ALGO_V1MERGE = 0, 1, 2
FLAG_DEVICE_PTRS, FLAG_PLAIN_KERNEL, FLAG_CUDA_GRAPH, FLAG_EXACT_SCAN = 1, 2, 4, 8


class IndexInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("dim", ctypes.c_int32), ("dist_type", ctypes.c_int32),
                ("maxlevel", ctypes.c_int32), ("enterpoint", ctypes.c_int32), ("maxM", ctypes.c_int32),
                ("maxM0", ctypes.c_int32), ("ef", ctypes.c_int32), ("algo", ctypes.c_int32),
                ("device", ctypes.c_int32), ("device_bytes", ctypes.c_int64)]


class LaunchConfig(ctypes.Structure):
    _fields_ = [("warps_per_block", ctypes.c_int32), ("rows_per_group", ctypes.c_int32),
                ("stage_rows", ctypes.c_int32), ("visited_hash_log2", ctypes.c_int32),
                ("plain_slots", ctypes.c_int32), ("queries_per_warp", ctypes.c_int32),
                ("row_copy", ctypes.c_int32), ("query_order", ctypes.c_int32), ("host_copy", ctypes.c_int32)]


_lib = None


def header_symbols():
    """Names of every function the C header declares."""
    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"NMSG_API\s+[\w\s\*]+?\b(nmsg_\w+)\s*\(", text)))


def load(path: str = LIB_PATH):
    """Load the engine library (once) and declare argument types."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"nmslib_b200 engine library not built ({path}); run `python -m nmslib_b200.build`")
    lib = ctypes.CDLL(path)
    P, I32, I64, U32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32
    lib.nmsg_index_load.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)]
    lib.nmsg_index_load.restype = ctypes.c_int
    lib.nmsg_index_save.argtypes = [P, ctypes.c_char_p]
    lib.nmsg_index_save.restype = ctypes.c_int
    lib.nmsg_index_load_with_data.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.POINTER(P)]
    lib.nmsg_index_load_with_data.restype = ctypes.c_int
    lib.nmsg_index_save_with_data.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p]
    lib.nmsg_index_save_with_data.restype = ctypes.c_int
    lib.nmsg_knn_batch_u8.argtypes = [P, P, I64, I32, I32, P, P, I32, P, P, P, P, U32, P]
    lib.nmsg_knn_batch_u8.restype = ctypes.c_int
    lib.nmsg_index_free.argtypes = [P]
    lib.nmsg_index_free.restype = None
    lib.nmsg_index_info_get.argtypes = [P, ctypes.POINTER(IndexInfo)]
    lib.nmsg_index_info_get.restype = ctypes.c_int
    lib.nmsg_set_query_params.argtypes = [P, ctypes.c_int, ctypes.c_int]
    lib.nmsg_set_query_params.restype = ctypes.c_int
    lib.nmsg_knn_batch.argtypes = [P, P, I64, I32, I32, P, P, I32, P, P, P, P, U32, P]
    lib.nmsg_knn_batch.restype = ctypes.c_int
    lib.nmsg_knn_batch_noalloc.argtypes = [P, P, I64, I32, I32, I32, P, P, P, P]
    lib.nmsg_knn_batch_noalloc.restype = ctypes.c_int
    lib.nmsg_bruteforce_knn.argtypes = [P, P, I64, I32, I32, I32, P, P, P, P, U32, P]
    lib.nmsg_bruteforce_knn.restype = ctypes.c_int
    lib.nmsg_server_create.argtypes = [P, I64, I32, I32, I32, ctypes.POINTER(P)]
    lib.nmsg_server_create.restype = ctypes.c_int
    lib.nmsg_server_lanes.argtypes = [P]
    lib.nmsg_server_lanes.restype = ctypes.c_int
    lib.nmsg_server_submit.argtypes = [P, P, I32, I32, I32, ctypes.POINTER(ctypes.c_int64)]
    lib.nmsg_server_submit.restype = ctypes.c_int
    lib.nmsg_server_wait.argtypes = [P, I64, P, P, P, ctypes.POINTER(ctypes.c_double)]
    lib.nmsg_server_wait.restype = ctypes.c_int
    lib.nmsg_server_run_trace.argtypes = [P, P, P, P, P, P, P, I64, P, ctypes.POINTER(ctypes.c_double)]
    lib.nmsg_server_run_trace.restype = ctypes.c_int
    lib.nmsg_server_free.argtypes = [P]
    lib.nmsg_server_free.restype = None
    lib.nmsg_set_launch_config.argtypes = [P, ctypes.POINTER(LaunchConfig)]
    lib.nmsg_set_launch_config.restype = ctypes.c_int
    lib.nmsg_last_device_status.argtypes = [P]
    lib.nmsg_last_device_status.restype = ctypes.c_int
    lib.nmsg_last_kernel_launches.argtypes = [P]
    lib.nmsg_last_kernel_launches.restype = ctypes.c_int
    lib.nmsg_build_index.argtypes = [P, I64, I32, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_uint64, ctypes.c_char_p]
    lib.nmsg_build_index.restype = ctypes.c_int
    lib.nmsg_build_index_device.argtypes = [P, I64, I32, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_uint64, ctypes.c_int, ctypes.c_char_p]
    lib.nmsg_build_index_device.restype = ctypes.c_int
    lib.nmsg_build_last_error.argtypes = []
    lib.nmsg_build_last_error.restype = ctypes.c_char_p
    lib.nmsg_query_server_start.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(P)]
    lib.nmsg_query_server_start.restype = ctypes.c_int
    lib.nmsg_query_server_port.argtypes = [P]
    lib.nmsg_query_server_port.restype = ctypes.c_int
    lib.nmsg_query_server_stop.argtypes = [P]
    lib.nmsg_query_server_stop.restype = None
    lib.nmsg_last_error.argtypes = []
    lib.nmsg_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


def last_error() -> str:
    return load().nmsg_last_error().decode(errors="replace")


def build_index(data, space: int, M: int = 16, ef_construction: int = 200, ids=None, nthreads: int = 0,
                seed: int = 0, out_path: str = "index.hnsw", device=None):
    """HNSW build writing the reference's optimized file format: on the host (nmsg_build_index),
    or with the level-0 construction searches on GPU `device` (nmsg_build_index_device)."""
    import numpy as np
    lib = load()
    x = np.ascontiguousarray(data, dtype=np.float32)
    idv = None if ids is None else np.ascontiguousarray(ids, dtype=np.int32)
    args = (x.ctypes.data_as(ctypes.c_void_p), x.shape[0], x.shape[1] if x.ndim == 2 else 0,
            None if idv is None else idv.ctypes.data_as(ctypes.c_void_p), space, M, ef_construction, nthreads, seed)
    if device is None:
        rc = lib.nmsg_build_index(*args, os.fsencode(out_path))
    else:
        rc = lib.nmsg_build_index_device(*args, int(device), os.fsencode(out_path))
    if rc != OK:
        msg = lib.nmsg_build_last_error().decode(errors="replace")
        raise (ValueError if rc == ERR_BAD_ARG else RuntimeError)(msg)
    return out_path


def check(rc: int):
    """Map a status to the exception type the reference raises for the same failure
    (std::invalid_argument -> ValueError, runtime_error -> RuntimeError)."""
    if rc == OK:
        return
    msg = last_error()
    if rc == ERR_BAD_ARG:
        raise ValueError(msg)
    if rc == ERR_OOM:
        raise MemoryError(msg)
    raise RuntimeError(msg)
