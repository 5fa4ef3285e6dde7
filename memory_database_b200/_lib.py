"""ctypes binding of ``libolapcore_b200.so`` (the C-ABI in ``include/olap_capi.h``).

The library is the only compute path: if it is missing this module raises at
import, and every compute call raises :class:`OlapError` when the library
reports a failure (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libolapcore_b200.so"

OLAP_OK = 0
OLAP_ERR_INVALID = -1
OLAP_ERR_CUDA = -2
OLAP_ERR_NO_DEVICE = -3
OLAP_ERR_NOMEM = -4
OLAP_ERR_RANGE = -5
OLAP_ERR_CAPACITY = -6
OLAP_ERR_TIMEOUT = -7
OLAP_ERR_UNSUPPORTED = -8

DIM_NULL = 127
GROUP_NULL = 32767
VECTOR_SIZE = 1024
MAX_DIMS = 4

AGG_M1_PLUS_M2 = 0
AGG_M1 = 1
AGG_M2 = 2
AGG_M1_TIMES_M2 = 3
AGG_COUNT = 4

CMP_LE = 0
CMP_LT = 1

TUNE_BLOCK_THREADS = 0
TUNE_BLOCKS_PER_SM = 1
TUNE_SMEM_DIM_BYTES = 2
TUNE_SMEM_ACC_BYTES = 3
TUNE_HOST_CHUNK_ROWS = 4
TUNE_UNROLL = 5
TUNE_PROBE_BITS = 6
TUNE_SMEM_BITS_BYTES = 7
TUNE_GROUP_COMBINE = 8
TUNE_GROUP_PLAN = 9
TUNE_ASYNC_LOADS = 10
TUNE_COMPACT = 11
TUNE_SMEM_NIB_BYTES = 12
TUNE_HOST_INPLACE = 13
TUNE_MERGE_PROBES = 14
TUNE_PROBE_ORDER = 15
TUNE_JOIN_BUILD = 16


class OlapError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"olap status {status}: {message}")
        self.status = status


class BatchQuery(C.Structure):
    """Mirror of ``olap_batch_query``."""

    _fields_ = [
        ("row_begin", C.c_int64),
        ("row_end", C.c_int64),
        ("lo", C.c_int32 * MAX_DIMS),
        ("hi", C.c_int32 * MAX_DIMS),
        ("factor", C.c_int32 * MAX_DIMS),
        ("uses", C.c_int32),
        ("grouped", C.c_int32),
        ("group_nums", C.c_int64),
    ]


class Q5Tables(C.Structure):
    """Mirror of ``olap_q5_tables``."""

    _fields_ = [
        ("r_regionkey", C.c_void_p), ("n_region", C.c_int64),
        ("n_regionkey", C.c_void_p), ("n_nation", C.c_int64),
        ("s_nationkey", C.c_void_p), ("n_supp", C.c_int64),
        ("c_nationkey", C.c_void_p), ("n_cust", C.c_int64),
        ("o_custkey", C.c_void_p), ("o_orderdate", C.c_void_p), ("n_orders", C.c_int64),
        ("l_orderkey", C.c_void_p), ("l_suppkey", C.c_void_p), ("l_price", C.c_void_p),
        ("l_discount", C.c_void_p), ("n_lines", C.c_int64),
    ]


class Q5Query(C.Structure):
    """Mirror of ``olap_q5_query``."""

    _fields_ = [("region", C.c_int32), ("date1", C.c_int32), ("date2", C.c_int32)]


Q5_MAX_BATCH = 64


class StarjoinQuery(C.Structure):
    """Mirror of ``olap_starjoin_query``."""

    _fields_ = [
        ("dimvec_nums", C.c_int32),
        ("n_aggs", C.c_int32),
        ("agg", C.c_int32 * 2),
        ("dimvec", C.c_void_p * MAX_DIMS),
        ("dimvec_len", C.c_int64 * MAX_DIMS),
        ("fk", C.c_void_p * MAX_DIMS),
        ("factor", C.c_int32 * MAX_DIMS),
        ("m1", C.c_void_p),
        ("m2", C.c_void_p),
        ("row_begin", C.c_int64),
        ("row_end", C.c_int64),
        ("group_nums", C.c_int64),
    ]


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m memory_database_b200.build` "
            "(the CUDA library is the only compute path; there is no fallback)")
    lib = C.CDLL(str(LIB_PATH))
    vp, i32, i64, u64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.c_double
    sigs = {
        "olap_ctx_create": (C.c_int, [C.c_int, C.c_size_t, C.POINTER(vp)]),
        "olap_ctx_destroy": (C.c_int, [vp]),
        "olap_ctx_set_stream": (C.c_int, [vp, vp]),
        "olap_ctx_get_stream": (vp, [vp]),
        "olap_ctx_synchronize": (C.c_int, [vp]),
        "olap_ctx_set_tuning": (C.c_int, [vp, C.c_int, i64]),
        "olap_ctx_take_range_errors": (C.c_int, [vp, C.POINTER(i64)]),
        "olap_ctx_take_host_bytes": (C.c_int, [vp, C.POINTER(i64)]),
        "olap_ctx_last_error": (C.c_char_p, [vp]),
        "olap_status_string": (C.c_char_p, [C.c_int]),
        "olap_device_count": (C.c_int, []),
        "olap_build_info": (C.c_char_p, []),
        "olap_starjoin_groupsum": (C.c_int, [vp, C.POINTER(StarjoinQuery), vp, vp]),
        "olap_starjoin_launch_count": (C.c_int, [vp, C.POINTER(StarjoinQuery), C.c_int, C.POINTER(C.c_int)]),
        "olap_starjoin_groupsum_host": (C.c_int, [vp, C.POINTER(StarjoinQuery), vp, vp]),
        "olap_starjoin_autotune": (C.c_int, [vp, C.POINTER(StarjoinQuery), i64, C.POINTER(i64),
                                             C.POINTER(C.c_double)]),
        "olap_OLAPcore": (C.c_int, [vp, vp, vp, vp, vp, C.c_int, vp, i64, i64, vp, vp, vp,
                                    C.POINTER(i64)]),
        "olap_plan_olapcore": (C.c_int, [vp, vp, vp, vp, vp, C.POINTER(C.c_int), C.POINTER(i64)]),
        "olap_starjoin_groupsum_noalloc": (C.c_int, [C.POINTER(StarjoinQuery), vp, vp, vp, vp]),
        "olap_select_rowids": (C.c_int, [vp, vp, i64, i32, C.c_int, vp, i64, vp, vp]),
        "olap_select_bitmap": (C.c_int, [vp, vp, i64, i32, C.c_int, vp]),
        "olap_selalgo": (C.c_int, [vp, i32, i64, vp, vp, vp, vp, vp, vp]),
        "olap_project_pairs": (C.c_int, [vp, i32, i64, vp, vp, vp, vp, vp]),
        "olap_project_pairs_rows": (C.c_int, [vp, i32, i64, vp, i64, i64, i64, vp, vp, vp]),
        "olap_gather_i32": (C.c_int, [vp, vp, i64, C.c_int, vp, i64, vp]),
        "olap_buffer_alloc": (C.c_int, [vp, C.c_size_t, C.POINTER(vp)]),
        "olap_buffer_free": (C.c_int, [vp, vp]),
        "olap_copy_h2d": (C.c_int, [vp, vp, vp, C.c_size_t]),
        "olap_copy_d2h": (C.c_int, [vp, vp, vp, C.c_size_t]),
        "olap_max_i32": (C.c_int, [vp, vp, i64, C.POINTER(i32)]),
        "olap_hashtable_capacity": (i64, [i64]),
        "olap_hashjoin_build": (C.c_int, [vp, vp, vp, i64, vp, i64]),
        "olap_hashjoin_probe": (C.c_int, [vp, vp, i64, vp, i64, vp, vp, vp, vp]),
        "olap_hashjoin_filter_words": (i64, [i64]),
        "olap_hashjoin_build_filter": (C.c_int, [vp, vp, i64, vp, i64]),
        "olap_hashjoin_build_filtered": (C.c_int, [vp, vp, vp, i64, vp, i64, vp, i64]),
        "olap_hashjoin_probe_filtered": (C.c_int, [vp, vp, i64, vp, i64, vp, i64, vp, vp, vp, vp]),
        "olap_vecjoin_build": (C.c_int, [vp, vp, vp, i64, vp, i64]),
        "olap_vecjoin_probe": (C.c_int, [vp, vp, i64, vp, i64, vp]),
        "olap_group_vector": (C.c_int, [vp, i64, vp, vp, vp, i64, vp, vp, vp]),
        "olap_group_hash_capacity": (i64, [i64]),
        "olap_group_hash": (C.c_int, [vp, i64, vp, i32, vp, vp, i64, vp, vp, vp, vp]),
        "olap_agg_fixed": (C.c_int, [vp, i64, vp, vp, vp, vp]),
        "olap_agg_f64": (C.c_int, [vp, i64, vp, vp, vp, vp]),
        "olap_join_cwm_sv": (C.c_int, [vp, vp, vp, vp, vp, C.c_int, vp, vp, i64]),
        "olap_agg_cwm_sv": (C.c_int, [vp, vp, i64, vp, vp, i64, vp, vp]),
        "olap_join_cwm_dv": (C.c_int, [vp, vp, vp, vp, vp, C.c_int, vp, vp, vp, vp, i64]),
        "olap_agg_cwm_dv": (C.c_int, [vp, vp, vp, i64, vp, vp, i64, i64, vp, vp]),
        "olap_starjoin_count": (C.c_int, [vp, i64, vp, vp, vp, vp]),
        "olap_starjoin_cwm_sv": (C.c_int, [vp, i64, vp, vp, vp, vp, vp]),
        "olap_starjoin_cwm_dv": (C.c_int, [vp, i64, vp, vp, vp, vp, vp, vp]),
        "olap_build_dimvec": (C.c_int, [vp, vp, vp, i64, i32, i32, C.c_int, vp]),
        "olap_batch_create": (C.c_int, [vp, C.c_int, C.POINTER(vp)]),
        "olap_batch_destroy": (C.c_int, [vp]),
        "olap_batch_set_dimension": (C.c_int, [vp, C.c_int, vp, vp, i64]),
        "olap_batch_run": (C.c_int, [vp, vp, C.c_int, vp, vp, vp, i64, C.c_int, vp, i64, vp, C.c_int]),
        "olap_batch_graph_captures": (C.c_int, [vp, C.POINTER(C.c_int64)]),
        "olap_batch_tune": (C.c_int, [vp, C.c_int, C.c_int]),
        "olap_batch_set_probe": (C.c_int, [vp, C.c_int]),
        "olap_batch_get_tuning": (C.c_int, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "olap_batch_autotune": (C.c_int, [vp, vp, C.c_int, vp, vp, vp, i64, C.c_int, vp, i64, vp, i64,
                                          C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        "olap_debug_wait_timeout": (C.c_int, [vp, C.c_uint32]),
        "olap_q5_chain": (C.c_int, [vp, C.POINTER(Q5Tables), i32, i32, i32, vp]),
        "olap_q5_batch": (C.c_int, [vp, C.POINTER(Q5Tables), C.POINTER(Q5Query), C.c_int, vp]),
        "olap_gen_uniform_i32_dev": (C.c_int, [vp, vp, i64, u64, u64, i32, i32]),
        "olap_gen_uniform_i32": (C.c_int, [vp, i64, u64, u64, i32, i32, C.c_int]),
        "olap_gen_zipf_i32_dev": (C.c_int, [vp, vp, i64, u64, u64, i64, f64]),
        "olap_gen_zipf_i32": (C.c_int, [vp, i64, u64, u64, i64, f64, C.c_int]),
        "olap_gen_dimvec_dev": (C.c_int, [vp, vp, i64, u64, u64, f64, i32]),
        "olap_gen_dimvec": (C.c_int, [vp, i64, u64, u64, f64, i32, C.c_int]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(status: int, ctx=None) -> int:
    """Raise :class:`OlapError` for a negative status; return it otherwise."""
    if status < 0:
        msg = lib.olap_status_string(status).decode()
        if ctx is not None:
            detail = lib.olap_ctx_last_error(ctx).decode()
            if detail:
                msg = f"{msg}: {detail}"
        raise OlapError(status, msg)
    return status


def device_count() -> int:
    return int(lib.olap_device_count())


def build_info() -> str:
    return lib.olap_build_info().decode()
