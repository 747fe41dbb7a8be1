"""ctypes binding of libordvec_b200.so (include/ordvec_b200.h).

The shared library is built in-tree (``ordvec_b200/libordvec_b200.so``) by
``ordvec_b200.build.build_library()``.  There is no fallback: if the library is
missing the import raises, so a GPU run can never silently route through a
CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libordvec_b200.so")

STATUS_NAMES = {
    0: "OK", 1: "NULL_POINTER", 2: "BAD_ARGUMENT", 3: "BAD_STRUCT_SIZE", 4: "UNSUPPORTED_FORMAT",
    5: "CORRUPT_INDEX", 6: "IO", 7: "DIM_MISMATCH", 8: "NONFINITE_QUERY", 9: "ROW_ID_OUT_OF_RANGE",
    10: "BUFFER_TOO_SMALL", 11: "UNSUPPORTED_OPERATION", 12: "PANIC", 13: "INTERNAL",
}

KIND_RANK_QUANT, KIND_BITMAP, KIND_SIGN_BITMAP, KIND_FASTSCAN, KIND_MULTIBUCKET, KIND_RANK = 1, 2, 3, 4, 5, 6


class OrdvecError(ValueError):
    """A non-OK status from the C ABI (ordvec-ffi status codes)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


class IndexInfo(C.Structure):
    _fields_ = [("struct_size", C.c_uint64), ("kind", C.c_uint32), ("format_version", C.c_uint32),
                ("dim", C.c_uint64), ("bit_width", C.c_uint32), ("n_top", C.c_uint32),
                ("vector_count", C.c_uint64), ("bytes_per_vec", C.c_uint64),
                ("source_file_size_bytes", C.c_uint64), ("capabilities", C.c_uint64),
                ("reserved", C.c_uint64 * 8)]


class SearchParams(C.Structure):
    _fields_ = [("struct_size", C.c_uint64), ("query", C.POINTER(C.c_float)), ("dim", C.c_uint64),
                ("k", C.c_uint64), ("candidate_rows", C.POINTER(C.c_uint32)),
                ("candidate_count", C.c_uint64), ("flags", C.c_uint64), ("user_tag", C.c_uint64),
                ("reserved", C.c_uint64 * 8)]


class SearchStats(C.Structure):
    _fields_ = [("struct_size", C.c_uint64), ("abi_version", C.c_uint32), ("kind", C.c_uint32),
                ("dim", C.c_uint64), ("bit_width", C.c_uint32), ("n_top", C.c_uint32),
                ("k", C.c_uint64), ("user_tag", C.c_uint64), ("vector_count", C.c_uint64),
                ("candidate_count", C.c_uint64), ("returned_count", C.c_uint64),
                ("total_ns", C.c_uint64), ("prepare_ns", C.c_uint64), ("score_ns", C.c_uint64),
                ("select_ns", C.c_uint64), ("vectors_scored", C.c_uint64), ("bytes_read", C.c_uint64),
                ("reserved", C.c_uint64 * 8)]


class ServerConfig(C.Structure):
    _fields_ = [("struct_size", C.c_uint64), ("workers", C.c_uint32), ("max_batch", C.c_uint32),
                ("hbm_budget_bytes", C.c_uint64), ("reserved", C.c_uint64 * 5)]


class ServerStats(C.Structure):
    _fields_ = [("struct_size", C.c_uint64), ("requests", C.c_uint64), ("queries", C.c_uint64),
                ("batches", C.c_uint64), ("peak_inflight_bytes", C.c_uint64),
                ("max_concurrent_batches", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double), ("warm_workers", C.c_uint64), ("reserved", C.c_uint64 * 3)]


class Hit(C.Structure):
    _fields_ = [("row_id", C.c_uint64), ("id", C.c_uint64), ("score", C.c_float), ("reserved", C.c_uint32)]


P, U32, U64, F, S = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_uint32
PP = C.POINTER(C.c_void_p)

SIGNATURES = {
    "ordvec_abi_version": (U32, []),
    "ordvec_version_string": (C.c_char_p, []),
    "ordvec_status_name": (C.c_char_p, [S]),
    "ordvec_last_error": (C.c_char_p, []),
    "ordvec_init": (S, []),
    "ordvec_index_info_init": (None, [P]),
    "ordvec_search_params_init": (None, [P]),
    "ordvec_search_stats_init": (None, [P]),
    "ordvec_index_load": (S, [C.c_char_p, U64, PP]),
    "ordvec_index_probe": (S, [C.c_char_p, U64, P]),
    "ordvec_index_info": (S, [P, P]),
    "ordvec_index_free": (None, [P]),
    "ordvec_index_search": (S, [P, P, P, U64, P, P]),
    "ovb_rankquant_new": (S, [U32, U32, PP]),
    "ovb_sign_bitmap_new": (S, [U32, PP]),
    "ovb_bitmap_new": (S, [U32, U32, PP]),
    "ovb_fastscan_new": (S, [U32, PP]),
    "ovb_multibucket_new": (S, [U32, U32, PP]),
    "ovb_rank_new": (S, [U32, PP]),
    "ovb_index_add": (S, [P, P, U64]),
    "ovb_index_add_device": (S, [P, P, U64]),
    "ovb_index_load_any": (S, [C.c_char_p, U64, PP]),
    "ovb_index_write": (S, [P, C.c_char_p]),
    "ovb_index_payload_bytes": (S, [P, C.POINTER(C.c_uint64)]),
    "ovb_index_payload": (S, [P, P, U64]),
    "ovb_rankquant_search": (S, [P, P, U64, U64, P, P]),
    "ovb_rankquant_search_subset": (S, [P, P, U64, P, P, U64, P, P]),
    "ovb_sign_bitmap_top_m": (S, [P, P, U64, U64, P]),
    "ovb_sign_bitmap_score_all": (S, [P, P, P]),
    "ovb_bitmap_search": (S, [P, P, U64, U64, P, P]),
    "ovb_bitmap_top_m": (S, [P, P, U64, U64, P]),
    "ovb_fastscan_search": (S, [P, P, U64, U64, P, P]),
    "ovb_multibucket_top_m": (S, [P, P, U64, P, U64, P]),
    "ovb_two_stage_search": (S, [P, P, P, U64, U64, U64, P, P]),
    "ovb_two_stage_search_device": (S, [P, P, P, U64, U64, U64, P, P, P]),
    "ovb_two_stage_search_device_ex": (S, [P, P, P, U64, U64, U64, P, P, P, U32]),
    "ovb_two_stage_profile": (S, [P, P, P, U64, U64, U64, P, P, P, P]),
    "ovb_rankquant_search_noalloc": (S, [P, P, U64, U64, P, P, P]),
    "ovb_last_launch_count": (U64, []),
    "ovb_set_device": (S, [C.c_int]),
    "ovb_synth_docs": (S, [U64, U64, U64, U32, F, P]),
    "ovb_synth_queries": (S, [U64, U64, U64, U32, F, F, P, P]),
    "ovb_rankquant_search_split": (S, [P, P, U64, U64, U32, P, P]),
    "ovb_rankquant_search_symmetric": (S, [P, P, U64, U64, P, P]),
    "ovb_rank_search": (S, [P, P, U64, U64, P, P]),
    "ovb_index_search_device": (S, [P, U32, P, U64, U64, P, P, P]),
    "ovb_selftest_bounded_wait": (S, [P, P]),
    "ovb_selftest_arm_tc_error": (S, []),
    "ovb_rank_search_asymmetric": (S, [P, P, U64, U64, P, P]),
    "ovb_rankquant_search_mixed": (S, [P, U32, P, P, P, U64, U64, P, P]),
    "ovb_mixed_plan_info": (S, [P, U64, U64, P, P, P]),
    "ovb_server_new": (S, [P, P]),
    "ovb_server_add_route": (S, [P, P, P, P]),
    "ovb_server_submit": (S, [P, U32, P, U64, U64, U64, P]),
    "ovb_server_wait": (S, [P, U64, P, P, U64, P, P]),
    "ovb_server_stats": (S, [P, P]),
    "ovb_server_free": (None, [P]),
}

_lib = None


def lib():
    """Load the library once; raise if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import ordvec_b200.build as b; b.build_library()'`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        msg = lib().ordvec_last_error()
        raise OrdvecError(status, msg.decode() if msg else "")
