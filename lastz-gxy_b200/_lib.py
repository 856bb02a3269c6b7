"""ctypes binding of libgxyseed.so, the C ABI declared in include/gxy_seed.h.

The product path runs only through this library: there is no CPU fallback.  If
the shared object is missing or the device is not a B200, every entry point
raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgxyseed.so")

(GXY_OK, GXY_EINVAL, GXY_ENOMEM, GXY_EUNSUPPORTED, GXY_ETIMEDOUT, GXY_ECUDA, GXY_ENOTREADY, GXY_EOVERFLOW,
 GXY_ECANCELED) = range(9)


class GxyError(RuntimeError):
    """A gxy_status other than GXY_OK, with the library's message."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"gxy status {status}: {msg}")
        self.status = status


class PackedSeqC(C.Structure):
    _fields_ = [("codes", C.c_void_p), ("valid", C.c_void_p), ("mask", C.c_void_p), ("len", C.c_uint64)]


class SearchParamsC(C.Structure):
    _fields_ = [
        ("sub", C.c_int32 * 16),
        ("ambig", C.c_int32),
        ("xdrop", C.c_int32),
        ("hspthresh", C.c_int32),
        ("step", C.c_uint32),
        ("transitions", C.c_uint8),
        ("has_entropy", C.c_uint8),
        ("pad_", C.c_uint8 * 2),
        ("entropy_thr", C.c_int32),
    ]


class HspC(C.Structure):
    _fields_ = [("t_start", C.c_uint32), ("q_start", C.c_uint32), ("length", C.c_uint32), ("score", C.c_int32)]


class HspBufC(C.Structure):
    _fields_ = [("hsps", C.POINTER(HspC)), ("len", C.c_uint64), ("cap", C.c_uint64)]


class StatsC(C.Structure):
    _fields_ = [("windows", C.c_uint64), ("raw_hits", C.c_uint64), ("candidates", C.c_uint64),
                ("hsps", C.c_uint64), ("device_ms", C.c_double), ("screen_ms", C.c_double),
                ("columns", C.c_uint64), ("enum_ms", C.c_double), ("passes", C.c_uint32), ("reruns", C.c_uint32),
                ("survivors", C.c_uint64), ("filter_columns", C.c_uint64), ("filter_ms", C.c_double),
                ("rounds", C.c_uint32), ("graph_updates", C.c_uint32)]


class SeqSetC(C.Structure):
    _fields_ = [("n", C.c_uint64), ("seqs", C.POINTER(C.c_void_p)), ("names", C.POINTER(C.c_char_p))]


class TuningC(C.Structure):
    _fields_ = [("screen_warps", C.c_uint32), ("screen_cap", C.c_uint32), ("screen_blocks_per_sm", C.c_uint32),
                ("walk_warps", C.c_uint32), ("max_hits_per_pass", C.c_uint32), ("initial_candidates", C.c_uint32),
                ("filter_cap", C.c_uint32), ("filter_claim", C.c_uint32), ("gapped_pool_blocks", C.c_uint32),
                ("gapped_cells", C.c_uint32)]


class UnitC(C.Structure):
    _fields_ = [("table", C.c_uint32), ("query", C.c_uint32), ("strand", C.c_uint32), ("primary_lo", C.c_uint32),
                ("primary_hi", C.c_uint32)]


class BatchResultC(C.Structure):
    _fields_ = [("hsps", C.POINTER(HspC)), ("unit_offsets", C.POINTER(C.c_uint64)), ("n_hsps", C.c_uint64),
                ("n_units", C.c_uint32)]


class PlaceC(C.Structure):
    _fields_ = [("group", C.c_uint32), ("t_offset", C.c_uint32)]


class RecordResultC(C.Structure):
    _fields_ = [("records", C.c_void_p), ("group_offsets", C.POINTER(C.c_uint64)), ("n_records", C.c_uint64),
                ("n_groups", C.c_uint32)]


class BatchOptsC(C.Structure):
    _fields_ = [("use_graph", C.c_uint32), ("reserved_", C.c_uint32 * 7)]


class ServerOptsC(C.Structure):
    _fields_ = [("max_device_bytes", C.c_uint64), ("max_units", C.c_uint32), ("max_streams", C.c_uint32),
                ("max_batch_units", C.c_uint32), ("both_strands", C.c_uint32),
                ("max_batch_bases", C.c_uint64), ("big_bases", C.c_uint64), ("max_big_inflight", C.c_uint32),
                ("reserved_", C.c_uint32), ("warm_bases", C.c_uint64)]


class ServerStatsC(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("batches", C.c_uint64),
                ("max_inflight_units", C.c_uint64), ("bytes_in_use", C.c_uint64), ("reruns", C.c_uint64),
                ("busy_ms", C.c_double), ("failed", C.c_uint64), ("canceled", C.c_uint64),
                ("isolated", C.c_uint64), ("mem_refreshes", C.c_uint64)]


class GappedParamsC(C.Structure):
    _fields_ = [("gap_open", C.c_int32), ("gap_extend", C.c_int32), ("y_drop", C.c_int32),
                ("gapped_threshold", C.c_int32)]


class GappedAlnC(C.Structure):
    _fields_ = [("t_start", C.c_uint32), ("q_start", C.c_uint32), ("t_len", C.c_uint32), ("q_len", C.c_uint32),
                ("score", C.c_int32), ("passed", C.c_uint32), ("script_off", C.c_uint64),
                ("script_len", C.c_uint32), ("pad_", C.c_uint32)]


class GappedResultC(C.Structure):
    _fields_ = [("alns", C.POINTER(GappedAlnC)), ("runs", C.POINTER(C.c_uint32)), ("n_alns", C.c_uint64),
                ("n_runs", C.c_uint64)]


class GappedStatsC(C.Structure):
    _fields_ = [("rows", C.c_uint64), ("cells", C.c_uint64), ("device_ms", C.c_double), ("reruns", C.c_uint32),
                ("warps_per_side", C.c_uint32), ("max_side_rows", C.c_uint64),
                ("second_pass_sides", C.c_uint64), ("cells_per_thread", C.c_uint32), ("pad_", C.c_uint32),
                ("second_pass_cells", C.c_uint64)]


V = C.c_void_p
P = C.POINTER
U32, U64, I32, U8 = C.c_uint32, C.c_uint64, C.c_int32, C.c_uint8

# name -> (restype, argtypes)
SIGNATURES = {
    "gxy_status_string": (C.c_char_p, [C.c_int]),
    "gxy_last_error": (C.c_char_p, []),
    "gxy_abi_version": (U32, []),
    "gxy_kernel_launches": (U64, []),
    "gxy_ctx_create": (C.c_int, [C.c_int, P(V)]),
    "gxy_ctx_destroy": (C.c_int, [V]),
    "gxy_ctx_set_tuning": (C.c_int, [V, P(TuningC)]),
    "gxy_ctx_get_tuning": (C.c_int, [V, P(TuningC)]),
    "gxy_ctx_mark": (C.c_int, [V, U32]),
    "gxy_ctx_elapsed_ms": (C.c_int, [V, U32, U32, P(C.c_double)]),
    "gxy_dseq_upload": (C.c_int, [V, P(PackedSeqC), P(V)]),
    "gxy_dseq_from_ascii": (C.c_int, [V, V, U64, P(V)]),
    "gxy_dseq_reverse_complement": (C.c_int, [V, V, P(V)]),
    "gxy_dseq_download": (C.c_int, [V, V, V, V]),
    "gxy_dseq_len": (U64, [V]),
    "gxy_dseq_free": (C.c_int, [V]),
    "gxy_table_build": (C.c_int, [V, P(PackedSeqC), C.c_char_p, U32, U32, P(V)]),
    "gxy_table_build_view": (C.c_int, [V, V, U64, U64, C.c_char_p, U32, U32, P(V)]),
    "gxy_table_build_views": (C.c_int, [V, V, U32, V, V, C.c_char_p, U32, U32, V]),
    "gxy_table_prune_hot_words": (C.c_int, [V, U32]),
    "gxy_table_build_static": (C.c_int, [P(PackedSeqC), C.c_char_p, U32, V, U64, V, U64, P(U64)]),
    "gxy_table_info": (C.c_int, [V, P(U64), P(U64), P(U32), P(U32)]),
    "gxy_table_download": (C.c_int, [V, V, V]),
    "gxy_table_free": (C.c_int, [V]),
    "gxy_search": (C.c_int, [V, V, P(PackedSeqC), P(PackedSeqC), P(SearchParamsC), P(HspBufC), P(StatsC)]),
    "gxy_search_dseq": (C.c_int, [V, V, V, P(SearchParamsC), P(HspBufC), P(StatsC)]),
    "gxy_hsp_buf_free": (None, [P(HspBufC)]),
    "gxy_batch_search": (C.c_int, [V, U32, P(V), U32, P(V), U32, P(UnitC), P(SearchParamsC), P(BatchOptsC),
                                   P(BatchResultC), P(StatsC)]),
    "gxy_batch_result_free": (None, [P(BatchResultC)]),
    "gxy_batch_records": (C.c_int, [V, U32, P(V), U32, P(V), U32, P(UnitC), P(PlaceC), P(SearchParamsC),
                                    P(BatchOptsC), P(RecordResultC), P(StatsC)]),
    "gxy_record_result_free": (None, [P(RecordResultC)]),
    "gxy_chunk_plan": (C.c_int, [U64, U32, U32, P(U64), U64, P(U64)]),
    "gxy_extend_hits": (C.c_int, [V, V, V, P(SearchParamsC), U64, V, V, U32, U32, V, V]),
    "gxy_server_create": (C.c_int, [V, U32, P(V), P(SearchParamsC), P(ServerOptsC), P(V)]),
    "gxy_server_submit": (C.c_int, [V, U32, P(PackedSeqC), P(U64)]),
    "gxy_server_wait": (C.c_int, [V, U64, U32, P(HspBufC), P(HspBufC), P(C.c_double)]),
    "gxy_server_get_stats": (C.c_int, [V, P(ServerStatsC)]),
    "gxy_server_destroy": (C.c_int, [V]),
    "gxy_server_cancel": (C.c_int, [V, U64]),
    "gxy_server_inject_fault": (C.c_int, [V, U64, C.c_int]),
    "gxy_choose_anchors": (C.c_int, [V, V, V, P(SearchParamsC), V, U64, U32, V, V]),
    "gxy_best_chain": (C.c_int, [V, U64, V, P(C.c_uint64)]),
    "gxy_best_chain_groups": (C.c_int, [V, V, V, U32, V, V]),
    "gxy_gapped_extend": (C.c_int, [V, V, U64, U64, V, P(SearchParamsC), P(GappedParamsC), V, V, U64,
                                    P(GappedResultC), P(GappedStatsC)]),
    "gxy_gapped_result_free": (None, [P(GappedResultC)]),
    "gxy_parse_fasta": (C.c_int, [V, V, U64, P(SeqSetC)]),
    "gxy_parse_2bit": (C.c_int, [V, V, U64, P(SeqSetC)]),
    "gxy_seq_set_free": (None, [P(SeqSetC)]),
}

_lib = None


def build() -> str:
    """Compiles libgxyseed.so for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(_HERE, "csrc")], check=True)
    return LIB_PATH


def lib():
    """Loads libgxyseed.so; raises when it was not built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with lastz_gxy_b200.build() (make -C csrc)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != GXY_OK:
        msg = lib().gxy_last_error()
        raise GxyError(status, msg.decode() if msg else "")
