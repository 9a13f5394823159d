"""ctypes binding of librnjgpu.so (the C ABI declared in include/rnj.h).

The shared library is built in-tree (``rapidnj_b200/librnjgpu.so``, see
``rapidnj_b200/build.py``).  There is no fallback: if the library is missing
or does not load, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librnjgpu.so")

RNJ_OK = 0
RNJ_DNA, RNJ_PROTEIN, RNJ_UNKNOWN = 0, 1, 2
RNJ_JC, RNJ_KIMURA = 0, 1
RNJ_FASTDIST, RNJ_COMPAT_PROTEIN_WRAP, RNJ_FULL_ROWS, RNJ_POPCOUNT = 1, 2, 4, 8
(RNJ_ERR_INVALID, RNJ_ERR_CUDA, RNJ_ERR_NOMEM, RNJ_ERR_IO, RNJ_ERR_FORMAT, RNJ_ERR_TIMEOUT,
 RNJ_ERR_BUSY, RNJ_ERR_UNSUPPORTED, RNJ_ERR_NOTREADY) = range(1, 10)

STATUS_NAMES = {
    0: "RNJ_OK", 1: "RNJ_ERR_INVALID", 2: "RNJ_ERR_CUDA", 3: "RNJ_ERR_NOMEM", 4: "RNJ_ERR_IO",
    5: "RNJ_ERR_FORMAT", 6: "RNJ_ERR_TIMEOUT", 7: "RNJ_ERR_BUSY", 8: "RNJ_ERR_UNSUPPORTED",
    9: "RNJ_ERR_NOTREADY",
}


class RnjError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None

c_int, c_size_t, c_float, c_void_p, c_char_p = (ctypes.c_int, ctypes.c_size_t, ctypes.c_float,
                                                 ctypes.c_void_p, ctypes.c_char_p)
P = ctypes.POINTER

# name -> (restype, argtypes)
SIGNATURES = {
    "rnj_version": (c_char_p, []),
    "rnj_last_error": (c_char_p, []),
    "rnj_ctx_create": (c_int, [c_int, P(c_void_p)]),
    "rnj_ctx_destroy": (c_int, [c_void_p]),
    "rnj_ctx_stream": (c_int, [c_void_p, P(c_void_p)]),
    "rnj_ctx_synchronize": (c_int, [c_void_p]),
    "rnj_set_wait_limit": (c_int, [ctypes.c_uint]),
    "rnj_ctx_memory": (c_int, [c_void_p, P(c_size_t), P(c_size_t)]),
    "rnj_distance_rows": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                  P(c_float), P(c_int)]),
    "rnj_test_wait_on_unset_flag": (c_int, [c_int]),
    "rnj_detect_type": (c_int, [c_char_p, c_int]),
    "rnj_ctx_set_profiling": (c_int, [c_void_p, c_int]),
    "rnj_ctx_stage_times": (c_int, [c_void_p, P(c_float)]),
    "rnj_probe_int_peaks": (c_int, [c_void_p, P(ctypes.c_double), P(ctypes.c_double)]),
    "rnj_probe_tc_peak": (c_int, [c_void_p, P(ctypes.c_double)]),
    "rnj_check_quotient16": (c_int, [c_void_p, P(ctypes.c_ulonglong)]),
    "rnj_aln_from_host": (c_int, [c_void_p, P(c_char_p), c_int, c_int, c_int, c_int, P(c_void_p)]),
    "rnj_aln_from_host_buffer": (c_int, [c_void_p, c_void_p, c_int, c_int, c_size_t, c_int, c_int,
                                         P(c_void_p)]),
    "rnj_aln_from_device": (c_int, [c_void_p, c_void_p, c_int, c_int, c_size_t, c_int, c_int,
                                    P(c_void_p)]),
    "rnj_aln_from_bitstrings": (c_int, [c_void_p, P(c_void_p), P(c_void_p), c_int, c_int, c_int,
                                        c_int, c_int, P(c_void_p)]),
    "rnj_aln_info": (c_int, [c_void_p, P(c_int), P(c_int), P(c_int)]),
    "rnj_aln_destroy": (c_int, [c_void_p]),
    "rnj_distance": (c_int, [c_void_p, c_void_p, c_int, P(c_void_p)]),
    "rnj_distance_into": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_size_t, P(c_float)]),
    "rnj_counts_into": (c_int, [c_void_p, c_void_p, c_void_p]),
    "rnj_mat_info": (c_int, [c_void_p, P(c_int), P(c_float)]),
    "rnj_mat_device_ptr": (c_int, [c_void_p, P(c_void_p), P(c_size_t)]),
    "rnj_mat_copy_rows": (c_int, [c_void_p, c_void_p, c_int, c_int, P(c_void_p), c_int]),
    "rnj_mat_destroy": (c_int, [c_void_p]),
    "rnj_distance_matrix_host": (c_int, [c_void_p, c_void_p, c_int, c_int, c_size_t, c_int, c_int,
                                         c_int, c_void_p, P(c_float)]),
    "rnj_distance_matrix_host_ex": (c_int, [c_void_p, c_void_p, c_int, c_int, c_size_t, c_int,
                                            c_int, c_int, c_int, c_void_p, P(c_float)]),
    "rnj_tune": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p]),
    "rnj_bootstrap": (c_int, [c_void_p, c_void_p, c_int, c_int, c_size_t, c_int, c_int, c_int,
                              c_int, c_void_p, c_void_p, c_size_t, c_void_p]),
    "rnj_tune_get": (c_int, [c_int, c_int, c_int, c_int, c_void_p]),
    "rnj_tune_set": (c_int, [c_int, c_int, c_int, c_int, c_void_p]),
    "rnj_tune_clear": (c_int, []),
    "rnj_tune_save": (c_int, [c_char_p]),
    "rnj_tune_load": (c_int, [c_char_p]),
    "rnj_distance_noalloc": (c_int, [c_void_p, c_int, c_int, c_size_t, c_int, c_int, c_int,
                                     c_void_p, c_size_t, c_void_p, P(c_float)]),
    "rnj_batch_create": (c_int, [c_void_p, c_int, ctypes.c_longlong, P(c_void_p)]),
    "rnj_batch_add": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_size_t, P(c_int)]),
    "rnj_batch_add_many": (c_int, [c_void_p, c_int, P(c_void_p), P(c_int), P(c_int), P(c_size_t),
                                   P(c_int), P(c_int), c_int, P(c_void_p), P(c_size_t), P(c_int)]),
    "rnj_batch_run": (c_int, [c_void_p]),
    "rnj_batch_synchronize": (c_int, [c_void_p]),
    "rnj_batch_output": (c_int, [c_void_p, c_int, P(c_void_p), P(c_size_t), P(c_float)]),
    "rnj_batch_take": (c_int, [c_void_p, c_int, P(c_void_p)]),
    "rnj_batch_size": (c_int, [c_void_p, P(c_int), P(ctypes.c_longlong)]),
    "rnj_batch_tuning": (c_int, [c_void_p, P(c_int), P(c_int)]),
    "rnj_distance_f64": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_size_t,
                                 P(ctypes.c_double)]),
    "rnj_batch_clear": (c_int, [c_void_p]),
    "rnj_batch_destroy": (c_int, [c_void_p]),
    "rnj_batch_poll": (c_int, [c_void_p, P(c_int)]),
    "rnj_server_create": (c_int, [c_int, c_size_t, c_int, P(c_void_p)]),
    "rnj_server_submit": (c_int, [c_void_p, c_void_p, c_int, c_int, c_size_t, c_int, c_int, c_int,
                                  P(ctypes.c_uint64)]),
    "rnj_server_poll": (c_int, [c_void_p, ctypes.c_uint64, P(c_int)]),
    "rnj_server_wait": (c_int, [c_void_p, ctypes.c_uint64, c_int]),
    "rnj_server_result": (c_int, [c_void_p, ctypes.c_uint64, c_void_p, P(c_void_p),
                                  P(ctypes.c_double)]),
    "rnj_server_stats": (c_int, [c_void_p, P(ctypes.c_uint64), P(ctypes.c_double),
                                 P(ctypes.c_double), P(c_size_t)]),
    "rnj_server_destroy": (c_int, [c_void_p]),
    "rnj_shard_tiles": (c_int, [c_int, c_int, c_int, c_int, P(ctypes.c_longlong),
                                P(ctypes.c_longlong), P(ctypes.c_longlong)]),
    "rnj_tile_coords": (c_int, [c_int, c_int, ctypes.c_longlong, P(c_int), P(c_int)]),
    "rnj_shard_create": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_size_t,
                                 P(c_void_p)]),
    "rnj_shard_run": (c_int, [c_void_p, P(c_float)]),
    "rnj_shard_finish": (c_int, [c_void_p, c_float]),
    "rnj_shard_output": (c_int, [c_void_p, P(c_void_p), P(c_size_t)]),
    "rnj_shard_copy_tiles": (c_int, [c_void_p, c_void_p, c_size_t, P(c_size_t)]),
    "rnj_shard_destroy": (c_int, [c_void_p]),
    "rnj_msa_read": (c_int, [c_char_p, c_char_p, P(c_void_p)]),
    "rnj_msa_info": (c_int, [c_void_p, P(c_int), P(c_int), P(c_int)]),
    "rnj_msa_name": (c_char_p, [c_void_p, c_int]),
    "rnj_msa_chars": (c_void_p, [c_void_p]),
    "rnj_msa_destroy": (c_int, [c_void_p]),
    "rnj_msa_read_device": (c_int, [c_void_p, c_char_p, c_char_p, P(c_void_p)]),
    "rnj_msa_device_chars": (c_int, [c_void_p, P(c_void_p), P(c_size_t)]),
    "rnj_write_matrix_text": (c_int, [c_char_p, P(c_char_p), P(c_void_p), c_int, c_int]),
    "rnj_nj_init": (c_int, [c_void_p, c_void_p, c_int, c_size_t, c_void_p]),
    "rnj_write_matrix_text_device": (c_int, [c_void_p, c_char_p, P(c_char_p), c_void_p, c_size_t,
                                             c_int]),
}


# rnj_rows_fn: int (*)(void *user, int row0, int nrows, const float *rows, size_t ld)
ROWS_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_int, c_int, P(c_float), c_size_t)


class NjData(ctypes.Structure):
    """rnj_nj_data (include/rnj.h): output pointers of rnj_nj_init."""
    _fields_ = [("separation_sums", c_void_p), ("separations", c_void_p),
                ("max_row_separations", c_void_p), ("max_separation", c_void_p),
                ("possible_redundant", c_void_p), ("index_to_id", c_void_p),
                ("redundant_to_master", c_void_p), ("redundant_count", c_void_p),
                ("sorted", c_void_p), ("sorted_ld", c_size_t), ("sorted_cap", c_int),
                ("row_lengths", c_void_p)]


def lib():
    """The loaded library; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RnjError(8, f"{LIB_PATH} is not built; run rapidnj_b200.build.build()")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != RNJ_OK:
        msg = lib().rnj_last_error()
        raise RnjError(status, msg.decode(errors="replace") if msg else "")
