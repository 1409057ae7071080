"""ctypes view of the C ABI declared in include/amethyst.h.

The shared library is built in-tree (amethyst_b200/libamethyst_b200.so, see build.py).  There
is no fallback: if the library is missing or fails to load, importing the operators raises.
"""
from __future__ import annotations

import ctypes as C
import os

PLAIN32, PLAIN64, SLAB, NOGAPS = 0, 1, 2, 3
FORMAT_NAMES = {PLAIN32: "plain32", PLAIN64: "plain64", SLAB: "slab", NOGAPS: "nogaps"}

(PRED_ALL, PRED_LT, PRED_LE, PRED_GT, PRED_GE, PRED_EQ, PRED_NE, PRED_BETWEEN, PRED_NOT_BETWEEN,
 PRED_HALF) = range(10)

(OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MOD, OP_MIN, OP_MAX, OP_AND, OP_OR, OP_XOR, OP_BOOL_OR,
 OP_BOOL_XOR, OP_MATH, OP_LHS) = range(14)

AGG_SUM, AGG_MIN, AGG_MAX, AGG_AND, AGG_OR, AGG_XOR = range(6)

STATUS = {
    0: "ok", 1: "invalid argument", 2: "unsupported", 3: "misaligned pointer",
    4: "workspace too small", 5: "CUDA error", 6: "device-side wait timed out",
    7: "size exceeds capacity",
}


class Column(C.Structure):
    _fields_ = [("data", C.c_void_p), ("n", C.c_uint64), ("format", C.c_uint32), ("bits", C.c_uint32)]


class Predicate(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("bits", C.c_uint32), ("k0", C.c_uint64), ("k1", C.c_uint64)]


class ChainDesc(C.Structure):
    _fields_ = [("op", C.c_uint32), ("value_bits", C.c_uint32), ("pred", Predicate),
                ("agg", C.c_uint32), ("reserved", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("staged_bytes", C.c_uint32), ("compact_stages", C.c_uint32), ("policy", C.c_int32),
                ("max_ctas", C.c_uint32)]


class BatchTuning(C.Structure):
    _fields_ = [("threads", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("words_per_thread", C.c_uint32),
                ("reserved", C.c_uint32)]


class BatchPlan(C.Structure):
    _fields_ = [("ncols", C.c_uint32), ("threads", C.c_uint32), ("grid", C.c_uint32), ("reserved", C.c_uint32),
                ("items", C.c_uint64), ("workspace_bytes", C.c_uint64)]


STEP_FILTER, STEP_COMPRESSSTORE, STEP_BINARY, STEP_REDUCE, STEP_GROUPBY = range(5)
FORMAT_FUSED = 0xFF
PROGRAM_MAX_STEPS = 32


class Step(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("op", C.c_uint32), ("value_bits", C.c_uint32), ("out_format", C.c_uint32),
                ("out_bits", C.c_uint32), ("reserved", C.c_uint32), ("pred", Predicate), ("aux", Column),
                ("d_result", C.c_void_p), ("group_keys", Column), ("group_sums", Column),
                ("group_counts", Column)]


LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libamethyst_b200.so")

_P = C.c_void_p
_COL = C.POINTER(Column)
_SIGS = {
    "amx_version": (C.c_int, []),
    "amx_status_string": (C.c_char_p, [C.c_int]),
    "amx_last_error": (C.c_char_p, []),
    "amx_storage_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint64]),
    "amx_mask_bytes": (C.c_uint64, [C.c_uint64]),
    "amx_binary_out_bits": (C.c_uint32, [C.c_uint32, C.c_uint32, C.c_uint32]),
    "amx_workspace_bytes": (C.c_uint64, [C.c_uint64]),
    "amx_workspace_status": (C.c_int, [_P, _P]),
    "amx_set_tuning": (C.c_int, [C.POINTER(Tuning)]),
    "amx_get_tuning": (C.c_int, [C.POINTER(Tuning)]),
    "amx_test_lookback_timeout": (C.c_int, [C.c_uint64, C.c_uint32]),
    "amx_filter": (C.c_int, [_COL, C.POINTER(Predicate), _P, _P, C.c_size_t, _P]),
    "amx_compressstore": (C.c_int, [_COL, _P, _COL, _P, _P, C.c_size_t, _P]),
    "amx_filter_compressstore": (C.c_int, [_COL, C.POINTER(Predicate), _COL, _P, _P, C.c_size_t, _P]),
    "amx_binary": (C.c_int, [C.c_uint32, _COL, _COL, _COL, _P, C.c_size_t, _P]),
    "amx_convert": (C.c_int, [_COL, _COL, _P, C.c_size_t, _P]),
    "amx_reduce": (C.c_int, [C.c_uint32, _COL, _P, _P, _P, C.c_size_t, _P]),
    "amx_chain": (C.c_int, [C.POINTER(ChainDesc), _COL, _COL, _COL, _P, _P, _P, _P, C.c_size_t, _P]),
    "amx_groupby_workspace_bytes": (C.c_uint64, [C.c_uint32]),
    "amx_groupby_wide_workspace_bytes": (C.c_uint64, [C.c_uint32, C.c_uint64]),
    "amx_groupby_status": (C.c_int, [_P, C.c_uint32, _P]),
    "amx_groupby": (C.c_int, [_COL, _COL, _P, _COL, _COL, _COL, _P, _P, C.c_size_t, _P]),
    "amx_groupby_sort_workspace_bytes": (C.c_uint64, [C.c_uint64, C.c_uint32, C.c_uint32]),
    "amx_groupby_sort": (C.c_int, [_COL, _COL, _P, _COL, _COL, _COL, _P, _P, C.c_size_t, _P]),
    "amx_groupby_sort_status": (C.c_int, [_P, _P]),
    "amx_matmul_workspace_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint32]),
    "amx_matmul_out_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                          C.c_uint32]),
    "amx_matmul": (C.c_int, [_COL, _COL, C.c_uint32, C.c_uint32, C.c_uint32, _COL, _P, _P, C.c_size_t, _P]),
    "amx_matmul_status": (C.c_int, [_P, _P]),
    "amx_batch_workspace_bytes": (C.c_uint64, [_COL, C.c_uint32, C.POINTER(BatchTuning)]),
    "amx_batch_prepare": (C.c_int, [_COL, C.POINTER(Predicate), _COL, C.c_uint32, C.POINTER(BatchTuning),
                                    C.POINTER(BatchPlan), _P, C.c_size_t, _P]),
    "amx_batch_run": (C.c_int, [C.POINTER(BatchPlan), _P, _P, _P, C.c_size_t, _P]),
    "amx_batch_status": (C.c_int, [_P, _P]),
    "amx_mlp_param_count": (C.c_uint32, [C.c_uint32]),
    "amx_mlp_forward": (C.c_int, [_P, C.c_uint32, _P, C.c_uint32, _P, _P]),
    "amx_mlp_train_step": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, _P, _P, C.c_uint32, C.c_float, _P, _P]),
    "amx_program_create": (C.c_int, [_COL, C.POINTER(Step), C.c_uint32, C.POINTER(C.c_void_p)]),
    "amx_program_workspace_bytes": (C.c_uint64, [_P]),
    "amx_program_run": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "amx_program_output": (C.c_int, [_P, _P, _COL, C.POINTER(C.c_void_p)]),
    "amx_program_status": (C.c_int, [_P, _P, _P]),
    "amx_program_destroy": (None, [_P]),
    "amx_graph_capture": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_uint64), C.c_uint32,
                                    C.c_uint32, C.POINTER(C.c_void_p)]),
    "amx_graph_launch": (C.c_int, [_P, _P]),
    "amx_graph_destroy": (None, [_P]),
    "amx_bit_histogram": (C.c_int, [_COL, _P, _P]),
    "amx_fill_uniform": (C.c_int, [_P, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, _P]),
    "amx_fill_from_cdf": (C.c_int, [_P, C.c_uint64, _P, C.c_uint32, C.c_uint64, _P]),
}

_lib = None


class AmxError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def lib():
    """Load libamethyst_b200.so once; raise if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run amethyst_b200.build.build() first")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise AmxError(status, lib().amx_last_error().decode())
