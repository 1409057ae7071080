"""Amethyst operator layer, rebuilt B200-native: packed-integer operators (filter, compressstore,
binary ops, aggregation, group-by, matrix multiply) over plain, slab and nogaps columns, as
hand-written sm_100a CUDA kernels behind the C ABI in include/amethyst.h.

The C ABI is the product; this package is its Python host mirror.  Importing `ops` loads
libamethyst_b200.so and fails loudly when it is missing.
"""
from . import _capi  # noqa: F401
from ._capi import (AGG_AND, AGG_MAX, AGG_MIN, AGG_OR, AGG_SUM, AGG_XOR, NOGAPS, OP_ADD, OP_AND,  # noqa: F401
                    OP_BOOL_OR, OP_BOOL_XOR, OP_DIV, OP_LHS, OP_MATH, OP_MAX, OP_MIN, OP_MOD, OP_MUL, OP_OR,
                    OP_SUB, OP_XOR, PLAIN32, PLAIN64, PRED_ALL, PRED_BETWEEN, PRED_EQ, PRED_GE, PRED_GT,
                    PRED_HALF, PRED_LE, PRED_LT, PRED_NE, PRED_NOT_BETWEEN, SLAB, AmxError)

__all__ = ["ops", "build"]
