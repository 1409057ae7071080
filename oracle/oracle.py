"""ctypes wrapper of the C oracle (amx_oracle.c) and of the reference's own code built into
oracle/_ref/.  TEST INFRASTRUCTURE ONLY (see oracle/__init__.py)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_HOST_SO = os.path.join(HERE, "_ref", "libamxref_host.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libamxref_gpu.so")
REF_ROOT = os.environ.get("AMX_REFERENCE_ROOT", "/root/reference")

PLAIN32, PLAIN64, SLAB, NOGAPS = 0, 1, 2, 3


class OraColumn(C.Structure):
    _fields_ = [("data", C.c_void_p), ("n", C.c_uint64), ("format", C.c_uint32), ("bits", C.c_uint32)]


class OraPred(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("bits", C.c_uint32), ("k0", C.c_uint64), ("k1", C.c_uint64)]


class OraChainResult(C.Structure):
    _fields_ = [("count", C.c_uint64), ("agg", C.c_uint64)]


def build(with_reference: bool = True) -> None:
    """Build liboracle.so (gcc) and, when the reference tree is present, oracle/_ref/."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    if with_reference and os.path.isdir(os.path.join(REF_ROOT, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_ROOT={REF_ROOT}"], check=True)


_ora = None


def ora():
    global _ora
    if _ora is None:
        if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(
                os.path.join(HERE, "amx_oracle.c")):
            build(with_reference=False)
        h = C.CDLL(ORACLE_SO)
        P, U64, U32 = C.c_void_p, C.c_uint64, C.c_uint32
        col, pred = C.POINTER(OraColumn), C.POINTER(OraPred)
        sig = {
            "ora_storage_bytes": (U64, [U32, U32, U64]),
            "ora_encode": (None, [U32, U32, P, U64, P]),
            "ora_decode": (None, [col, P]),
            "ora_filter": (None, [col, pred, P]),
            "ora_compressstore": (U64, [col, P, col]),
            "ora_filter_compressstore": (U64, [col, pred, col]),
            "ora_binary": (None, [U32, col, col, col]),
            "ora_binop": (U64, [U32, U64, U64, U32]),
            "ora_binop_out_bits": (U32, [U32, U32, U32]),
            "ora_reduce": (U64, [U32, col, P]),
            "ora_chain": (OraChainResult, [U32, col, col, U32, pred, U32, col]),
            "ora_chain_mt": (OraChainResult, [U32, col, col, U32, pred, U32, C.c_int]),
            "ora_chain_compress_mt": (OraChainResult, [U32, col, col, U32, pred, U32, col, C.c_int]),
            "ora_groupby_dense": (U64, [col, col, P, P]),
            "ora_groupby_sorted": (U64, [col, col, P, P, P, P]),
            "ora_matmul": (None, [col, col, U64, U64, U64, P, C.c_int]),
            "ora_matrix_words": (U64, [U32, U32, U64, U64]),
            "ora_matrix_encode": (None, [U32, U32, P, U64, U64, P]),
            "ora_pcg32_seed": (None, [P, U64]),
            "ora_pcg32_next": (U32, [P]),
            "ora_reference_inputs": (None, [U64, P, P, U64]),
            "ora_mask_uniform": (None, [P, U64, U64, C.c_double]),
            "ora_mask_clusters": (None, [P, C.c_double, U64, U64]),
            "ora_uniform_values": (None, [U64, U32, P, U64]),
            "ora_pred_eval": (C.c_int, [pred, U64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _ora = h
    return _ora


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def storage_bytes(fmt, bits, n):
    return int(ora().ora_storage_bytes(fmt, bits, n))


def _buf(fmt, bits, n):
    return np.zeros(max(16, storage_bytes(fmt, bits, n) + 16), dtype=np.uint8)


def column(raw: np.ndarray, n: int, fmt: int, bits: int) -> OraColumn:
    return OraColumn(raw.ctypes.data, n, fmt, bits)


def encode(fmt: int, bits: int, values: np.ndarray) -> np.ndarray:
    values = np.ascontiguousarray(values, dtype=np.uint64)
    out = _buf(fmt, bits, len(values))
    ora().ora_encode(fmt, bits, _p(values), len(values), _p(out))
    return out


def decode(raw: np.ndarray, n: int, fmt: int, bits: int) -> np.ndarray:
    out = np.zeros(max(n, 1), dtype=np.uint64)
    c = column(raw, n, fmt, bits)
    ora().ora_decode(C.byref(c), _p(out))
    return out[:n]


def pred(kind, k0=0, k1=0, bits=0):
    return OraPred(kind, bits, k0, k1)


def filter(raw, n, fmt, bits, p) -> np.ndarray:
    mask = np.zeros((n + 31) // 32 + 4, dtype=np.uint32)
    ora().ora_filter(C.byref(column(raw, n, fmt, bits)), C.byref(p), _p(mask))
    return mask[: (n + 31) // 32]


def compressstore(raw, n, fmt, bits, mask, out_fmt, out_bits):
    out = _buf(out_fmt, out_bits, n)
    oc = column(out, n, out_fmt, out_bits)
    m = np.ascontiguousarray(mask, dtype=np.uint32)
    cnt = ora().ora_compressstore(C.byref(column(raw, n, fmt, bits)), _p(m), C.byref(oc))
    return out[: storage_bytes(out_fmt, out_bits, cnt)], int(cnt)


def filter_compressstore(raw, n, fmt, bits, p, out_fmt, out_bits):
    out = _buf(out_fmt, out_bits, n)
    oc = column(out, n, out_fmt, out_bits)
    cnt = ora().ora_filter_compressstore(C.byref(column(raw, n, fmt, bits)), C.byref(p), C.byref(oc))
    return out[: storage_bytes(out_fmt, out_bits, cnt)], int(cnt)


def binary(op, lraw, lfmt, lbits, rraw, rfmt, rbits, n, out_fmt, out_bits):
    out = _buf(out_fmt, out_bits, n)
    ora().ora_binary(op, C.byref(column(lraw, n, lfmt, lbits)), C.byref(column(rraw, n, rfmt, rbits)),
                     C.byref(column(out, n, out_fmt, out_bits)))
    return out[: storage_bytes(out_fmt, out_bits, n)]


def reduce(agg, raw, n, fmt, bits, mask=None) -> int:
    m = np.ascontiguousarray(mask, dtype=np.uint32) if mask is not None else None
    return int(ora().ora_reduce(agg, C.byref(column(raw, n, fmt, bits)), _p(m)))


def chain(op, lcol, rcol, vbits, p, agg, out_fmt=None, out_bits=None, n=None):
    """lcol/rcol: (raw, fmt, bits) tuples; returns (out bytes or None, count, agg)."""
    lc = column(lcol[0], n, lcol[1], lcol[2])
    rc = column(rcol[0], n, rcol[1], rcol[2]) if rcol is not None else None
    out = None
    oc = None
    if out_fmt is not None:
        out = _buf(out_fmt, out_bits, n)
        oc = column(out, n, out_fmt, out_bits)
    res = ora().ora_chain(op, C.byref(lc), C.byref(rc) if rc is not None else None, vbits, C.byref(p), agg,
                          C.byref(oc) if oc is not None else None)
    if out is not None:
        out = out[: storage_bytes(out_fmt, out_bits, res.count)]
    return out, int(res.count), int(res.agg)


def chain_mt(op, lcol, rcol, vbits, p, agg, n, threads):
    lc = column(lcol[0], n, lcol[1], lcol[2])
    rc = column(rcol[0], n, rcol[1], rcol[2]) if rcol is not None else None
    res = ora().ora_chain_mt(op, C.byref(lc), C.byref(rc) if rc is not None else None, vbits, C.byref(p), agg,
                             threads)
    return int(res.count), int(res.agg)


def chain_compress_mt(op, lcol, rcol, vbits, p, agg, out_fmt, out_bits, n, threads):
    """chain_mt that also compacts the survivors into out_fmt / out_bits: (out bytes, count, agg)."""
    lc = column(lcol[0], n, lcol[1], lcol[2])
    rc = column(rcol[0], n, rcol[1], rcol[2]) if rcol is not None else None
    out = _buf(out_fmt, out_bits, n)
    oc = column(out, n, out_fmt, out_bits)
    res = ora().ora_chain_compress_mt(op, C.byref(lc), C.byref(rc) if rc is not None else None, vbits, C.byref(p),
                                      agg, C.byref(oc), threads)
    return out[: storage_bytes(out_fmt, out_bits, res.count)], int(res.count), int(res.agg)


def groupby_dense(kraw, kfmt, kbits, vraw, vfmt, vbits, n):
    space = 1 << kbits
    sums = np.zeros(space, dtype=np.uint64)
    counts = np.zeros(space, dtype=np.uint64)
    g = ora().ora_groupby_dense(C.byref(column(kraw, n, kfmt, kbits)), C.byref(column(vraw, n, vfmt, vbits)),
                                _p(sums), _p(counts))
    return int(g), sums, counts


def groupby_sorted(kraw, kfmt, kbits, vraw, vfmt, vbits, n, mask=None):
    """(groups, ascending keys, uint64 sums, uint64 counts) of the masked elements, any key width."""
    ok = np.zeros(max(n, 1), dtype=np.uint64)
    os_ = np.zeros(max(n, 1), dtype=np.uint64)
    oc = np.zeros(max(n, 1), dtype=np.uint64)
    m = np.ascontiguousarray(mask, dtype=np.uint32) if mask is not None else None
    g = ora().ora_groupby_sorted(C.byref(column(kraw, n, kfmt, kbits)), C.byref(column(vraw, n, vfmt, vbits)), _p(m),
                                 _p(ok), _p(os_), _p(oc))
    return int(g), ok[:g], os_[:g], oc[:g]


def matrix_encode(fmt, bits, values: np.ndarray, rows, cols) -> np.ndarray:
    values = np.ascontiguousarray(values, dtype=np.uint64)
    words = int(ora().ora_matrix_words(fmt, bits, rows, cols))
    out = np.zeros(max(16, words * (4 if fmt == PLAIN32 else 8) + 16), dtype=np.uint8)
    ora().ora_matrix_encode(fmt, bits, _p(values), rows, cols, _p(out))
    return out


def matmul(araw, afmt, abits, braw, bfmt, bbits, m, n, k, threads=1) -> np.ndarray:
    out = np.zeros(m * n, dtype=np.int64)
    ora().ora_matmul(C.byref(column(araw, m * k, afmt, abits)), C.byref(column(braw, k * n, bfmt, bbits)), m, n, k,
                     _p(out), threads)
    return out.reshape(m, n)


def uniform_values(seed: int, bits: int, n: int) -> np.ndarray:
    out = np.zeros(max(n, 1), dtype=np.uint64)
    ora().ora_uniform_values(seed, bits, _p(out), n)
    return out[:n]


def reference_inputs(seed: int, n: int):
    d1 = np.zeros(n, dtype=np.uint64)
    d2 = np.zeros(n, dtype=np.uint64)
    ora().ora_reference_inputs(seed, _p(d1), _p(d2), n)
    return d1, d2


def mask_uniform(nbytes: int, selectivity: float) -> np.ndarray:
    out = np.zeros(nbytes, dtype=np.uint8)
    ora().ora_mask_uniform(_p(out), 0, nbytes, selectivity)
    return out


def mask_clusters(selectivity: float, clusters: int, total: int) -> np.ndarray:
    out = np.zeros(max(1, total // 8), dtype=np.uint8)
    ora().ora_mask_clusters(_p(out), selectivity, clusters, total)
    return out[: total // 8]


def pcg32(seed: int, count: int) -> np.ndarray:
    state = np.zeros(2, dtype=np.uint64)
    ora().ora_pcg32_seed(_p(state), seed)
    return np.array([ora().ora_pcg32_next(_p(state)) for _ in range(count)], dtype=np.uint32)


# ---- the reference's own code (oracle/_ref) ---------------------------------------------------
_ref_host = None
_ref_gpu = None


def ref_host():
    """The reference's host code (accessors, operators, main()); None if it was not built."""
    global _ref_host
    if _ref_host is None and os.path.exists(REF_HOST_SO):
        h = C.CDLL(REF_HOST_SO)
        P, U64 = C.c_void_p, C.c_uint64
        for name, res, args in [
            ("amxref_get_element", U64, [C.c_int, P, U64]),
            ("amxref_get_element_baseline", U64, [C.c_int, P, U64]),
            ("amxref_get_elem_nogaps", U64, [C.c_int, P, U64]),
            ("amxref_get_bitmask_element", C.c_int, [P, U64]),
            ("amxref_filter_predicate", C.c_int, [C.c_int, U64]),
            ("amxref_binary_op_default", U64, [C.c_int, U64, U64]),
            ("amxref_binary_op_outbits", C.c_int, [C.c_int]),
            ("amxref_op_add_outbits", C.c_int, [C.c_int]),
            ("amxref_op_mul_outbits", C.c_int, [C.c_int]),
            ("amxref_op_mod_outbits", C.c_int, [C.c_int]),
            ("amxref_op", U64, [C.c_int, C.c_int, U64, U64]),
            ("amxref_prng", None, [U64, P, U64]),
            ("amxref_run_main", C.c_int, [C.c_int, C.POINTER(C.c_char_p), P, P, U64]),
        ]:
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _ref_host = h
    return _ref_host


def ref_gpu():
    """The reference's kernels compiled for sm_100a; None if they were not built."""
    global _ref_gpu
    if _ref_gpu is None and os.path.exists(REF_GPU_SO):
        h = C.CDLL(REF_GPU_SO)
        P, U64, I = C.c_void_p, C.c_uint64, C.c_int
        for name, args in [
            ("amxref_gpu_filter_slabs", [I, I, P, U64, P, I]),
            ("amxref_gpu_filter_nogaps", [I, I, P, U64, P, I]),
            ("amxref_gpu_filter_baseline", [I, I, P, U64, P, I]),
            ("amxref_gpu_compressstore_slabs", [I, P, P, P, U64, P, I]),
            ("amxref_gpu_compressstore_cub", [P, P, P, U64, P]),
            ("amxref_gpu_binary_op_slabs", [I, I, P, P, P, U64, I]),
            ("amxref_gpu_binary_op_nogaps", [I, I, P, P, P, U64, I]),
            ("amxref_gpu_binary_op_baseline", [I, I, P, P, P, U64, I]),
            ("amxref_gpu_hop_slabs", [I, P, U64, P, I]),
            ("amxref_gpu_hop_nogaps", [I, P, U64, P, I]),
            ("amxref_gpu_hop_cub", [P, U64, P]),
            ("amxref_gpu_groupby_sm_array", [I, P, P, P, P, U64, P, I]),
        ]:
            f = getattr(h, name)
            f.restype = C.c_int
            f.argtypes = args
        _ref_gpu = h
    return _ref_gpu


def run_reference_main(args, n):
    h = ref_host()
    d1 = np.zeros(n, dtype=np.uint64)
    d2 = np.zeros(n, dtype=np.uint64)
    arr = (C.c_char_p * len(args))(*[a.encode() for a in args])
    ok = h.amxref_run_main(len(args), arr, _p(d1), _p(d2), n)
    return ok, d1, d2
