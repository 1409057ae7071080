"""Python host mirror of the Amethyst operator layer, on top of the C ABI.

Device buffers are torch tensors (torch is used for device memory and streams only); every
operator call goes through libamethyst_b200.so.  These helpers allocate their outputs and
workspaces with torch, which the C ABI itself never does.

The operator names follow the reference's kernels and launchers (src/lib.cuh:4-46,
src/kernels/*.cuh): filter, compressstore, binary_op, hop (= reduce), groupby, matmul.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import torch

from . import _capi as A
from ._capi import check, lib


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def storage_bytes(fmt: int, bits: int, n: int) -> int:
    return int(lib().amx_storage_bytes(fmt, bits, n))


def alloc_bytes(nbytes: int, device="cuda") -> torch.Tensor:
    """A 16-byte-padded device byte buffer (torch allocations are 512-byte aligned)."""
    return torch.zeros(max(16, (nbytes + 15) // 16 * 16 + 16), dtype=torch.uint8, device=device)


@dataclass
class PackedColumn:
    """n elements of `bits` bits in `fmt`, stored in the byte tensor `data`."""
    data: torch.Tensor
    n: int
    fmt: int
    bits: int

    @property
    def desc(self) -> A.Column:
        return A.Column(self.data.data_ptr(), self.n, self.fmt, self.bits)

    @property
    def nbytes(self) -> int:
        return storage_bytes(self.fmt, self.bits, self.n)

    @staticmethod
    def empty(n: int, fmt: int, bits: int, device="cuda", capacity: int | None = None) -> "PackedColumn":
        cap = n if capacity is None else capacity
        return PackedColumn(alloc_bytes(storage_bytes(fmt, bits, cap), device), n, fmt, bits)

    @staticmethod
    def from_bytes(raw: bytes | memoryview, n: int, fmt: int, bits: int, device="cuda") -> "PackedColumn":
        col = PackedColumn.empty(n, fmt, bits, device)
        host = torch.frombuffer(bytearray(raw), dtype=torch.uint8)
        col.data[: host.numel()].copy_(host)
        return col

    def host_bytes(self, n: int | None = None) -> bytes:
        nb = storage_bytes(self.fmt, self.bits, self.n if n is None else n)
        return self.data[:nb].cpu().numpy().tobytes()


def predicate(kind: int, k0: int = 0, k1: int = 0, bits: int = 0) -> A.Predicate:
    return A.Predicate(kind, bits, k0, k1)


def workspace(n: int, device="cuda") -> torch.Tensor:
    return torch.empty(int(lib().amx_workspace_bytes(n)), dtype=torch.uint8, device=device)


def mask_words(n: int) -> int:
    return (n + 31) // 32


def filter(col: PackedColumn, pred: A.Predicate, ws=None, stream=None) -> torch.Tensor:
    """Bitmask (int32 words, LSB-first) of pred over the column."""
    mask = torch.zeros(mask_words(col.n) + 4, dtype=torch.int32, device=col.data.device)
    ws = workspace(col.n, col.data.device) if ws is None else ws
    check(lib().amx_filter(C.byref(col.desc), C.byref(pred), _ptr(mask), _ptr(ws), ws.numel(), _stream_ptr(stream)))
    return mask


def compressstore(col: PackedColumn, mask: torch.Tensor, out_fmt: int, out_bits: int, ws=None, stream=None):
    """Survivors of the mask in order; returns (output column sized for n, count tensor)."""
    out = PackedColumn.empty(col.n, out_fmt, out_bits, col.data.device)
    cnt = torch.zeros(2, dtype=torch.int64, device=col.data.device)
    ws = workspace(col.n, col.data.device) if ws is None else ws
    check(lib().amx_compressstore(C.byref(col.desc), _ptr(mask), C.byref(out.desc), _ptr(cnt), _ptr(ws), ws.numel(),
                                  _stream_ptr(stream)))
    return out, cnt


def filter_compressstore(col: PackedColumn, pred: A.Predicate, out_fmt: int, out_bits: int, ws=None, stream=None):
    out = PackedColumn.empty(col.n, out_fmt, out_bits, col.data.device)
    cnt = torch.zeros(2, dtype=torch.int64, device=col.data.device)
    ws = workspace(col.n, col.data.device) if ws is None else ws
    check(lib().amx_filter_compressstore(C.byref(col.desc), C.byref(pred), C.byref(out.desc), _ptr(cnt), _ptr(ws),
                                         ws.numel(), _stream_ptr(stream)))
    return out, cnt


def binary_op(op: int, lhs: PackedColumn, rhs: PackedColumn, out_fmt: int, out_bits: int | None = None, ws=None,
              stream=None) -> PackedColumn:
    if out_bits is None:
        out_bits = int(lib().amx_binary_out_bits(op, lhs.bits, rhs.bits))
    out = PackedColumn.empty(lhs.n, out_fmt, out_bits, lhs.data.device)
    ws = workspace(lhs.n, lhs.data.device) if ws is None else ws
    check(lib().amx_binary(op, C.byref(lhs.desc), C.byref(rhs.desc), C.byref(out.desc), _ptr(ws), ws.numel(),
                           _stream_ptr(stream)))
    return out


def convert(col: PackedColumn, out_fmt: int, out_bits: int, ws=None, stream=None) -> PackedColumn:
    out = PackedColumn.empty(col.n, out_fmt, out_bits, col.data.device)
    ws = workspace(col.n, col.data.device) if ws is None else ws
    check(lib().amx_convert(C.byref(col.desc), C.byref(out.desc), _ptr(ws), ws.numel(), _stream_ptr(stream)))
    return out


def hop(agg: int, col: PackedColumn, mask: torch.Tensor | None = None, ws=None, stream=None) -> torch.Tensor:
    """Aggregation into one uint64 (returned in an int64 tensor of one element)."""
    res = torch.zeros(2, dtype=torch.int64, device=col.data.device)
    ws = workspace(col.n, col.data.device) if ws is None else ws
    check(lib().amx_reduce(agg, C.byref(col.desc), _ptr(mask), _ptr(res), _ptr(ws), ws.numel(), _stream_ptr(stream)))
    return res[:1]


reduce = hop


def chain(lhs: PackedColumn, rhs: PackedColumn | None, op: int, value_bits: int, pred: A.Predicate,
          agg: int = A.AGG_SUM, out_fmt: int | None = None, out_bits: int | None = None, want_mask: bool = False,
          want_agg: bool = True, ws=None, stream=None):
    """Fused v = op(lhs, rhs) -> filter pred(v) -> compressstore / mask / count / aggregate."""
    dev = lhs.data.device
    desc = A.ChainDesc(op, value_bits, pred, agg, 0)
    out = PackedColumn.empty(lhs.n, out_fmt, out_bits or value_bits, dev) if out_fmt is not None else None
    mask = torch.zeros(mask_words(lhs.n) + 4, dtype=torch.int32, device=dev) if want_mask else None
    cnt = torch.zeros(2, dtype=torch.int64, device=dev)
    ag = torch.zeros(2, dtype=torch.int64, device=dev) if want_agg else None
    ws = workspace(lhs.n, dev) if ws is None else ws
    check(lib().amx_chain(C.byref(desc), C.byref(lhs.desc), C.byref(rhs.desc) if rhs is not None else None,
                          C.byref(out.desc) if out is not None else None, _ptr(mask), _ptr(cnt), _ptr(ag), _ptr(ws),
                          ws.numel(), _stream_ptr(stream)))
    return out, mask, cnt, ag


def groupby_workspace(key_bits: int, max_groups: int | None = None, device="cuda") -> torch.Tensor:
    """A 256-byte-aligned group-by workspace: the dense table for keys of at most 24 bits, a hash
    table for `max_groups` distinct keys above that."""
    if key_bits <= 24:
        nb = int(lib().amx_groupby_workspace_bytes(key_bits))
    else:
        nb = int(lib().amx_groupby_wide_workspace_bytes(key_bits, max_groups or (1 << 20)))
    return aligned_bytes(nb, 256, device)


def groupby(keys: PackedColumn, vals: PackedColumn, key_fmt: int = A.PLAIN32, sum_fmt: int = A.PLAIN64,
            sum_bits: int = 64, count_fmt: int | None = A.PLAIN64, mask: torch.Tensor | None = None, ws=None,
            stream=None, max_groups: int | None = None):
    """Group-by sum + count (kernel_groupby_sm_array's successor): returns (keys, sums, counts,
    groups tensor) with groups in ascending key order.  Keys of 25..32 bits hold up to
    `max_groups` (default 2^20) distinct keys."""
    dev = keys.data.device
    g = 1 << keys.bits if keys.bits <= 24 else (max_groups or (1 << 20))
    ok = PackedColumn.empty(g, key_fmt, keys.bits if key_fmt != A.PLAIN32 or keys.bits <= 32 else 32, dev)
    os_ = PackedColumn.empty(g, sum_fmt, sum_bits, dev)
    oc = PackedColumn.empty(g, count_fmt, 64 if count_fmt != A.PLAIN32 else 32, dev) if count_fmt is not None else None
    ng = torch.zeros(2, dtype=torch.int64, device=dev)
    if ws is None:
        ws = groupby_workspace(keys.bits, max_groups, dev)
    check(lib().amx_groupby(C.byref(keys.desc), C.byref(vals.desc), _ptr(mask), C.byref(ok.desc), C.byref(os_.desc),
                            C.byref(oc.desc) if oc is not None else None, _ptr(ng), _ptr(ws), ws.numel(),
                            _stream_ptr(stream)))
    return ok, os_, oc, ng


def groupby_sort(keys: PackedColumn, vals: PackedColumn, key_fmt: int = A.PLAIN32, sum_fmt: int = A.PLAIN64,
                 sum_bits: int = 64, count_fmt: int | None = A.PLAIN64, mask: torch.Tensor | None = None, ws=None,
                 stream=None, max_groups: int | None = None):
    """Sort-based group-by sum + count (the reference's radix sort + reduce-by-key path): returns
    (keys, sums, counts, groups tensor), groups in ascending key order; outputs hold `max_groups`
    groups (default: every pair could be its own group)."""
    dev = keys.data.device
    g = max_groups if max_groups is not None else max(1, min(keys.n, 1 << keys.bits))
    ok = PackedColumn.empty(g, key_fmt, keys.bits if key_fmt != A.PLAIN32 or keys.bits <= 32 else 32, dev)
    os_ = PackedColumn.empty(g, sum_fmt, sum_bits, dev)
    oc = PackedColumn.empty(g, count_fmt, 64 if count_fmt != A.PLAIN32 else 32, dev) if count_fmt is not None else None
    ng = torch.zeros(2, dtype=torch.int64, device=dev)
    if ws is None:
        ws = aligned_bytes(int(lib().amx_groupby_sort_workspace_bytes(keys.n, keys.bits, vals.bits)), 256, dev)
    check(lib().amx_groupby_sort(C.byref(keys.desc), C.byref(vals.desc), _ptr(mask), C.byref(ok.desc),
                                 C.byref(os_.desc), C.byref(oc.desc) if oc is not None else None, _ptr(ng), _ptr(ws),
                                 ws.numel(), _stream_ptr(stream)))
    return ok, os_, oc, ng


def groupby_auto(keys: PackedColumn, vals: PackedColumn, groups_hint: int, **kw):
    """Group-by through the variant that the expected number of groups favours: the hash tables
    (amx_groupby) below n / 128 groups, radix sort + reduce-by-key (amx_groupby_sort) from there
    on.  Measured on 2^26 32-bit keys (bench line groupby_wide): 100,000 groups 2.67 vs 3.19 ms
    (hash faster), 2^20 groups 6.54 vs 3.30 ms, 2^23 groups 10.79 vs 3.51 ms, 6.7e7 groups 29.0 vs
    5.30 ms (sort faster).  Keys of at most 24 bits always take the dense tables."""
    if keys.bits > 24 and groups_hint * 128 >= max(keys.n, 1):
        return groupby_sort(keys, vals, max_groups=kw.pop("max_groups", None) or max(1, min(keys.n, groups_hint * 2)),
                            **{k: v for k, v in kw.items() if k != "ws"})
    return groupby(keys, vals, max_groups=kw.pop("max_groups", None) or max(1024, 2 * groups_hint), **kw)


def matmul_workspace(m: int, n: int, k: int, device="cuda") -> torch.Tensor:
    """A 1024-byte-aligned workspace for amx_matmul (torch hands out 512-byte-aligned blocks)."""
    nb = int(lib().amx_matmul_workspace_bytes(m, n, k))
    raw = torch.empty(nb + 1024, dtype=torch.uint8, device=device)
    off = (-raw.data_ptr()) % 1024
    return raw[off: off + nb]


def matmul(a: PackedColumn, b: PackedColumn, m: int, n: int, k: int, out_fmt: int = A.SLAB, out_bits: int = 0,
           ws=None, stream=None):
    """C = A (m x k) * B (k x n) on the integer tensor cores.  out_bits 0 picks the narrowest width
    holding the largest entry; returns (C column, device tensor holding the width used)."""
    dev = a.data.device
    nb = int(lib().amx_matmul_out_bytes(out_fmt, out_bits, m, n, k, a.bits, b.bits))
    if nb == 0 and m * n:
        raise ValueError("unsupported matmul widths")
    out = PackedColumn(alloc_bytes(nb, dev), m * n, out_fmt, out_bits)
    width = torch.zeros(4, dtype=torch.int32, device=dev)
    ws = matmul_workspace(m, n, k, dev) if ws is None else ws
    check(lib().amx_matmul(C.byref(a.desc), C.byref(b.desc), m, n, k, C.byref(out.desc), _ptr(width), _ptr(ws),
                           ws.numel(), _stream_ptr(stream)))
    return out, width


class Batch:
    """A prepared batch of slab columns for one-launch filter + compressstore + sum
    (amx_batch_prepare / amx_batch_run).  Keeps the column arrays, outputs and workspace alive."""

    def __init__(self, cols: list, preds: list, tuning: A.BatchTuning | None = None, device="cuda"):
        self.cols = cols
        self.outs = [PackedColumn.empty(c.n, A.SLAB, c.bits, device) for c in cols]
        n = len(cols)
        self.ins_arr = (A.Column * max(n, 1))(*[c.desc for c in cols])
        self.outs_arr = (A.Column * max(n, 1))(*[o.desc for o in self.outs])
        self.preds_arr = (A.Predicate * max(n, 1))(*preds)
        self.tuning = tuning
        tp = C.byref(tuning) if tuning is not None else None
        nb = int(lib().amx_batch_workspace_bytes(self.ins_arr, n, tp))
        self.ws = torch.empty(max(nb, 256) + 256, dtype=torch.uint8, device=device)
        off = (-self.ws.data_ptr()) % 256
        self.ws = self.ws[off: off + max(nb, 256)]
        self.plan = A.BatchPlan()
        self.counts = torch.zeros(max(n, 1), dtype=torch.int64, device=device)
        self.sums = torch.zeros(max(n, 1), dtype=torch.int64, device=device)
        check(lib().amx_batch_prepare(self.ins_arr, self.preds_arr, self.outs_arr, n, tp, C.byref(self.plan),
                                      _ptr(self.ws), self.ws.numel(), _stream_ptr()))

    def run(self, stream=None):
        check(lib().amx_batch_run(C.byref(self.plan), _ptr(self.counts), _ptr(self.sums), _ptr(self.ws),
                                  self.ws.numel(), _stream_ptr(stream)))
        return self.counts, self.sums

    def status(self, stream=None):
        check(lib().amx_batch_status(_ptr(self.ws), _stream_ptr(stream)))


def bit_histogram(col: PackedColumn, stream=None) -> torch.Tensor:
    """65 counters: elements whose value needs exactly k bits (amx_bit_histogram)."""
    h = torch.zeros(65, dtype=torch.int64, device=col.data.device)
    check(lib().amx_bit_histogram(C.byref(col.desc), _ptr(h), _stream_ptr(stream)))
    return h


def aligned_bytes(nbytes: int, align: int = 256, device="cuda") -> torch.Tensor:
    raw = torch.empty(max(nbytes, 1) + align, dtype=torch.uint8, device=device)
    off = (-raw.data_ptr()) % align
    return raw[off: off + max(nbytes, 1)]


class Program:
    """An operator-chain program (amx_program_*): the steps run on the device with every
    intermediate length kept there, so a run can be captured into a CUDA graph.  Holds its
    workspace and the objects its steps point to."""

    def __init__(self, x: PackedColumn, steps: list, keep: list | None = None, device="cuda"):
        self.x = x
        self.keep = keep or []
        self.nsteps = len(steps)
        self.steps = (A.Step * max(1, len(steps)))(*steps)
        h = C.c_void_p()
        check(lib().amx_program_create(C.byref(x.desc), self.steps, len(steps), C.byref(h)))
        self.h = h
        self.ws_bytes = int(lib().amx_program_workspace_bytes(h))
        self.ws = aligned_bytes(self.ws_bytes, 256, device)

    def run(self, stream=None):
        check(lib().amx_program_run(self.h, _ptr(self.ws), self.ws_bytes, _stream_ptr(stream)))

    def output(self):
        """(final column descriptor, device length pointer or None)."""
        col = A.Column()
        dl = C.c_void_p()
        check(lib().amx_program_output(self.h, _ptr(self.ws), C.byref(col), C.byref(dl)))
        return col, dl.value

    def status(self, stream=None):
        check(lib().amx_program_status(self.h, _ptr(self.ws), _stream_ptr(stream)))

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            lib().amx_program_destroy(h)
            self.h = None


class Graph:
    """Many programs captured into one CUDA graph (amx_graph_capture), programs spread over
    `lanes` streams that fork from and join the launching stream."""

    def __init__(self, programs: list, lanes: int = 4):
        self.programs = programs
        n = len(programs)
        hs = (C.c_void_p * max(1, n))(*[p.h.value for p in programs])
        ws = (C.c_void_p * max(1, n))(*[p.ws.data_ptr() for p in programs])
        wb = (C.c_uint64 * max(1, n))(*[p.ws_bytes for p in programs])
        g = C.c_void_p()
        check(lib().amx_graph_capture(hs, ws, wb, n, lanes, C.byref(g)))
        self.h = g

    def launch(self, stream=None):
        check(lib().amx_graph_launch(self.h, _stream_ptr(stream)))

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            lib().amx_graph_destroy(h)
            self.h = None


def groupby_status(ws: torch.Tensor, key_bits: int, stream=None) -> None:
    check(lib().amx_groupby_status(_ptr(ws), key_bits, _stream_ptr(stream)))


def workspace_status(ws: torch.Tensor, stream=None) -> None:
    check(lib().amx_workspace_status(_ptr(ws), _stream_ptr(stream)))
