"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline / reference arm.  Never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from ultraprecise_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    P = C.c_void_p
    lib.orc_compact_bytes.restype = C.c_int32
    lib.orc_compact_bytes.argtypes = [C.c_int32]
    lib.orc_precision_words.restype = C.c_int32
    lib.orc_precision_words.argtypes = [C.c_int32]
    lib.orc_eval_expr.restype = C.c_int32
    lib.orc_eval_expr.argtypes = [P, C.c_int32, C.c_int32, P, P, C.c_int64, C.c_int64, P, C.c_int32, P, P]
    lib.orc_eval_expr_mt.restype = C.c_int32
    lib.orc_eval_expr_mt.argtypes = [P, C.c_int32, C.c_int32, P, P, C.c_int64, P, C.c_int32, P, C.c_int32]
    lib.orc_group_agg.restype = C.c_int32
    lib.orc_group_agg.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, P, C.c_int64, C.c_int32, P]
    lib.orc_query.restype = C.c_int32
    lib.orc_query.argtypes = [P, C.c_int32, P, P, P, C.c_int32, P, C.c_int64, C.c_int32, P, C.c_int32]
    lib.orc_division_int64.restype = None
    lib.orc_division_int64.argtypes = [P, C.c_int64, P]
    _lib = lib
    return lib


def _ptrs(bufs):
    arr = (C.c_void_p * max(1, len(bufs)))()
    keep = []
    for i, b in enumerate(bufs):
        cb = (C.c_char * len(b)).from_buffer_copy(b) if not isinstance(b, C.Array) else b
        keep.append(cb)
        arr[i] = C.cast(cb, C.c_void_p)
    return arr, keep


def eval_expr(built, root: int, cols: list[bytes], rows: int, out_bytes: int, threads: int = 1,
              row_errors: bool = False):
    """Evaluate `built.nodes` at `root` over host columns; returns
    (bytes, err_word[, per-row error bytes])."""
    lib = load()
    arr, keep = _ptrs(cols)
    out = (C.c_uint8 * max(1, rows * out_bytes))()
    err = C.c_uint32(0)
    if threads > 1 and not row_errors:
        rc = lib.orc_eval_expr_mt(built.nodes, built.n_nodes, root, built.col_types, arr, rows, out, out_bytes,
                                  C.byref(err), threads)
        rerr = None
    else:
        rerr = (C.c_uint8 * max(1, rows))()
        rc = lib.orc_eval_expr(built.nodes, built.n_nodes, root, built.col_types, arr, 0, rows, out, out_bytes,
                               C.byref(err), rerr)
    if rc != 0:
        raise RuntimeError("oracle rejected the expression")
    res = bytes(out)[:rows * out_bytes]
    if row_errors:
        return res, err.value, bytes(rerr)[:rows]
    return res, err.value


def group_agg(vals: bytes, value_bytes: int, scale: int, kind: int, gids: bytes, rows: int, n_groups: int) -> bytes:
    lib = load()
    width = 8 if kind == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES
    out = (C.c_uint8 * max(1, n_groups * width))()
    v = (C.c_char * max(1, len(vals))).from_buffer_copy(vals or b"\0")
    g = (C.c_char * max(1, len(gids))).from_buffer_copy(gids or b"\0")
    lib.orc_group_agg(v, value_bytes, scale, kind, g, rows, n_groups, out)
    return bytes(out)[:n_groups * width]


def query(built, aggs: list[tuple[int, int]], cols: list[bytes], gids: bytes, rows: int, n_groups: int,
          threads: int = 1) -> list[bytes]:
    """aggs: (kind, root) pairs; returns one output buffer per aggregate."""
    lib = load()
    arr, keep = _ptrs(cols)
    qa = (abi.UpQueryAgg * len(aggs))()
    outs = []
    optr = (C.c_void_p * len(aggs))()
    for i, (k, r) in enumerate(aggs):
        qa[i].kind = k
        qa[i].root = r
        width = 8 if k == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES
        o = (C.c_uint8 * max(1, n_groups * width))()
        outs.append((o, width))
        optr[i] = C.cast(o, C.c_void_p)
    g = (C.c_char * max(1, len(gids))).from_buffer_copy(gids or b"\0")
    lib.orc_query(built.nodes, built.n_nodes, built.col_types, arr, qa, len(aggs), g, rows, n_groups, optr,
                  threads)
    return [bytes(o)[:n_groups * w] for o, w in outs]


def division_int64(sum_img: bytes, count: int) -> bytes:
    lib = load()
    out = (C.c_uint8 * abi.UP_AGG_DECIMAL_BYTES)()
    s = (C.c_char * len(sum_img)).from_buffer_copy(sum_img)
    lib.orc_division_int64(s, count, out)
    return bytes(out)


def compact_bytes(p: int) -> int:
    """B(p) from the oracle's own table (the reference's byte table,
    decimal.cu:92, with the p >= 300 extension)."""
    b = load().orc_compact_bytes(p)
    if b < 1:
        raise ValueError(f"precision {p} out of range")
    return b


def _type_binary(kind: int, p1: int, s1: int, p2: int, s2: int) -> tuple[int, int]:
    """Result (precision, scale) of one operator node, ListToBinTree's rules
    (AriesEngineShell.cpp:115-141): ADD/SUB take the wider integer part plus a
    carry digit over the larger scale; MUL adds integer digits and scales; DIV
    (DIV_FIX_EX_FRAC = 4) is p1 - p2 + s2 + 4 + 1 over s1 + 4; MOD keeps the
    divisor's precision at scale 0.  A DIV precision that would not exceed its
    scale is widened to scale + 1 (the reference's uint16 fields wrap there)."""
    if kind in (abi.UP_NODE_ADD, abi.UP_NODE_SUB):
        s = max(s1, s2)
        return max(p1 - s1, p2 - s2) + 1 + s, s
    if kind == abi.UP_NODE_MUL:
        return (p1 - s1) + (p2 - s2) + s1 + s2, s1 + s2
    if kind == abi.UP_NODE_DIV:
        p, s = p1 - p2 + s2 + 5, s1 + 4
        return (p if p > s else s + 1), s
    if kind == abi.UP_NODE_MOD:
        return p2, 0
    raise ValueError(f"node kind {kind} has no binary typing rule")


def derive_types(built, root: int | None = None):
    """Fill every inner node's (precision, scale) in place, children first,
    with the reference's typing rules; the oracle's restatement of the
    library's up_expr_derive_types, so that CPU-only callers (the reference
    arm of the benchmark) never load the product library.  Integer literals
    type as Decimal(int32_t) / Decimal(int64_t) do (decimal.cu:291-309):
    precision 10 or 19, scale 0; comparisons and AND/OR give (1, 0); constants
    and RESCALE nodes keep the type they were given."""
    nodes = built.nodes
    roots = [root] if root is not None else list(built.roots)
    done: set[int] = set()

    def visit(k: int) -> None:
        stack = [(k, False)]
        while stack:
            i, expanded = stack.pop()
            if i in done:
                continue
            nd = nodes[i]
            if not expanded:
                stack.append((i, True))
                for ch in (nd.left, nd.right):
                    if ch >= 0 and ch not in done:
                        stack.append((ch, False))
                continue
            if nd.kind == abi.UP_NODE_COLUMN:
                ct = built.col_types[nd.column]
                nd.precision, nd.scale = ct.precision, ct.scale
            elif nd.kind == abi.UP_NODE_INT:
                fits32 = -2147483648 <= nd.int_value <= 2147483647
                nd.precision, nd.scale = (10 if fits32 else 19), 0
            elif nd.kind in (abi.UP_NODE_CONST, abi.UP_NODE_RESCALE):
                pass
            elif nd.kind in abi.COMPARE_KINDS:
                nd.precision, nd.scale = 1, 0
            else:
                a, b = nodes[nd.left], nodes[nd.right]
                nd.precision, nd.scale = _type_binary(nd.kind, a.precision, a.scale, b.precision, b.scale)
            done.add(i)

    for r in roots:
        visit(r)
    return built
