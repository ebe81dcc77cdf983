"""ctypes driver of the reference harness (oracle/_ref/libariesref.so, built
from the reference's own AriesDecimal<LEN> code by oracle/ref/Makefile).

TEST INFRASTRUCTURE: used by tests and by make_golden.py on a GPU host.
"""
from __future__ import annotations

import ctypes as C
import os

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB = os.path.join(ROOT, "oracle", "_ref", "libariesref.so")

OPS = {"add": 0, "sub": 1, "mul": 2, "div": 3, "mod": 4, "lt": 10, "le": 11, "gt": 12, "ge": 13, "eq": 14,
       "ne": 15, "mad": 20, "q_dp": 30, "q_charge": 31}
LENS = [2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32]

_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def load():
    global _lib
    if _lib is None:
        lib = C.CDLL(LIB)
        lib.ref_eval.restype = C.c_int
        lib.ref_eval.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                 C.c_void_p, C.c_int, C.c_int, C.c_int64, C.c_void_p, C.c_int, C.c_int]
        lib.ref_supported_len.restype = C.c_int
        _lib = lib
    return _lib


def bits_pow10(k: int) -> int:
    return (10 ** k).bit_length() if k > 0 else 0


def need_limbs(op: str, ba: int, sa: int, bb: int, sb: int, bc: int = 0, sc: int = 0) -> int:
    """Limbs that hold every intermediate of the operation exactly."""
    A, Bv = 8 * ba, 8 * bb
    if op in ("add", "sub") or op in ("lt", "le", "gt", "ge", "eq", "ne"):
        bits = max(A + bits_pow10(max(0, sb - sa)), Bv + bits_pow10(max(0, sa - sb))) + 1
    elif op == "mul":
        bits = A + Bv
    elif op == "div":
        bits = max(A + bits_pow10(sb + 4), Bv) + 1
    elif op == "mod":
        bits = max(A, Bv)
    elif op == "mad":
        s = max(sc, sa + sb)
        bits = max(A + Bv + bits_pow10(s - sa - sb), 8 * bc + bits_pow10(s - sc)) + 1
    else:  # query shapes
        bits = A + 2 * 64 + 8
    return (bits + 31) // 32


def pick_len(op: str, need: int) -> int:
    want = need + 2 if op in ("div", "mod") else need
    for L in LENS:
        if L >= want:
            return L
    raise ValueError("needs more limbs than the harness instantiates")


def run(op: str, a_dev, pa, sa, b_dev, pb, sb, rows, out_dev, out_bytes, c_dev=None, pc=0, sc=0, length=None,
        need=None, b_host: bytes | None = None):
    """Evaluate with the reference.  For MOD the divisor column must also be
    given on the host (b_host): the reference's ModCalc faults on a zero
    divisor (no check before its top-limb scan, AriesDecimal.hxx:970-973), so
    such rows are refused here before anything reaches the GPU."""
    lib = load()
    if op == "mod":
        from ultraprecise_b200 import codec as _codec
        bb = _codec.compact_bytes(pb)
        if b_host is None or len(b_host) < rows * bb:
            raise ValueError("MOD needs the divisor column on the host for the zero check")
        for i in range(rows):
            v = bytearray(b_host[i * bb:(i + 1) * bb])
            v[-1] &= 0x7F
            if not any(v):
                raise ValueError("zero divisor given to the reference's MOD")
    if need is None:
        from ultraprecise_b200 import codec
        need = need_limbs(op, codec.compact_bytes(pa), sa, codec.compact_bytes(pb), sb,
                          codec.compact_bytes(pc) if c_dev is not None else 0, sc)
    L = length or pick_len(op, need)
    rc = lib.ref_eval(OPS[op], L, a_dev, pa, sa, b_dev, pb, sb, c_dev, pc, sc, rows, out_dev, out_bytes,
                      need if op in ("div", "mod") else 0)
    if rc != 0:
        raise RuntimeError(f"reference harness refused or failed: {rc} (op {op}, LEN {L})")
    return L


# ------------------------------------------------------------------------
# The 32-limb Decimal harness (oracle/_ref/libariesref_agg.so): grouped SUM by
# the XMP segmented-reduction add, AVG by Decimal /= int64, CSV-import text
# parse and GetDecimal text output, each run by the reference's own code.
AGG_LIB = os.path.join(ROOT, "oracle", "_ref", "libariesref_agg.so")
_agg = None
FORMAT_WIDTH = 8 * 32 + 8


def agg_available() -> bool:
    return os.path.exists(AGG_LIB)


def agg_load():
    global _agg
    if _agg is None:
        lib = C.CDLL(AGG_LIB)
        P = C.c_void_p
        lib.refagg_compact_bytes.restype = C.c_int
        lib.refagg_compact_bytes.argtypes = [C.c_int]
        lib.refagg_sum.restype = C.c_int
        lib.refagg_sum.argtypes = [P, C.c_int, C.c_int, P, P, C.c_int, C.c_int64, P]
        lib.refagg_div_int64.restype = C.c_int
        lib.refagg_div_int64.argtypes = [P, P, C.c_int, P]
        lib.refagg_parse.restype = C.c_int
        lib.refagg_parse.argtypes = [P, P, P, C.c_int64, C.c_int, C.c_int, P, P]
        lib.refagg_format.restype = C.c_int
        lib.refagg_format.argtypes = [P, C.c_int64, C.c_int, C.c_int, P, C.c_int]
        _agg = lib
    return _agg


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference harness refused or failed: {rc} ({what})")


def sum_segments(vals: bytes, prec: int, scale: int, starts, rows: int, assoc=None) -> bytes:
    """133-byte SUM images of each segment [starts[g], starts[g+1]) of a host
    compact column (visited through `assoc` when given)."""
    import torch
    lib = agg_load()
    d = torch.frombuffer(bytearray(vals or b"\0"), dtype=torch.uint8).cuda()
    st = torch.tensor(list(starts) or [0], dtype=torch.int32).cuda()
    asc = torch.tensor(list(assoc), dtype=torch.int32).cuda() if assoc is not None else None
    out = torch.zeros(max(1, len(starts)) * 133, dtype=torch.uint8).cuda()
    _check(lib.refagg_sum(d.data_ptr(), prec, scale, asc.data_ptr() if asc is not None else None, st.data_ptr(),
                          len(starts), rows, out.data_ptr()), "sum")
    return bytes(out.cpu().numpy().tobytes())[:len(starts) * 133]


def div_int64(images: bytes, counts) -> bytes:
    import torch
    lib = agg_load()
    n = len(counts)
    s = torch.frombuffer(bytearray(images or b"\0"), dtype=torch.uint8).cuda()
    c = torch.tensor(list(counts) or [0], dtype=torch.int64).cuda()
    out = torch.zeros(max(1, n) * 133, dtype=torch.uint8).cuda()
    _check(lib.refagg_div_int64(s.data_ptr(), c.data_ptr(), n, out.data_ptr()), "div_int64")
    return bytes(out.cpu().numpy().tobytes())[:n * 133]


def parse(fields, prec: int, scale: int):
    """(compact bytes, per-row error codes) of text fields."""
    import torch
    lib = agg_load()
    text = b"".join(fields)
    offs = [0]
    for f in fields:
        offs.append(offs[-1] + len(f))
    host_offs = (C.c_int64 * len(offs))(*offs)
    t = torch.frombuffer(bytearray(text or b"\0"), dtype=torch.uint8).cuda()
    o = torch.tensor(offs, dtype=torch.int64).cuda()
    nb = lib.refagg_compact_bytes(prec)
    out = torch.zeros(max(1, len(fields) * nb), dtype=torch.uint8).cuda()
    err = torch.zeros(max(1, len(fields)), dtype=torch.uint8).cuda()
    _check(lib.refagg_parse(t.data_ptr(), o.data_ptr(), host_offs, len(fields), prec, scale, out.data_ptr(),
                            err.data_ptr()), "parse")
    return bytes(out.cpu().numpy().tobytes())[:len(fields) * nb], bytes(err.cpu().numpy().tobytes())[:len(fields)]


def format_hex(compact: bytes, rows: int, prec: int, scale: int):
    """GetDecimal strings of a host compact column."""
    import torch
    lib = agg_load()
    d = torch.frombuffer(bytearray(compact or b"\0"), dtype=torch.uint8).cuda()
    out = torch.zeros(max(1, rows) * FORMAT_WIDTH, dtype=torch.uint8).cuda()
    _check(lib.refagg_format(d.data_ptr(), rows, prec, scale, out.data_ptr(), FORMAT_WIDTH), "format")
    raw = bytes(out.cpu().numpy().tobytes())
    return [raw[i * FORMAT_WIDTH:(i + 1) * FORMAT_WIDTH].split(b"\0", 1)[0].decode() for i in range(rows)]
