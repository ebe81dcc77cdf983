"""Device-side runtime over the C ABI.

torch is used only for device memory and streams; every computation runs in
libultraprecise.so's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import torch

from . import abi, codec
from .expr import Built, ColType, Expr, build, derive_types


def _stream_ptr(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


@dataclass
class DeviceColumn:
    """A compact decimal column in HBM: rows x value_bytes uint8."""
    data: torch.Tensor | None
    precision: int
    scale: int
    nullable: bool = False
    indices: torch.Tensor | None = None   # int32 row indirection (-1 = NULL)
    # block list (the reference's multi-block AriesColumnDataIterator): the
    # rows live in several device buffers; block_ptrs holds their addresses
    # and block_prefix the int64 row prefix sums (n_blocks + 1), both on the
    # device, and blocks keeps the buffers alive
    blocks: list | None = None
    block_ptrs: torch.Tensor | None = None
    block_prefix: torch.Tensor | None = None

    @staticmethod
    def from_blocks(blocks, precision: int, scale: int, nullable: bool = False) -> "DeviceColumn":
        """A column whose rows are spread over several device buffers (uint8
        tensors of whole values), in order."""
        vb = codec.compact_bytes(precision) + (1 if nullable else 0)
        counts = [b.numel() // vb for b in blocks]
        prefix = [0]
        for n in counts:
            prefix.append(prefix[-1] + n)
        ptrs = torch.tensor([b.data_ptr() for b in blocks], dtype=torch.int64, device="cuda")
        pre = torch.tensor(prefix, dtype=torch.int64, device="cuda")
        return DeviceColumn(None, precision, scale, nullable, None, list(blocks), ptrs, pre)

    @property
    def value_bytes(self) -> int:
        return codec.compact_bytes(self.precision) + (1 if self.nullable else 0)

    @property
    def rows(self) -> int:
        if self.indices is not None:
            return self.indices.numel()
        if self.blocks is not None:
            return int(self.block_prefix[-1].item())
        return self.data.numel() // self.value_bytes

    def up_column(self) -> abi.UpColumn:
        c = abi.UpColumn()
        c.data = self.data.data_ptr() if self.data is not None else None
        c.blocks = self.block_ptrs.data_ptr() if self.blocks is not None else None
        c.block_prefix = self.block_prefix.data_ptr() if self.blocks is not None else None
        c.n_blocks = len(self.blocks) if self.blocks is not None else 0
        c.indices = self.indices.data_ptr() if self.indices is not None else None
        c.precision = self.precision
        c.scale = self.scale
        c.value_bytes = self.value_bytes
        c.nullable = 1 if self.nullable else 0
        return c

    @staticmethod
    def from_host(raw: bytes, precision: int, scale: int, device="cuda", nullable=False) -> "DeviceColumn":
        t = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(device) if raw else torch.empty(
            0, dtype=torch.uint8, device=device)
        return DeviceColumn(t, precision, scale, nullable)

    def col_type(self) -> ColType:
        return ColType(self.precision, self.scale, self.nullable)


def _columns_array(cols: Sequence[DeviceColumn]):
    arr = (abi.UpColumn * max(1, len(cols)))()
    for i, c in enumerate(cols):
        arr[i] = c.up_column()
    return arr


class ExprModule:
    """A compiled projection kernel (the reference's AEExprCalcNode kernel)."""

    def __init__(self, built: Built, root: int, threads_per_value: int = 0, block_threads: int = 0):
        lib = abi.load()
        self.built = built
        self.root = root
        opts = abi.UpCompileOpts(threads_per_value, block_threads, 0)
        h = C.c_void_p()
        abi.check(lib.up_module_compile(built.nodes, built.n_nodes, root, built.col_types, built.n_cols,
                                        C.byref(opts), C.byref(h)), "up_module_compile")
        self._h = h
        p, s, vb = C.c_int32(), C.c_int32(), C.c_int32()
        abi.check(lib.up_module_result_type(h, C.byref(p), C.byref(s), C.byref(vb)), "up_module_result_type")
        self.precision, self.scale, self.value_bytes = p.value, s.value, vb.value

    @property
    def threads_per_value(self) -> int:
        return int(abi.load().up_module_threads_per_value(self._h))

    def source(self) -> str:
        lib = abi.load()
        n = lib.up_module_source(self._h, None, 0)
        buf = C.create_string_buffer(int(n) + 1)
        lib.up_module_source(self._h, buf, n + 1)
        return buf.value.decode()

    def launch(self, cols: Sequence[DeviceColumn], rows: int | None = None, out: torch.Tensor | None = None,
               err: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        lib = abi.load()
        if rows is None:
            rows = cols[0].rows if cols else 0
        if out is None:
            out = torch.empty(rows * self.value_bytes, dtype=torch.uint8, device="cuda")
        arr = _columns_array(cols)
        abi.check(lib.up_expr_launch(self._h, arr, len(cols), rows, out.data_ptr(),
                                     err.data_ptr() if err is not None else None, _stream_ptr(stream)),
                  "up_expr_launch")
        return out

    def launch_host(self, cols: Sequence[torch.Tensor], types: Sequence[ColType], rows: int, out: torch.Tensor,
                    chunk_rows: int = 0) -> int:
        """Launch over HOST columns (uint8 CPU tensors, ideally pinned): the
        rows stream through the GPU in overlapped chunks; `out` (uint8 CPU
        tensor of rows*value_bytes) receives the results.  Returns the OR of
        the row errors."""
        lib = abi.load()
        arr = (abi.UpColumn * max(1, len(cols)))()
        for i, (t, ct) in enumerate(zip(cols, types)):
            arr[i].data = t.data_ptr()
            arr[i].precision = ct.precision
            arr[i].scale = ct.scale
            arr[i].value_bytes = codec.compact_bytes(ct.precision)
        err = C.c_uint32(0)
        abi.check(lib.up_expr_launch_host(self._h, arr, len(cols), rows, out.data_ptr(), C.byref(err), chunk_rows),
                  "up_expr_launch_host")
        return err.value

    def __del__(self):
        try:
            abi.load().up_module_release(self._h)
        except Exception:
            pass


def compile_expr(root: Expr, cols: Sequence[ColType], **kw) -> ExprModule:
    b = build([root], cols)
    derive_types(b)
    return ExprModule(b, b.roots[0], **kw)


class QueryModule:
    """A compiled fused expression + grouped aggregate kernel pair."""

    def __init__(self, built: Built, aggs: Sequence[tuple[int, int]]):
        lib = abi.load()
        self.built = built
        self.aggs = list(aggs)
        qa = (abi.UpQueryAgg * len(aggs))()
        for i, (k, r) in enumerate(aggs):
            qa[i].kind = k
            qa[i].root = r
        h = C.c_void_p()
        abi.check(lib.up_query_compile(built.nodes, built.n_nodes, built.col_types, built.n_cols, qa, len(aggs),
                                       None, C.byref(h)), "up_query_compile")
        self._h = h

    def launch(self, cols: Sequence[DeviceColumn], group_ids: torch.Tensor, n_groups: int,
               outs: Sequence[torch.Tensor] | None = None, err: torch.Tensor | None = None,
               stream=None, rows: int | None = None) -> list[torch.Tensor]:
        lib = abi.load()
        if rows is None:
            rows = group_ids.numel()
        if outs is None:
            outs = [torch.empty(n_groups * (8 if k == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES),
                                dtype=torch.uint8, device="cuda") for k, _ in self.aggs]
        optr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        arr = _columns_array(cols)
        abi.check(lib.up_query_launch(self._h, arr, len(cols), rows, group_ids.data_ptr(), n_groups, optr,
                                      err.data_ptr() if err is not None else None, _stream_ptr(stream)),
                  "up_query_launch")
        return list(outs)

    def launch_keys(self, cols: Sequence[DeviceColumn], keys: Sequence[torch.Tensor], key_bytes: Sequence[int],
                    key_table: torch.Tensor, n_groups: int, outs: Sequence[torch.Tensor] | None = None,
                    err: torch.Tensor | None = None, stream=None, rows: int | None = None) -> list[torch.Tensor]:
        """The query with its GROUP BY key columns read by the kernel
        (up_query_launch_keys); key_table / n_groups from group_table_from_keys."""
        lib = abi.load()
        if rows is None:
            rows = keys[0].numel() // key_bytes[0]
        if outs is None:
            outs = [torch.empty(n_groups * (8 if k == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES),
                                dtype=torch.uint8, device="cuda") for k, _ in self.aggs]
        optr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        arr = _columns_array(cols)
        kp = (C.c_void_p * len(keys))(*[k.data_ptr() for k in keys])
        kb = (C.c_int32 * len(keys))(*key_bytes)
        abi.check(lib.up_query_launch_keys(self._h, arr, len(cols), rows, kp, kb, len(keys), key_table.data_ptr(),
                                           n_groups, optr, err.data_ptr() if err is not None else None,
                                           _stream_ptr(stream)), "up_query_launch_keys")
        return list(outs)

    def launch_keys_async(self, cols: Sequence[DeviceColumn], keys: Sequence[torch.Tensor],
                          key_bytes: Sequence[int], key_table: torch.Tensor, max_groups: int,
                          outs: Sequence[torch.Tensor] | None = None, err: torch.Tensor | None = None,
                          stream=None, rows: int | None = None) -> list[torch.Tensor]:
        """The query over key columns with the group count read on the device
        from the key table (up_query_launch_keys_async): no host round trip.
        Outputs hold `max_groups` groups, the first n_groups of them written."""
        lib = abi.load()
        if rows is None:
            rows = keys[0].numel() // key_bytes[0]
        if outs is None:
            outs = [torch.empty(max_groups * (8 if k == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES),
                                dtype=torch.uint8, device="cuda") for k, _ in self.aggs]
        optr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
        arr = _columns_array(cols)
        kp = (C.c_void_p * len(keys))(*[k.data_ptr() for k in keys])
        kb = (C.c_int32 * len(keys))(*key_bytes)
        abi.check(lib.up_query_launch_keys_async(self._h, arr, len(cols), rows, kp, kb, len(keys),
                                                 key_table.data_ptr(), max_groups, optr,
                                                 err.data_ptr() if err is not None else None, _stream_ptr(stream)),
                  "up_query_launch_keys_async")
        return list(outs)

    def __del__(self):
        try:
            abi.load().up_module_release(self._h)
        except Exception:
            pass


def compile_query(exprs: Sequence[Expr], aggs: Sequence[tuple[int, int]], cols: Sequence[ColType]) -> QueryModule:
    """exprs: aggregate expressions; aggs: (kind, index into exprs)."""
    b = build(list(exprs), cols)
    derive_types(b)
    return QueryModule(b, [(k, b.roots[i]) for k, i in aggs])


def group_agg(vals: Sequence[DeviceColumn], kinds: Sequence[int], group_ids: torch.Tensor, n_groups: int,
              err: torch.Tensor | None = None, stream=None) -> list[torch.Tensor]:
    lib = abi.load()
    outs = [torch.empty(n_groups * (8 if k == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES), dtype=torch.uint8,
                        device="cuda") for k in kinds]
    arr = _columns_array(vals)
    karr = (C.c_int32 * len(kinds))(*kinds)
    optr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    abi.check(lib.up_group_agg(arr, karr, len(kinds), group_ids.data_ptr(), n_groups, group_ids.numel(), optr,
                               err.data_ptr() if err is not None else None, _stream_ptr(stream)), "up_group_agg")
    return outs


def gen_digits(rows: int, precision: int, seed: int, signed: bool = True, nonzero: bool = False,
               stream=None) -> torch.Tensor:
    lib = abi.load()
    out = torch.empty(rows * codec.compact_bytes(precision), dtype=torch.uint8, device="cuda")
    abi.check(lib.up_util_gen_digits(out.data_ptr(), rows, precision, seed, 1 if signed else 0,
                                     1 if nonzero else 0, _stream_ptr(stream)), "up_util_gen_digits")
    return out


def gen_range(rows: int, precision: int, lo: int, hi: int, step: int, seed: int, stream=None) -> torch.Tensor:
    lib = abi.load()
    out = torch.empty(rows * codec.compact_bytes(precision), dtype=torch.uint8, device="cuda")
    abi.check(lib.up_util_gen_range(out.data_ptr(), rows, precision, lo, hi, step, seed, _stream_ptr(stream)),
              "up_util_gen_range")
    return out


def group_ids_from_keys(keys: Sequence[torch.Tensor], key_bytes: Sequence[int], stream=None):
    """Dense group ids in key order from fixed-width byte key columns."""
    lib = abi.load()
    rows = keys[0].numel() // key_bytes[0]
    gid = torch.empty(rows, dtype=torch.int32, device="cuda")
    total = sum(key_bytes)
    gkeys = torch.empty(65536 * total, dtype=torch.uint8, device="cuda")
    kp = (C.c_void_p * len(keys))(*[k.data_ptr() for k in keys])
    kb = (C.c_int32 * len(keys))(*key_bytes)
    n = C.c_int32()
    abi.check(lib.up_group_ids_from_keys(kp, kb, len(keys), rows, gid.data_ptr(), C.byref(n), gkeys.data_ptr(),
                                         _stream_ptr(stream)), "up_group_ids_from_keys")
    return gid, n.value, gkeys[: n.value * total]


def group_table_from_keys(keys: Sequence[torch.Tensor], key_bytes: Sequence[int], stream=None,
                          table: torch.Tensor | None = None, distinct: bool = True):
    """The key -> dense group id table (up_group_table_from_keys); returns
    (table, n_groups, distinct keys or None)."""
    lib = abi.load()
    rows = keys[0].numel() // key_bytes[0]
    if table is None:
        table = torch.empty(abi.UP_KEY_TABLE_ENTRIES, dtype=torch.int32, device="cuda")
    total = sum(key_bytes)
    gkeys = torch.empty(65536 * total, dtype=torch.uint8, device="cuda") if distinct else None
    kp = (C.c_void_p * len(keys))(*[k.data_ptr() for k in keys])
    kb = (C.c_int32 * len(keys))(*key_bytes)
    n = C.c_int32()
    abi.check(lib.up_group_table_from_keys(kp, kb, len(keys), rows, table.data_ptr(), C.byref(n),
                                           gkeys.data_ptr() if distinct else None, _stream_ptr(stream)),
              "up_group_table_from_keys")
    return table, n.value, (gkeys[: n.value * total] if distinct else None)


def group_table_from_keys_async(keys: Sequence[torch.Tensor], key_bytes: Sequence[int], table: torch.Tensor,
                                stream=None) -> torch.Tensor:
    """The key table without synchronising (up_group_table_from_keys_async);
    the group count stays on the device at table[UP_KEY_TABLE_COUNT]."""
    lib = abi.load()
    rows = keys[0].numel() // key_bytes[0]
    kp = (C.c_void_p * len(keys))(*[k.data_ptr() for k in keys])
    kb = (C.c_int32 * len(keys))(*key_bytes)
    abi.check(lib.up_group_table_from_keys_async(kp, kb, len(keys), rows, table.data_ptr(), None,
                                                 _stream_ptr(stream)), "up_group_table_from_keys_async")
    return table


def _text_buffers(fields: Sequence[bytes]):
    import numpy as np
    lens = np.fromiter((len(f) for f in fields), dtype=np.int64, count=len(fields))
    offsets = np.zeros(len(fields) + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])
    text = np.frombuffer(b"".join(fields) or b"\0", dtype=np.uint8)
    return torch.from_numpy(text.copy()).cuda(), torch.from_numpy(offsets).cuda()


def parse_decimal(fields: Sequence[bytes], precision: int, scale: int, text: torch.Tensor | None = None,
                  offsets: torch.Tensor | None = None, stream=None):
    """Decimal text -> a compact DECIMAL(precision, scale) column on the GPU
    (up_parse_decimal).  Either byte strings, or device `text` (uint8) and
    `offsets` (int64, rows+1).  Returns (compact uint8 tensor, row-error word)."""
    lib = abi.load()
    if text is None:
        text, offsets = _text_buffers(fields)
    rows = offsets.numel() - 1
    out = torch.empty(max(1, rows * codec.compact_bytes(precision)), dtype=torch.uint8, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    abi.check(lib.up_parse_decimal(text.data_ptr(), offsets.data_ptr(), rows, precision, scale, out.data_ptr(),
                                   err.data_ptr(), _stream_ptr(stream)), "up_parse_decimal")
    return out[:rows * codec.compact_bytes(precision)], int(err.item())


def format_decimal(col: torch.Tensor, rows: int, precision: int, scale: int, hex_image: bool = False,
                   stream=None):
    """A compact column -> (device text slots uint8 [rows, width], lengths int32)
    (up_format_decimal)."""
    lib = abi.load()
    width = lib.up_format_width(precision, 1 if hex_image else 0)
    text = torch.empty((max(1, rows), width), dtype=torch.uint8, device="cuda")
    lens = torch.empty(max(1, rows), dtype=torch.int32, device="cuda")
    abi.check(lib.up_format_decimal(col.data_ptr(), rows, precision, scale, 1 if hex_image else 0, text.data_ptr(),
                                    width, lens.data_ptr(), _stream_ptr(stream)), "up_format_decimal")
    return text[:rows], lens[:rows]


def format_strings(col: torch.Tensor, rows: int, precision: int, scale: int, hex_image: bool = False) -> list:
    """format_decimal, copied back as Python strings."""
    text, lens = format_decimal(col, rows, precision, scale, hex_image)
    t, ln = text.cpu().numpy(), lens.cpu().numpy()
    return [bytes(t[i, :ln[i]]).decode() for i in range(rows)]


def filter_flags(flags: torch.Tensor, rows: int, stream=None) -> torch.Tensor:
    """Indices (int32, in row order) of the rows whose flag byte is nonzero
    (up_filter_flags)."""
    lib = abi.load()
    idx = torch.empty(max(1, rows), dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    abi.check(lib.up_filter_flags(flags.data_ptr(), rows, idx.data_ptr(), cnt.data_ptr(), _stream_ptr(stream)),
              "up_filter_flags")
    return idx[:int(cnt.item())]
