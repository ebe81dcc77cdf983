"""Serving loop (include/ultraprecise_serve.h) for Python callers: a session
that admits decimal requests over resident device columns by memory,
launches them concurrently as they arrive, and reports latency percentiles."""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import torch

from . import abi
from .runtime import DeviceColumn, ExprModule, QueryModule

QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3


class UpServeOpts(C.Structure):
    _fields_ = [("n_streams", C.c_int32), ("max_inflight", C.c_int32), ("memory_cap_bytes", C.c_int64),
                ("reserve_bytes", C.c_int64), ("heavy_work", C.c_double), ("merge", C.c_int32),
                ("max_batch", C.c_int32), ("batch_window_us", C.c_double)]


class UpServeRequest(C.Structure):
    _fields_ = [("module", C.c_void_p), ("in_", C.c_void_p), ("n_in", C.c_int32), ("rows", C.c_int64),
                ("group_ids", C.c_void_p), ("n_groups", C.c_int32), ("arrival_ms", C.c_double)]


class UpServeStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("deferred", C.c_int64),
                ("outstanding_bytes", C.c_int64), ("max_outstanding_bytes", C.c_int64),
                ("budget_bytes", C.c_int64), ("max_inflight_seen", C.c_int32), ("pad", C.c_int32),
                ("p50_ms", C.c_double), ("p95_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("max_ms", C.c_double), ("merged_launches", C.c_int64), ("merged_requests", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class _DevBuf:
    """A device pointer viewed as a torch uint8 tensor (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def percentiles(lat_ms: Sequence[float]):
    """(p50, p95, p99) by the session's rule: the sorted sample at round(f*(n-1))."""
    v = sorted(lat_ms)
    if not v:
        return (0.0, 0.0, 0.0)
    q = lambda f: v[min(len(v) - 1, int(f * (len(v) - 1) + 0.5))]
    return (q(0.50), q(0.95), q(0.99))


class Session:
    def __init__(self, n_streams: int = 0, max_inflight: int = 0, memory_cap_bytes: int = 0,
                 reserve_bytes: int = 0, heavy_work: float = 0.0, merge: bool = False, max_batch: int = 0,
                 batch_window_us: float = 0.0):
        lib = abi.load()
        o = UpServeOpts(n_streams, max_inflight, memory_cap_bytes, reserve_bytes, heavy_work, 1 if merge else 0,
                        max_batch, batch_window_us)
        h = C.c_void_p()
        abi.check(lib.up_serve_create(C.byref(o), C.byref(h)), "up_serve_create")
        self._h = h
        self._keep = {}

    def clock_ms(self) -> float:
        return abi.load().up_serve_clock_ms(self._h)

    def submit(self, module: ExprModule | QueryModule, cols: Sequence[DeviceColumn], rows: int,
               group_ids: torch.Tensor | None = None, n_groups: int = 0, arrival_ms: float = -1.0) -> int:
        lib = abi.load()
        arr = (abi.UpColumn * max(1, len(cols)))(*[c.up_column() for c in cols])
        r = UpServeRequest(module._h.value, C.cast(arr, C.c_void_p), len(cols), rows,
                           group_ids.data_ptr() if group_ids is not None else None, n_groups, arrival_ms)
        rid = C.c_int64()
        abi.check(lib.up_serve_submit(self._h, C.byref(r), C.byref(rid)), "up_serve_submit")
        self._keep[rid.value] = (module, cols, group_ids)
        return rid.value

    def poll(self, rid: int):
        st, lat = C.c_int32(), C.c_double()
        abi.check(abi.load().up_serve_poll(self._h, rid, C.byref(st), C.byref(lat)), "up_serve_poll")
        return st.value, lat.value

    def wait(self, rid: int, timeout_ms: float = -1.0) -> int:
        st = C.c_int32()
        abi.check(abi.load().up_serve_wait(self._h, rid, timeout_ms, C.byref(st)), "up_serve_wait")
        return st.value

    def result(self, rid: int, part: int = 0):
        """(device uint8 tensor view of output `part`, row-error word)."""
        p, n, e = C.c_void_p(), C.c_int64(), C.c_uint32()
        abi.check(abi.load().up_serve_result(self._h, rid, part, C.byref(p), C.byref(n), C.byref(e)),
                  "up_serve_result")
        if n.value == 0:
            return torch.empty(0, dtype=torch.uint8, device="cuda"), e.value
        return torch.as_tensor(_DevBuf(p.value, n.value), device="cuda"), e.value

    def release(self, rid: int) -> None:
        abi.check(abi.load().up_serve_release(self._h, rid), "up_serve_release")
        self._keep.pop(rid, None)

    def stats(self, reset: bool = False) -> dict:
        s = UpServeStats()
        abi.check(abi.load().up_serve_stats_get(self._h, 1 if reset else 0, C.byref(s)), "up_serve_stats_get")
        return s.as_dict()

    def close(self) -> None:
        if self._h:
            abi.load().up_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
