"""Batched persistent-kernel mode (include/ultraprecise_batch.h) for Python
callers: many decimal tasks in one module, one graph launch per step."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import torch

from . import abi
from .expr import ColType, Expr, build, derive_types
from .runtime import DeviceColumn, _stream_ptr


class UpBatchTask(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("n_nodes", C.c_int32), ("root", C.c_int32), ("cols", C.c_void_p),
                ("n_cols", C.c_int32), ("agg_kind", C.c_int32)]


class UpBatchOpts(C.Structure):
    _fields_ = [("autotune", C.c_int32), ("block_threads", C.c_int32), ("ctas_per_sm", C.c_int32),
                ("tile_rows", C.c_int32), ("use_graph", C.c_int32), ("tpv_policy", C.c_int32),
                ("solo_rows", C.c_int64)]


@dataclass
class TaskSpec:
    expr: Expr
    cols: Sequence[ColType]
    agg_kind: int = -1     # -1 projection, else abi.UP_AGG_*


def task_array(tasks: Sequence[TaskSpec]):
    """ctypes up_batch_task array (and the Built objects it points into)."""
    built = []
    arr = (UpBatchTask * len(tasks))()
    for i, t in enumerate(tasks):
        b = build([t.expr], t.cols)
        derive_types(b)
        built.append(b)
        arr[i].nodes = C.cast(b.nodes, C.c_void_p)
        arr[i].n_nodes = b.n_nodes
        arr[i].root = b.roots[0]
        arr[i].cols = C.cast(b.col_types, C.c_void_p)
        arr[i].n_cols = b.n_cols
        arr[i].agg_kind = t.agg_kind
    return arr, built


# threads-per-value policies of projection tasks (up_batch_opts.tpv_policy)
TPV_AUTO, TPV_ONE, TPV_MEASURED = 0, 1, 2


def compile_only(tasks: Sequence[TaskSpec], tpv: Sequence[int] | None = None) -> None:
    """NVRTC-compile the batch module into the cubin cache (no GPU needed);
    tpv: each task's threads per value (None: the automatic choice)."""
    arr, built = task_array(tasks)
    tv = None if tpv is None else (C.c_int32 * len(tasks))(*tpv)
    abi.check(abi.load().up_util_compile_batch_only(arr, len(tasks), tv), "up_util_compile_batch_only")


def tpv_candidates(task: TaskSpec):
    """Threads per value the measured policy times for a task."""
    arr, built = task_array([task])
    out = (C.c_int32 * 8)()
    n = abi.load().up_util_batch_tpv_candidates(arr, out, 8)
    if n < 0:
        raise ValueError("bad task")
    return list(out[:n])


class Batch:
    def __init__(self, tasks: Sequence[TaskSpec], autotune: bool = False, use_graph: bool = True,
                 block_threads: int = 0, ctas_per_sm: int = 0, tile_rows: int = 0, solo_rows: int = 0,
                 tpv_policy: int = TPV_AUTO):
        lib = abi.load()
        self.specs = list(tasks)
        arr, self.built = task_array(tasks)
        opts = UpBatchOpts(1 if autotune else 0, block_threads, ctas_per_sm, tile_rows, 1 if use_graph else 0,
                           tpv_policy, solo_rows)
        h = C.c_void_p()
        abi.check(lib.up_batch_create(arr, len(tasks), C.byref(opts), C.byref(h)), "up_batch_create")
        self._h = h
        self._keep = {}

    def task_type(self, k: int):
        """(precision, scale, value_bytes, band) of task k."""
        lib = abi.load()
        p, s, vb, band = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        abi.check(lib.up_batch_task_type(self._h, k, C.byref(p), C.byref(s), C.byref(vb), C.byref(band)),
                  "up_batch_task_type")
        return p.value, s.value, vb.value, band.value

    def bind(self, k: int, cols: Sequence[DeviceColumn], rows: int, out: torch.Tensor,
             group_ids: torch.Tensor | None = None, n_groups: int = 0):
        lib = abi.load()
        arr = (abi.UpColumn * len(cols))(*[c.up_column() for c in cols])
        abi.check(lib.up_batch_bind(self._h, k, arr, len(cols), rows,
                                    group_ids.data_ptr() if group_ids is not None else None, n_groups,
                                    out.data_ptr()), "up_batch_bind")
        self._keep[k] = (cols, out, group_ids)

    def launch(self, err: torch.Tensor | None = None, stream=None):
        lib = abi.load()
        abi.check(lib.up_batch_launch(self._h, err.data_ptr() if err is not None else None, _stream_ptr(stream)),
                  "up_batch_launch")

    def set_task_tpv(self, k: int, threads_per_value: int) -> None:
        """Pin task k's threads per value (projection tasks; rebuilt on the next launch)."""
        abi.check(abi.load().up_batch_set_task_tpv(self._h, k, threads_per_value), "up_batch_set_task_tpv")

    def task_tpv(self, k: int) -> int:
        """Threads per value task k runs with."""
        t = C.c_int32()
        abi.check(abi.load().up_batch_task_tpv(self._h, k, C.byref(t)), "up_batch_task_tpv")
        return t.value

    def shape(self, band: int):
        lib = abi.load()
        t, c, r, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        abi.check(lib.up_batch_shape(self._h, band, C.byref(t), C.byref(c), C.byref(r), C.byref(ms)),
                  "up_batch_shape")
        return {"block_threads": t.value, "ctas_per_sm": c.value, "tile_rows": r.value, "tuned_ms": ms.value}

    def __del__(self):
        try:
            abi.load().up_batch_release(self._h)
        except Exception:
            pass
