"""The learned cost model (include/ultraprecise_costmodel.h) from Python.

A small perceptron that predicts log(ms) of an expression launch; it is
trained on the GPU by the library's own kernels on launch times measured on
the device (collect_samples), and chooses the threads per value of an
expression by the lowest predicted time.  It never changes a result.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from typing import Sequence

import numpy as np

from . import abi
from . import expr as E

FEATURES = 16
HIDDEN = 64
PARAMS = FEATURES * HIDDEN + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN + 1
BATCH_MAX = 128
TPV_CHOICES = (1, 2, 4, 8, 16, 32)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def features(root: E.Expr, cols: Sequence[E.ColType], tpv: int, rows: int):
    """(feature vector, whether the expression has a cooperative form)."""
    lib = abi.load()
    b = E.build([root], cols)
    E.derive_types(b)
    out = np.zeros(FEATURES, dtype=np.float32)
    ok = C.c_int32(0)
    abi.check(lib.up_costmodel_expr_features(b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, tpv, rows,
                                             _fptr(out), C.byref(ok)), "up_costmodel_expr_features")
    return out, bool(ok.value)


def rule_tpv(root: E.Expr, cols: Sequence[E.ColType], use_model: bool = False) -> int:
    """Threads per value of an automatic compile (no GPU): the width rule, or
    the default cost model's choice when use_model and one is set."""
    lib = abi.load()
    b = E.build([root], cols)
    E.derive_types(b)
    t = C.c_int32(1)
    abi.check(lib.up_util_auto_tpv(b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, 1 if use_model else 0,
                                   C.byref(t)), "up_util_auto_tpv")
    return t.value


class CostModel:
    def __init__(self, seed: int = 0):
        lib = abi.load()
        h = C.c_void_p()
        abi.check(lib.up_costmodel_create(seed, C.byref(h)), "up_costmodel_create")
        self._h = h

    def train(self, X: np.ndarray, y: np.ndarray, epochs: int = 400, batch: int = 64, lr: float = 3e-3,
              seed: int = 1) -> float:
        """Train on features X [n, 16] and targets y = log(ms); returns the
        final mean squared error in standardised units."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = C.c_float(0)
        abi.check(abi.load().up_costmodel_train(self._h, _fptr(X), _fptr(y), len(y), epochs, batch, lr, seed,
                                                C.byref(loss)), "up_costmodel_train")
        return float(loss.value)

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, FEATURES)
        out = np.zeros(len(X), dtype=np.float32)
        abi.check(abi.load().up_costmodel_predict(self._h, _fptr(X), len(X), _fptr(out)), "up_costmodel_predict")
        return out

    def gradients(self, X: np.ndarray, y: np.ndarray):
        """Gradients of the mean squared error of the raw network (no
        standardisation) at the current parameters, from the GPU kernel."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = np.zeros(PARAMS, dtype=np.float32)
        loss = C.c_float(0)
        abi.check(abi.load().up_costmodel_gradients(self._h, _fptr(X), _fptr(y), len(y), _fptr(g), C.byref(loss)),
                  "up_costmodel_gradients")
        return g, float(loss.value)

    def params(self):
        p = np.zeros(PARAMS, dtype=np.float32)
        norm = np.zeros(2 * FEATURES + 2, dtype=np.float32)
        abi.check(abi.load().up_costmodel_get_params(self._h, _fptr(p), _fptr(norm)), "up_costmodel_get_params")
        return p, norm

    def set_params(self, params: np.ndarray, norm: np.ndarray | None = None) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        n = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        abi.check(abi.load().up_costmodel_set_params(self._h, _fptr(p), None if n is None else _fptr(n)),
                  "up_costmodel_set_params")

    def choose_tpv(self, root: E.Expr, cols: Sequence[E.ColType], rows: int):
        """(threads per value of the lowest predicted time, predicted ms)."""
        lib = abi.load()
        b = E.build([root], cols)
        E.derive_types(b)
        t = C.c_int32(1)
        ms = C.c_float(0)
        abi.check(lib.up_costmodel_choose_tpv(self._h, b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, rows,
                                              C.byref(t), C.byref(ms)), "up_costmodel_choose_tpv")
        return t.value, float(ms.value)

    def add_member(self, other: "CostModel") -> None:
        """Average this model's predictions with a copy of `other`'s network."""
        abi.check(abi.load().up_costmodel_add_member(self._h, other._h), "up_costmodel_add_member")

    def set_guard(self, margin: float) -> None:
        """Keep the width rule's choice unless at least `margin` of its time
        is predicted saved."""
        abi.check(abi.load().up_costmodel_set_guard(self._h, margin), "up_costmodel_set_guard")

    def set_default(self) -> None:
        """Make this model the one up_module_compile uses for automatic
        threads per value."""
        abi.check(abi.load().up_costmodel_set_default(self._h), "up_costmodel_set_default")

    @staticmethod
    def clear_default() -> None:
        abi.check(abi.load().up_costmodel_set_default(None), "up_costmodel_set_default")

    def __del__(self):
        try:
            abi.load().up_costmodel_release(self._h)
        except Exception:
            pass


def time_launch(module, cols, rows: int, reps: int = 3, stream=None) -> float:
    """Median device time (ms) of launching a compiled expression module over
    resident columns, with CUDA events on the launching stream."""
    import torch
    s = stream or torch.cuda.current_stream()
    out = torch.empty(max(1, rows * module.value_bytes), dtype=torch.uint8, device="cuda")
    module.launch(cols, rows, out=out, stream=s)  # warm-up (and first-launch costs)
    times = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        module.launch(cols, rows, out=out, stream=s)
        e1.record(s)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    return sorted(times)[len(times) // 2]


def collect_samples(shapes, rows_list: Sequence[int], seed: int = 7, reps: int = 3, tpvs=TPV_CHOICES,
                    max_bytes: int = 1 << 30):
    """Measure every (shape, threads per value, rows) launch on the device:
    shapes are (name, expr, column types); inputs are seeded digit columns
    kept resident.  Returns (features [n, 16], log ms [n], records)."""
    import torch
    from . import codec, runtime
    X, y, recs = [], [], []
    t0 = time.perf_counter()
    for si, (name, e, cols) in enumerate(shapes):
        p = cols[0].precision
        vb = codec.compact_bytes(p)
        rmax = max(r for r in rows_list if r * vb * len(cols) <= max_bytes) if any(
            r * vb * len(cols) <= max_bytes for r in rows_list) else min(rows_list)
        data = [runtime.DeviceColumn(runtime.gen_digits(rmax, p, seed + 31 * si + k, nonzero=True), p,
                                     cols[k].scale) for k in range(len(cols))]
        _, coop = features(e, cols, 1, rmax)
        for tpv in (tpvs if coop else (1,)):
            m = runtime.compile_expr(e, cols, threads_per_value=tpv)
            for rows in rows_list:
                if rows > rmax:
                    continue
                ms = time_launch(m, data, rows, reps)
                f, _ = features(e, cols, tpv, rows)
                X.append(f)
                y.append(math.log(max(ms, 1e-4)))
                recs.append({"shape": name, "p": p, "tpv": tpv, "rows": rows, "ms": ms})
        del data
        torch.cuda.empty_cache()
    return np.array(X, dtype=np.float32), np.array(y, dtype=np.float32), recs, time.perf_counter() - t0
