"""Build-time JIT prewarm: compile the benchmark's kernels with NVRTC into
the in-tree cubin cache (no GPU needed), so a fresh GPU host loads them
instead of compiling."""
from __future__ import annotations

import ctypes as C

from . import abi, workloads
from . import expr as E


def _compile(roots, cols, aggs=None):
    lib = abi.load()
    b = E.build(roots, cols)
    E.derive_types(b)
    if aggs is None:
        st = lib.up_util_compile_only(b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, 0, None, 0)
    else:
        qa = (abi.UpQueryAgg * len(aggs))()
        for i, (k, r) in enumerate(aggs):
            qa[i].kind = k
            qa[i].root = b.roots[r]
        st = lib.up_util_compile_only(b.nodes, b.n_nodes, 0, b.col_types, b.n_cols, 1, qa, len(aggs))
    abi.check(st, "prewarm compile")


def prewarm(verbose: bool = False) -> None:
    for p, _ in workloads.SWEEP:
        for op in workloads.SWEEP_OPS:
            e, cols = workloads.sweep_expr(p, op)
            _compile([e], cols)
            if verbose:
                print("prewarmed", p, op)
    exprs, aggs, cols = workloads.query_exprs()
    _compile(exprs, cols, aggs)
    from . import batch
    tasks, _ = workloads.batch_tasks()
    batch.compile_only(workloads.batch_specs(tasks))
    if verbose:
        print("prewarmed batch module,", len(tasks), "tasks")


if __name__ == "__main__":
    prewarm(verbose=True)
