"""Build-time JIT prewarm: compile the benchmark's kernels with NVRTC into
the in-tree cubin cache (no GPU needed), so a fresh GPU host loads them
instead of compiling."""
from __future__ import annotations

import ctypes as C

from . import abi, workloads
from . import expr as E


def compile_expr_only(root, cols, threads_per_value: int = 0) -> None:
    """NVRTC-compile one expression module with the given threads per value."""
    lib = abi.load()
    b = E.build([root], cols)
    E.derive_types(b)
    opts = abi.UpCompileOpts(threads_per_value, 0, 0)
    abi.check(lib.up_util_compile_expr_only(b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, C.byref(opts)),
              "compile")


def expr_source(root, cols, threads_per_value: int = 0) -> str:
    """Generated CUDA source of an expression module (CPU only)."""
    lib = abi.load()
    b = E.build([root], cols)
    E.derive_types(b)
    opts = abi.UpCompileOpts(threads_per_value, 0, 0)
    n = lib.up_util_expr_source(b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, C.byref(opts), None, 0)
    if n < 0:
        raise ValueError("expression rejected")
    buf = C.create_string_buffer(int(n) + 1)
    lib.up_util_expr_source(b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, C.byref(opts), buf, n + 1)
    return buf.value.decode()


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
    """Compile every module the benchmarks and GPU tests load, in parallel
    (the library's compile path releases the GIL and is thread-safe)."""
    import concurrent.futures as cf
    import os
    from . import batch
    jobs = []
    for p, _ in workloads.SWEEP:
        for op in workloads.SWEEP_OPS:
            e, cols = workloads.sweep_expr(p, op)
            jobs.append((f"sweep p={p} {op}", [e], cols, None))
    exprs, aggs, cols = workloads.query_exprs()
    jobs.append(("query", exprs, cols, aggs))
    for p, _ in workloads.SIN:
        e, cols = workloads.sin_expr(p)
        jobs.insert(0, (f"sin p={p}", [e], cols, None))  # the longest compiles first
    tasks, _ = workloads.batch_tasks()
    # the plain per-task modules the batched mode is compared against
    for k, t in enumerate(tasks):
        aggs = None if t["agg"] < 0 else [(t["agg"], 0)]
        jobs.append((f"batch task {k} plain", [t["expr"]], t["cols"], aggs))
    workers = max(1, min(32, os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        futs = {ex.submit(_compile, r, c, a): name for name, r, c, a in jobs}
        for f in cf.as_completed(futs):
            f.result()
            if verbose:
                print("prewarmed", futs[f])
    specs = workloads.batch_specs(tasks)
    batch.compile_only(specs)
    batch.compile_only(specs, [1] * len(tasks))  # the one-thread-per-value policy
    # the pinned cooperative configurations of the GPU tests (at their row cap,
    # the tasks of at least 2000 rows also run solo)
    from .expr import ColType  # noqa: F401
    data_rows = [min(t["rows"], 3001) for t in tasks]
    for sizes, solo in (((4, 8, 16, 32), False), ((8, 16), True)):
        tv = workloads.batch_pinned_tpv(tasks, sizes)
        batch.compile_only(specs, tv)
        if solo:
            solo_jobs = [(t["expr"], t["cols"], v) for t, v, r in zip(tasks, tv, data_rows)
                         if t["agg"] < 0 and r >= 2000]
            with cf.ThreadPoolExecutor(max_workers=workers) as ex:
                list(ex.map(lambda j: compile_expr_only(*j), solo_jobs))
    # every candidate the measured threads-per-value policy times
    cand_jobs = [(t["expr"], t["cols"], v) for t, spec in zip(tasks, specs)
                 for v in batch.tpv_candidates(spec) if t["agg"] < 0]
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        list(ex.map(lambda j: compile_expr_only(*j), cand_jobs))
    if verbose:
        print("prewarmed batch modules,", len(tasks), "tasks,", len(cand_jobs), "threads-per-value candidates")
    # the cooperative-evaluation cases of the GPU tests, with their group sizes
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        list(ex.map(lambda c: compile_expr_only(c[2], c[3], c[4]), workloads.coop_cases()))
    if verbose:
        print("prewarmed cooperative cases")
    prewarm_costmodel(workers)
    if verbose:
        print("prewarmed cost-model shapes")


def prewarm_costmodel(workers: int = 8) -> None:
    """Every cost-model training and held-out shape at every threads per value
    (the launches the model is trained and evaluated on)."""
    import concurrent.futures as cf
    shapes = workloads.costmodel_train_shapes() + workloads.costmodel_eval_shapes()
    jobs = [(e, cols, t) for _, e, cols in shapes for t in (1, 2, 4, 8, 16, 32)]
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        list(ex.map(lambda j: compile_expr_only(*j), jobs))


def compress(verbose: bool = False) -> None:
    """Store the in-tree cache gzip-compressed (the JIT reads `<entry>.gz`
    when the plain file is absent), so the library and its prebuilt kernels
    stay small enough to travel."""
    import gzip
    import os
    from . import build as B
    cache = os.path.join(os.path.dirname(os.path.abspath(B.__file__)), "_jitcache")
    before = after = 0
    for name in sorted(os.listdir(cache)):
        if not (name.endswith(".cubin") or name.endswith(".key")):
            continue
        path = os.path.join(cache, name)
        data = open(path, "rb").read()
        with gzip.open(path + ".gz.tmp", "wb", compresslevel=6) as f:
            f.write(data)
        os.replace(path + ".gz.tmp", path + ".gz")
        os.remove(path)
        before += len(data)
        after += os.path.getsize(path + ".gz")
    if verbose:
        print(f"compressed cache: {before / 1e6:.1f} MB -> {after / 1e6:.1f} MB")


def prune(verbose: bool = False) -> None:
    """Rebuild the in-tree cache with only the entries prewarm() uses: the old
    cache seeds a fresh directory, which then replaces it."""
    import os
    import shutil
    import subprocess
    import sys
    from . import build as B
    cache = os.path.join(os.path.dirname(os.path.abspath(B.__file__)), "_jitcache")
    fresh = cache + ".fresh"
    shutil.rmtree(fresh, ignore_errors=True)
    env = dict(os.environ, UP_JIT_CACHE_DIR=fresh, UP_JIT_CACHE_SEED_DIR=cache)
    subprocess.run([sys.executable, "-m", "ultraprecise_b200.prewarm"] + (["-v"] if verbose else []), env=env,
                   check=True)
    shutil.rmtree(cache)
    os.rename(fresh, cache)


if __name__ == "__main__":
    import sys
    try:
        # The benchmark and test processes import torch before the library,
        # so they run torch's NVRTC; compiling with the same one keeps the
        # cache keys (which name the NVRTC version) theirs.
        import torch  # noqa: F401
    except ImportError:
        pass
    if "--prune" in sys.argv:
        prune(verbose="-v" in sys.argv)
    elif "--compress" in sys.argv:
        compress(verbose=True)
    else:
        prewarm(verbose=True)
