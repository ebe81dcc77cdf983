"""GPU: the no-allocation grouped-aggregate launch.

Callers that cannot allocate device memory at launch time (a host runtime that
owns the whole device memory budget, or a latency-critical path that must not
enter the allocator) use up_query_launch_noalloc, whose accumulators live in
the library's static device array.  Its results must equal the allocating
up_query_launch on the same inputs, on two calls in a row (the array keeps
the previous call's contents, so each call must clear what it uses); with
no rows; at the largest group count the array holds (the next one is
refused); and after a call with more groups than the next one uses.
This file is collected last on purpose.
"""
import ctypes as C

import pytest

torch = pytest.importorskip("torch")

from ultraprecise_b200 import abi, runtime, workloads

pytestmark = pytest.mark.gpu


def _launch_noalloc(q, cols, gid, n_groups, outs, err):
    lib = abi.load()
    arr = (abi.UpColumn * len(cols))(*[c.up_column() for c in cols])
    optr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    return lib.up_query_launch_noalloc(q._h, arr, len(cols), gid.numel(), gid.data_ptr(), n_groups, optr,
                                       err.data_ptr(), torch.cuda.current_stream().cuda_stream)


def test_query_launch_noalloc_matches_allocating_launch():
    rows = 200_003
    exprs, aggs, cols = workloads.query_exprs()
    q = runtime.compile_query(exprs, aggs, cols)
    ranges = workloads.QUERY_RANGES
    data = [runtime.gen_range(rows, 15, *ranges[k], seed=41 + i) for i, k in enumerate(("qty", "price", "disc", "tax"))]
    dev = [runtime.DeviceColumn(t, 15, 2) for t in data]
    n_groups = 1000
    gid = torch.randint(0, n_groups, (rows,), dtype=torch.int32, device="cuda",
                        generator=torch.Generator(device="cuda").manual_seed(3))
    err_ref = torch.zeros(1, dtype=torch.int32, device="cuda")
    ref = q.launch(dev, gid, n_groups, err=err_ref)
    torch.cuda.synchronize()
    ref_bytes = [bytes(o.cpu().numpy().tobytes()) for o in ref]
    for call in range(2):
        outs = [torch.full_like(o, 0xA5) for o in ref]
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        abi.check(_launch_noalloc(q, dev, gid, n_groups, outs, err), "up_query_launch_noalloc")
        torch.cuda.synchronize()
        assert int(err.item()) == int(err_ref.item())
        for k, o in enumerate(outs):
            assert bytes(o.cpu().numpy().tobytes()) == ref_bytes[k], f"call {call}, aggregate {k}"


def test_query_launch_noalloc_rejects_oversized_request():
    exprs, aggs, cols = workloads.query_exprs()
    q = runtime.compile_query(exprs, aggs, cols)
    dev = [runtime.DeviceColumn(torch.zeros(7 * 16, dtype=torch.uint8, device="cuda"), 15, 2) for _ in range(4)]
    gid = torch.zeros(16, dtype=torch.int32, device="cuda")
    n_groups = 1 << 22  # far beyond what the static array holds
    outs = [torch.empty(1, dtype=torch.uint8, device="cuda") for _ in aggs]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = _launch_noalloc(q, dev, gid, n_groups, outs, err)
    assert st == abi.UP_ERR_INVALID_ARG
    assert b"no-alloc scratch too small" in abi.load().up_last_error_message()


def _query_and_columns(rows, seed=41):
    exprs, aggs, cols = workloads.query_exprs()
    q = runtime.compile_query(exprs, aggs, cols)
    ranges = workloads.QUERY_RANGES
    data = [runtime.gen_range(max(rows, 1), 15, *ranges[k], seed=seed + i)
            for i, k in enumerate(("qty", "price", "disc", "tax"))]
    return q, aggs, [runtime.DeviceColumn(t, 15, 2) for t in data]


def _both(q, dev, gid, n_groups, rows):
    """(allocating launch bytes, no-alloc launch bytes) on the same inputs."""
    ref = q.launch(dev, gid, n_groups, rows=rows)
    outs = [torch.full_like(o, 0x5A) for o in ref]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib = abi.load()
    arr = (abi.UpColumn * len(dev))(*[c.up_column() for c in dev])
    optr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    abi.check(lib.up_query_launch_noalloc(q._h, arr, len(dev), rows, gid.data_ptr(), n_groups, optr,
                                          err.data_ptr(), torch.cuda.current_stream().cuda_stream),
              "up_query_launch_noalloc")
    torch.cuda.synchronize()
    return [bytes(o.cpu().numpy().tobytes()) for o in ref], [bytes(o.cpu().numpy().tobytes()) for o in outs]


def _accepts(q, dev, n_groups):
    lib = abi.load()
    gid = torch.zeros(1, dtype=torch.int32, device="cuda")
    outs = [torch.empty(n_groups * 133, dtype=torch.uint8, device="cuda") for _ in range(8)]
    arr = (abi.UpColumn * len(dev))(*[c.up_column() for c in dev])
    optr = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    st = lib.up_query_launch_noalloc(q._h, arr, len(dev), 0, gid.data_ptr(), n_groups, optr, None,
                                     torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return st == abi.UP_OK


def test_query_launch_noalloc_without_rows():
    q, aggs, dev = _query_and_columns(0)
    gid = torch.zeros(1, dtype=torch.int32, device="cuda")
    ref, got = _both(q, dev, gid, 7, 0)
    assert got == ref


def test_query_launch_noalloc_at_the_largest_group_count_then_fewer_groups():
    q, aggs, dev = _query_and_columns(100_000, seed=7)
    lo, hi = 1, 1 << 22  # lo is accepted, hi refused
    assert _accepts(q, dev, lo) and not _accepts(q, dev, hi)
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if _accepts(q, dev, mid):
            lo = mid
        else:
            hi = mid
    n_max = lo
    assert n_max > 1000 and not _accepts(q, dev, n_max + 1)
    rows = 100_000
    g = torch.Generator(device="cuda").manual_seed(9)
    for n_groups in (n_max, 37, 3):  # the array keeps the large call's contents: each call clears its part
        gid = torch.randint(0, n_groups, (rows,), dtype=torch.int32, device="cuda", generator=g)
        ref, got = _both(q, dev, gid, n_groups, rows)
        assert got == ref, n_groups
