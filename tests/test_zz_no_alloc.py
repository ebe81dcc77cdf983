"""GPU: the no-allocation grouped-aggregate launch.

Callers that cannot allocate device memory at launch time (a host runtime that
owns the whole device memory budget, or a latency-critical path that must not
enter the allocator) use up_query_launch_noalloc, whose accumulators live in
the library's static device array.  Its results must equal the allocating
up_query_launch on the same inputs, on two calls in a row (the array keeps
the previous call's contents, so each call must clear what it uses).
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
