"""GPU tests of the serving loop: results in a concurrent mix are byte-equal to
each query run alone through the plain launch path, admission keeps the
outstanding memory under the cap, and the latency report is consistent."""
import pytest

torch = pytest.importorskip("torch")

from ultraprecise_b200 import abi, runtime, serve, workloads
from ultraprecise_b200 import expr as E

pytestmark = pytest.mark.gpu


def _shapes():
    """Resident columns and modules of four request shapes (narrow and wide
    expressions, a division, a grouped query)."""
    shapes = []
    for p, op, rows in ((18, "mad", 200_000), (76, "div", 50_000), (300, "mad", 20_000)):
        e, cols = workloads.sweep_expr(p, op)
        m = runtime.compile_expr(e, cols)
        dev = [runtime.DeviceColumn(runtime.gen_digits(rows, p, 50 + p + k, nonzero=(op == "div" and k == 1)),
                                    p, p // 4) for k in range(len(cols))]
        shapes.append({"mod": m, "cols": dev, "rows": rows, "gid": None, "G": 0})
    exprs, aggs, ct = workloads.query_exprs()
    q = runtime.compile_query(exprs, aggs, ct)
    rows = 300_000
    R = workloads.QUERY_RANGES
    dev = [runtime.DeviceColumn(runtime.gen_range(rows, 15, *R[n], 7 + i), 15, 2)
           for i, n in enumerate(("qty", "price", "disc", "tax"))]
    gid = torch.randint(0, 37, (rows,), dtype=torch.int32, device="cuda",
                        generator=torch.Generator(device="cuda").manual_seed(5))
    shapes.append({"mod": q, "cols": dev, "rows": rows, "gid": gid, "G": 37, "n_parts": len(aggs)})
    for s in shapes:  # each alone through the plain path, with its row-error word
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        if s["gid"] is None:
            s["alone"] = [bytes(s["mod"].launch(s["cols"], s["rows"], err=err).cpu().numpy().tobytes())]
        else:
            outs = s["mod"].launch(s["cols"], s["gid"], s["G"], err=err)
            s["alone"] = [bytes(o.cpu().numpy().tobytes()) for o in outs]
        torch.cuda.synchronize()
        s["err"] = int(err.item())
    return shapes


@pytest.fixture(scope="module")
def shapes():
    return _shapes()


def test_mixed_requests_match_alone(shapes):
    sess = serve.Session(n_streams=4)
    ids = []
    for i in range(120):
        s = shapes[(i * 7) % len(shapes)]
        ids.append((sess.submit(s["mod"], s["cols"], s["rows"], s["gid"], s["G"]), s))
    for rid, s in ids:
        assert sess.wait(rid, 60_000) == serve.DONE
        for part in range(s.get("n_parts", 1)):
            out, err = sess.result(rid, part)
            assert err == s["err"]  # e.g. the p=76 quotient overflows DECIMAL(24,23) when a/b >= 10
            assert bytes(out.cpu().numpy().tobytes()) == s["alone"][part]
        st, lat = sess.poll(rid)
        assert st == serve.DONE and lat >= 0
        sess.release(rid)
    st = sess.stats()
    assert st["submitted"] == st["completed"] == 120 and st["failed"] == 0
    assert 0 <= st["p50_ms"] <= st["p95_ms"] <= st["p99_ms"] <= st["max_ms"]
    assert st["max_inflight_seen"] >= 2  # requests overlapped
    assert st["outstanding_bytes"] == 0
    sess.close()


def test_admission_respects_memory_cap(shapes):
    s = shapes[2]  # the p=300 expression: ~250 B per row of output
    one = s["rows"] * s["mod"].value_bytes + 256
    cap = 3 * one + 1024
    sess = serve.Session(n_streams=4, memory_cap_bytes=cap)
    pending = [sess.submit(s["mod"], s["cols"], s["rows"]) for _ in range(12)]
    done = 0
    while pending:
        rid = pending.pop(0)
        assert sess.wait(rid, 60_000) == serve.DONE
        out, _ = sess.result(rid)
        assert bytes(out.cpu().numpy().tobytes()) == s["alone"][0]
        sess.release(rid)  # frees room for the next admission
        done += 1
    st = sess.stats()
    assert done == 12 and st["completed"] == 12
    assert st["max_outstanding_bytes"] <= cap
    assert st["deferred"] >= 1
    assert st["budget_bytes"] == cap
    sess.close()


def test_request_larger_than_budget_is_refused(shapes):
    s = shapes[0]
    sess = serve.Session(memory_cap_bytes=4096)
    with pytest.raises(abi.UpError) as ei:
        sess.submit(s["mod"], s["cols"], s["rows"])
    assert ei.value.status == abi.UP_ERR_NO_MEMORY
    sess.close()


def test_merged_launch_matches_requests_alone(shapes):
    """up_expr_launch_many: several requests of one module in one kernel
    (different row counts, an empty request, offset column bases) give the
    bytes and row errors of each request launched alone."""
    import ctypes as C
    s = shapes[1]  # p=76 division: row errors occur (quotients that overflow the result type)
    lib = abi.load()
    vb = s["cols"][0].value_bytes
    reqs = [(0, s["rows"]), (17, 1000), (5, 0), (123, 20_000), (1, 333)]  # (first row, rows)
    ins, rows, outs, errs, alone = [], [], [], [], []
    for r0, n in reqs:
        cols = [runtime.DeviceColumn(c.data[r0 * vb:], c.precision, c.scale) for c in s["cols"]]
        ins += [c.up_column() for c in cols]
        rows.append(n)
        outs.append(torch.full((max(1, n * s["mod"].value_bytes),), 0x3C, dtype=torch.uint8, device="cuda"))
        errs.append(torch.zeros(1, dtype=torch.int32, device="cuda"))
        e1 = torch.zeros(1, dtype=torch.int32, device="cuda")
        alone.append((bytes(s["mod"].launch(cols, n, err=e1).cpu().numpy().tobytes()) if n else b"", e1))
    arr = (abi.UpColumn * len(ins))(*ins)
    rr = (C.c_int64 * len(rows))(*rows)
    oo = (C.c_void_p * len(outs))(*[o.data_ptr() for o in outs])
    ee = (C.c_void_p * len(errs))(*[e.data_ptr() for e in errs])
    abi.check(lib.up_expr_launch_many(s["mod"]._h, arr, len(s["cols"]), rr, len(reqs), oo, ee,
                                      torch.cuda.current_stream().cuda_stream), "up_expr_launch_many")
    torch.cuda.synchronize()
    for (r0, n), o, e, (a, ae) in zip(reqs, outs, errs, alone):
        assert bytes(o[:n * s["mod"].value_bytes].cpu().numpy().tobytes()) == a
        assert int(e.item()) == int(ae.item())


def test_session_merges_same_module_requests(shapes):
    """With merging on and a batching window, requests of one expression
    module admitted together run as merged launches; every result still
    equals the request run alone."""
    sess = serve.Session(n_streams=4, merge=True, batch_window_us=2000.0)
    ids = []
    for i in range(60):
        s = shapes[i % 3]  # expression shapes only
        ids.append((sess.submit(s["mod"], s["cols"], s["rows"]), s))
    for rid, s in ids:
        assert sess.wait(rid, 60_000) == serve.DONE
        out, err = sess.result(rid, 0)
        assert err == s["err"]
        assert bytes(out.cpu().numpy().tobytes()) == s["alone"][0]
        sess.release(rid)
    st = sess.stats()
    assert st["completed"] == 60 and st["failed"] == 0
    assert st["merged_launches"] >= 1 and st["merged_requests"] >= 2
    sess.close()
