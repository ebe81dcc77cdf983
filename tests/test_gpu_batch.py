"""GPU parity of the batched persistent-kernel mode (include/ultraprecise_batch.h):
every task's output is byte-identical to the oracle and to the same task run
alone through the plain per-expression / per-query launch path, across graph
replays, the non-graph path and autotuned launch shapes."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from ultraprecise_b200 import abi, batch, codec, runtime, workloads
from ultraprecise_b200 import expr as E

pytestmark = pytest.mark.gpu

ROW_CAP = 3001  # the bench's 64 tasks at a size the oracle checks in seconds


def _bind_all(b, tasks, data):
    outs, gids = [], []
    for k, (t, (rows, cols, gid)) in enumerate(zip(tasks, data)):
        dev = [runtime.DeviceColumn(c, t["p"], t["s"]) for c in cols]
        if t["agg"] < 0:
            _, _, vb, _ = b.task_type(k)
            out = torch.empty(max(1, rows * vb), dtype=torch.uint8, device="cuda")
            b.bind(k, dev, rows, out)
            gids.append(None)
        else:
            g = torch.from_numpy(gid).cuda()
            width = 8 if t["agg"] == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES
            out = torch.empty(max(1, t["groups"] * width), dtype=torch.uint8, device="cuda")
            b.bind(k, dev, rows, out, g, t["groups"])
            gids.append(g)
        outs.append(out)
    return outs, gids


def _expected(b, tasks, data):
    """Oracle bytes per task (and the OR of the oracle's error words)."""
    exp, err = [], 0
    for k, (t, (rows, cols, gid)) in enumerate(zip(tasks, data)):
        built = b.built[k]
        raws = [bytes(c.cpu().numpy().tobytes()) for c in cols]
        if t["agg"] < 0:
            _, _, vb, _ = b.task_type(k)
            o, e = oracle.eval_expr(built, built.roots[0], raws, rows, vb, threads=8)
            exp.append(o)
            err |= e
        else:
            exp.append(oracle.query(built, [(t["agg"], built.roots[0])], raws, gid.tobytes(), rows, t["groups"],
                                    threads=8)[0])
            if t["agg"] != abi.UP_AGG_COUNT:  # the aggregated expression's row errors (e.g. a zero divisor)
                vb = codec.compact_bytes(built.nodes[built.roots[0]].precision)
                err |= oracle.eval_expr(built, built.roots[0], raws, rows, vb, threads=8)[1]
    return exp, err


def _host(outs, tasks, data, b):
    res = []
    for k, (t, (rows, _, _)) in enumerate(zip(tasks, data)):
        if t["agg"] < 0:
            _, _, vb, _ = b.task_type(k)
            res.append(bytes(outs[k][:rows * vb].cpu().numpy().tobytes()))
        else:
            width = 8 if t["agg"] == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES
            res.append(bytes(outs[k][:t["groups"] * width].cpu().numpy().tobytes()))
    return res


@pytest.fixture(scope="module")
def bench_batch():
    tasks, _ = workloads.batch_tasks()
    data = workloads.batch_columns(tasks, seed=7, row_cap=ROW_CAP)
    b = batch.Batch(workloads.batch_specs(tasks), use_graph=True)
    exp, exp_err = _expected(b, tasks, data)
    return tasks, data, b, exp, exp_err


def test_bench_tasks_match_oracle_across_replays(bench_batch):
    tasks, data, b, exp, exp_err = bench_batch
    outs, _ = _bind_all(b, tasks, data)
    bands = {b.task_type(k)[3] for k in range(len(tasks))}
    assert bands == {0, 1, 2}, "the bench batch spans every precision band"
    for rep in range(3):
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        for o in outs:
            o.fill_(0xA5)
        b.launch(err)
        torch.cuda.synchronize()
        got = _host(outs, tasks, data, b)
        for k in range(len(tasks)):
            assert got[k] == exp[k], f"replay {rep}: task {k} (p={tasks[k]['p']}, agg={tasks[k]['agg']})"
        assert int(err.item()) == exp_err


def test_bench_tasks_without_graph_and_with_forced_shapes(bench_batch):
    tasks, data, _, exp, exp_err = bench_batch
    specs = workloads.batch_specs(tasks)
    for kw in ({"use_graph": False}, {"block_threads": 64, "ctas_per_sm": 1, "tile_rows": 256},
               {"block_threads": 256, "ctas_per_sm": 8, "tile_rows": 4096},
               {"solo_rows": 2000}, {"solo_rows": 2000, "use_graph": False}, {"solo_rows": -1}):
        b = batch.Batch(specs, **kw)
        outs, _ = _bind_all(b, tasks, data)
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        b.launch(err)
        b.launch(err)
        torch.cuda.synchronize()
        got = _host(outs, tasks, data, b)
        for k in range(len(tasks)):
            assert got[k] == exp[k], f"{kw}: task {k}"
        assert int(err.item()) == exp_err


def test_bench_tasks_match_plain_path(bench_batch):
    """Each task alone through up_expr_launch / up_query_launch gives the same bytes."""
    tasks, data, b, exp, _ = bench_batch
    for k, (t, (rows, cols, gid)) in enumerate(zip(tasks, data)):
        dev = [runtime.DeviceColumn(c, t["p"], t["s"]) for c in cols]
        if t["agg"] < 0:
            m = runtime.compile_expr(t["expr"], t["cols"])
            got = bytes(m.launch(dev, rows).cpu().numpy().tobytes())
        else:
            q = runtime.compile_query([t["expr"]], [(t["agg"], 0)], t["cols"])
            got = bytes(q.launch(dev, torch.from_numpy(gid).cuda(), t["groups"])[0].cpu().numpy().tobytes())
        assert got == exp[k], f"task {k}"


def _small_tasks():
    """Narrow tasks covering AVG, COUNT, a comparison root, an empty task and
    a task with more groups than rows."""
    c15 = [E.ColType(15, 2)] * 3
    c30 = [E.ColType(30, 7), E.ColType(30, 7)]
    a, b_, c = E.col(0), E.col(1), E.col(2)
    return [
        (batch.TaskSpec(a * b_ + c, c15, abi.UP_AGG_AVG), 5000, 7),
        (batch.TaskSpec(a - b_, c15, abi.UP_AGG_COUNT), 4099, 3),
        (batch.TaskSpec(E.Expr(abi.UP_NODE_LT, a, b_), c30, -1), 6000, 0),
        (batch.TaskSpec(a / b_, c30, -1), 0, 0),
        (batch.TaskSpec(a / b_, c30, abi.UP_AGG_SUM), 50, 200),
        (batch.TaskSpec(a * b_, c30, abi.UP_AGG_AVG), 1, 1),
    ]


def test_small_tasks_avg_count_compare_empty(tmp_path, monkeypatch):
    monkeypatch.setenv("UP_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    specs = _small_tasks()
    tasks, data = [], []
    for k, (spec, rows, groups) in enumerate(specs):
        p, s = spec.cols[0].precision, spec.cols[0].scale
        cols = [runtime.gen_digits(rows, p, 100 + 10 * k + i, signed=True, nonzero=True) if rows else
                torch.zeros(codec.compact_bytes(p), dtype=torch.uint8, device="cuda") for i in range(len(spec.cols))]
        gid = workloads.batch_group_ids(rows, groups, 5 + k) if spec.agg_kind >= 0 else None
        tasks.append({"expr": spec.expr, "cols": spec.cols, "p": p, "s": s, "agg": spec.agg_kind, "groups": groups})
        data.append((rows, cols, gid))
    for autotune in (False, True):
        b = batch.Batch([s for s, _, _ in specs], autotune=autotune)
        exp, exp_err = _expected(b, tasks, data)
        outs, _ = _bind_all(b, tasks, data)
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        b.launch(err)
        b.launch(err)
        torch.cuda.synchronize()
        got = _host(outs, tasks, data, b)
        for k in range(len(tasks)):
            assert got[k] == exp[k], f"autotune={autotune}: task {k}"
        assert int(err.item()) == exp_err
        if autotune:
            for band in range(3):
                sh = b.shape(band)
                assert sh["block_threads"] in (64, 128, 256) and sh["ctas_per_sm"] >= 1 and sh["tile_rows"] >= 1


def test_rebind_changes_rows():
    """Rebinding a task after a launch re-captures the step with the new sizes."""
    specs = [s for s, _, _ in _small_tasks()][:2]
    b = batch.Batch(specs)
    c15 = 15
    results = []
    for rows in (1000, 3000):
        cols = [runtime.gen_digits(rows, c15, 900 + i, nonzero=True) for i in range(3)]
        dev = [runtime.DeviceColumn(c, 15, 2) for c in cols]
        gid = torch.from_numpy(workloads.batch_group_ids(rows, 7, 1)).cuda()
        o0 = torch.empty(7 * abi.UP_AGG_DECIMAL_BYTES, dtype=torch.uint8, device="cuda")
        o1 = torch.empty(7 * 8, dtype=torch.uint8, device="cuda")
        b.bind(0, dev, rows, o0, gid, 7)
        b.bind(1, dev, rows, o1, gid, 7)
        b.launch()
        torch.cuda.synchronize()
        counts = np.frombuffer(o1.cpu().numpy().tobytes(), dtype=np.int64)
        assert int(counts.sum()) == rows
        results.append(bytes(o0.cpu().numpy().tobytes()))
    assert results[0] != results[1]


def _wide_projections(tasks):
    """Projection tasks of the bench batch wide enough for cooperative threads."""
    return [k for k, t in enumerate(tasks) if t["agg"] < 0 and t["p"] > 120]


def test_bench_tasks_with_pinned_threads_per_value(bench_batch):
    """Projection tasks run cooperatively inside the band kernels (and as solo
    kernels) with every group size: the bytes stay the oracle's."""
    tasks, data, _, exp, exp_err = bench_batch
    specs = workloads.batch_specs(tasks)
    wide = _wide_projections(tasks)
    assert len(wide) >= 4
    for kw, sizes in (({}, (4, 8, 16, 32)), ({"solo_rows": 2000}, (8, 16))):
        b = batch.Batch(specs, tpv_policy=batch.TPV_ONE, **kw)
        for k, t in enumerate(workloads.batch_pinned_tpv(tasks, sizes)):
            if t > 1:
                b.set_task_tpv(k, t)
        outs, _ = _bind_all(b, tasks, data)
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        b.launch(err)
        b.launch(err)
        torch.cuda.synchronize()
        assert any(b.task_tpv(k) > 1 for k in wide)
        got = _host(outs, tasks, data, b)
        for k in range(len(tasks)):
            assert got[k] == exp[k], f"{kw}: task {k} at {b.task_tpv(k)} threads per value"
        assert int(err.item()) == exp_err


def test_measured_threads_per_value_policy(bench_batch, tmp_path, monkeypatch):
    """The measured policy times each projection task at its candidate group
    sizes, keeps one of them, caches the choice, and the bytes stay the
    oracle's; a second batch reads the cached choices."""
    monkeypatch.setenv("UP_AUTOTUNE_CACHE", str(tmp_path / "autotune.txt"))
    tasks, data, _, exp, exp_err = bench_batch
    specs = workloads.batch_specs(tasks)
    chosen = []
    for _ in range(2):
        b = batch.Batch(specs, tpv_policy=batch.TPV_MEASURED)
        outs, _ = _bind_all(b, tasks, data)
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        b.launch(err)
        torch.cuda.synchronize()
        got = _host(outs, tasks, data, b)
        for k in range(len(tasks)):
            assert got[k] == exp[k], f"task {k} at {b.task_tpv(k)} threads per value"
        assert int(err.item()) == exp_err
        chosen.append([b.task_tpv(k) for k in range(len(tasks))])
        assert all(chosen[-1][k] == 1 for k in range(len(tasks)) if tasks[k]["agg"] >= 0)
    assert chosen[0] == chosen[1]
    assert "tpv " in (tmp_path / "autotune.txt").read_text()
