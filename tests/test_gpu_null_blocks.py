"""GPU: the full kernel input descriptor of the reference
(AriesColumnDataIterator, AriesColumnDataIterator.cu:60-115) and NULLs.

* Block lists: a column's rows spread over several device buffers (row
  prefix sums, the iterator's binary search); projections and grouped
  queries give the bytes of the same rows held contiguously.
* Nullable values (a flag byte before each value, 0 = NULL,
  AriesExprCalcNode.cpp:1411-1413): a projection's result is NULL when any
  of its columns is; SUM/AVG of an expression skip the rows where it is NULL
  and a group with none has SUM and AVG flag 0 (agg_sum_t on nullable_type,
  operators.hxx:1176-1193); COUNT is the group's row count (COUNT(*)).
  Checked against the oracle, which restates those rules.
* A -1 row index on a column that is not nullable is a domain error.
"""
import random

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from ultraprecise_b200 import abi, codec, runtime, workloads
from ultraprecise_b200 import expr as E

pytestmark = pytest.mark.gpu


def _split_blocks(raw: bytes, vb: int, rng: random.Random, n_blocks: int):
    rows = len(raw) // vb
    cuts = sorted(rng.sample(range(1, rows), n_blocks - 1)) if rows > n_blocks else []
    edges = [0] + cuts + [rows]
    return [torch.frombuffer(bytearray(raw[a * vb:b * vb] or b"\0"), dtype=torch.uint8).cuda()[:(b - a) * vb]
            for a, b in zip(edges, edges[1:])]


def _nullable_raw(vals, p, rng, null_frac, force_null_rows=()):
    """flag byte + compact value per row; NULL rows keep random value bytes
    (they must not be read)."""
    nb = codec.compact_bytes(p)
    out, flags = bytearray(), []
    for i, v in enumerate(vals):
        is_null = i in force_null_rows or rng.random() < null_frac
        flags.append(0 if is_null else 1)
        out.append(0 if is_null else 1)
        out += codec.encode([v], p) if not is_null else bytes(rng.getrandbits(8) for _ in range(nb))
    return bytes(out), flags


def _vals(rng, p, n, nonzero=False):
    out = []
    for _ in range(n):
        while True:
            m = rng.randrange(10 ** p)
            if m or not nonzero:
                break
        out.append((rng.randint(0, 1), m))
    return out


@pytest.mark.parametrize("p", [15, 38, 150])
@pytest.mark.parametrize("op", ["mad", "div"])
def test_block_list_projection(p, op):
    rng = random.Random(p * 7 + len(op))
    s = p // 4
    rows = 5000
    e, ct = workloads.sweep_expr(p, op)
    m = runtime.compile_expr(e, ct)
    raws = [codec.encode(_vals(rng, p, rows, nonzero=(op == "div" and k == 1)), p) for k in range(len(ct))]
    vb = codec.compact_bytes(p)
    cols = [runtime.DeviceColumn.from_blocks(_split_blocks(r, vb, rng, rng.randint(2, 9)), p, s) for r in raws]
    out = m.launch(cols, rows)
    torch.cuda.synchronize()
    exp, _ = oracle.eval_expr(m.built, m.root, raws, rows, m.value_bytes)
    assert bytes(out.cpu().numpy().tobytes()) == exp


def test_block_list_grouped_query():
    rng = random.Random(11)
    rows, G = 7000, 6
    exprs, aggs, ct = workloads.query_exprs()
    q = runtime.compile_query(exprs, aggs, ct)
    R = workloads.QUERY_RANGES
    raws = [codec.encode([(0, rng.randrange(R[n][0], R[n][1] + 1, R[n][2])) for _ in range(rows)], 15)
            for n in ("qty", "price", "disc", "tax")]
    gid = np.array([rng.randrange(G) for _ in range(rows)], dtype=np.int32)
    cols = [runtime.DeviceColumn.from_blocks(_split_blocks(r, 7, rng, 5), 15, 2) for r in raws]
    outs = q.launch(cols, torch.from_numpy(gid).cuda(), G)
    torch.cuda.synchronize()
    exp = oracle.query(q.built, q.aggs, raws, gid.tobytes(), rows, G)
    for o, e in zip(outs, exp):
        assert bytes(o.cpu().numpy().tobytes()) == e


@pytest.mark.parametrize("p", [18, 76])
def test_nullable_projection(p):
    rng = random.Random(p)
    s = p // 4
    rows = 3000
    ct = [E.ColType(p, s, nullable=True), E.ColType(p, s), E.ColType(p, s, nullable=True)]
    a, b, c = E.col(0), E.col(1), E.col(2)
    for expr in (a * b + c, a / b, (a + c).ge(b)):
        m = runtime.compile_expr(expr, ct)
        ra, _ = _nullable_raw(_vals(rng, p, rows), p, rng, 0.15)
        rb = codec.encode(_vals(rng, p, rows, nonzero=True), p)
        rc, _ = _nullable_raw(_vals(rng, p, rows), p, rng, 0.15)
        cols = [runtime.DeviceColumn.from_host(ra, p, s, nullable=True), runtime.DeviceColumn.from_host(rb, p, s),
                runtime.DeviceColumn.from_host(rc, p, s, nullable=True)]
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        out = m.launch(cols, rows, err=err)
        torch.cuda.synchronize()
        exp, eerr = oracle.eval_expr(m.built, m.root, [ra, rb, rc], rows, m.value_bytes)
        assert bytes(out.cpu().numpy().tobytes()) == exp
        assert int(err.item()) == eerr


def test_nullable_grouped_query_semantics():
    rng = random.Random(5)
    rows, G = 4000, 5
    ct = [E.ColType(15, 2, nullable=True), E.ColType(15, 2), E.ColType(15, 2, nullable=True)]
    x, y, z = E.col(0), E.col(1), E.col(2)
    exprs = [x, y, x * y, z / y]
    aggs = [(abi.UP_AGG_SUM, 0), (abi.UP_AGG_SUM, 1), (abi.UP_AGG_AVG, 2), (abi.UP_AGG_AVG, 3),
            (abi.UP_AGG_SUM, 2), (abi.UP_AGG_COUNT, 0)]
    q = runtime.compile_query(exprs, aggs, ct)
    gid = np.array([rng.randrange(G) for _ in range(rows)], dtype=np.int32)
    g4 = {i for i in range(rows) if gid[i] == 4}  # group 4: every x and z NULL
    rx, fx = _nullable_raw(_vals(rng, 15, rows), 15, rng, 0.2, g4)
    ry = codec.encode(_vals(rng, 15, rows, nonzero=True), 15)
    rz, fz = _nullable_raw(_vals(rng, 15, rows), 15, rng, 0.2, g4)
    cols = [runtime.DeviceColumn.from_host(rx, 15, 2, nullable=True), runtime.DeviceColumn.from_host(ry, 15, 2),
            runtime.DeviceColumn.from_host(rz, 15, 2, nullable=True)]
    outs = q.launch(cols, torch.from_numpy(gid).cuda(), G)
    torch.cuda.synchronize()
    got = [bytes(o.cpu().numpy().tobytes()) for o in outs]
    exp = oracle.query(q.built, q.aggs, [rx, ry, rz], gid.tobytes(), rows, G)
    assert got == exp
    img = abi.UP_AGG_DECIMAL_BYTES
    assert got[0][4 * img] == 0 and got[2][4 * img] == 0   # SUM(x), AVG(x*y) of an all-NULL group
    assert got[1][4 * img] == 1                             # SUM(y) there is a value
    counts = np.frombuffer(got[5], dtype=np.int64)
    assert counts.tolist() == np.bincount(gid, minlength=G).tolist()  # COUNT(*) counts NULL rows too


def test_minus_one_index_on_non_nullable_query_column_is_a_domain_error():
    rng = random.Random(9)
    rows, G = 1000, 3
    exprs, aggs, ct = workloads.query_exprs()
    q = runtime.compile_query(exprs, aggs, ct)
    raws = [codec.encode([(0, rng.randrange(1, 10 ** 6)) for _ in range(rows)], 15) for _ in range(4)]
    idx = torch.arange(rows, dtype=torch.int32, device="cuda")
    idx[17] = -1
    cols = [runtime.DeviceColumn(torch.frombuffer(bytearray(r), dtype=torch.uint8).cuda(), 15, 2, indices=idx)
            for r in raws]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    gid = torch.zeros(rows, dtype=torch.int32, device="cuda")
    outs = q.launch(cols, gid, G, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) & abi.UP_ROWERR_DOMAIN
    counts = np.frombuffer(bytes(outs[-1].cpu().numpy().tobytes()), dtype=np.int64)
    assert counts[0] == rows - 1
