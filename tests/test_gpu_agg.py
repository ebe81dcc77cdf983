"""GPU parity of grouped SUM/COUNT/AVG (fused and plain) against the oracle."""
import ctypes as C
import random

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from ultraprecise_b200 import abi, codec, runtime
from ultraprecise_b200 import expr as E

pytestmark = pytest.mark.gpu

KEYS = [(b"A", b"F", 0.25), (b"N", b"F", 0.007), (b"N", b"O", 0.493), (b"R", b"F", 0.25)]


def grouped_query_columns(rows: int, seed: int):
    """The grouped-query columns: qty 1-50, price 900.00-104949.50, disc 0.00-0.10,
    tax 0.00-0.08, all DECIMAL(15,2); two CHAR(1) keys with the Q1 weights."""
    qty = runtime.gen_range(rows, 15, 100, 5000, 100, seed + 1)
    price = runtime.gen_range(rows, 15, 90000, 10494950, 1, seed + 2)
    disc = runtime.gen_range(rows, 15, 0, 10, 1, seed + 3)
    tax = runtime.gen_range(rows, 15, 0, 8, 1, seed + 4)
    g = torch.Generator(device="cuda").manual_seed(seed)
    w = torch.tensor([k[2] for k in KEYS], device="cuda")
    pick = torch.multinomial(w, rows, replacement=True, generator=g)
    k1 = torch.tensor([k[0][0] for k in KEYS], dtype=torch.uint8, device="cuda")[pick]
    k2 = torch.tensor([k[1][0] for k in KEYS], dtype=torch.uint8, device="cuda")[pick]
    return qty, price, disc, tax, k1.contiguous(), k2.contiguous()


def grouped_query():
    cols = [E.ColType(15, 2)] * 4
    qty, price, disc, tax = [E.col(i) for i in range(4)]
    disc_price = price * (E.dec("1.00") - disc)
    charge = disc_price * (E.dec("1.00") + tax)
    exprs = [qty, price, disc_price, charge, disc]
    aggs = [(abi.UP_AGG_SUM, 0), (abi.UP_AGG_SUM, 1), (abi.UP_AGG_SUM, 2), (abi.UP_AGG_SUM, 3),
            (abi.UP_AGG_AVG, 0), (abi.UP_AGG_AVG, 1), (abi.UP_AGG_AVG, 4), (abi.UP_AGG_COUNT, 0)]
    return exprs, aggs, cols


@pytest.mark.parametrize("rows", [1, 1000, 100_003, 1_000_000])
def test_grouped_query_fused_parity(rows):
    qty, price, disc, tax, k1, k2 = grouped_query_columns(rows, 20261203)
    gid, G, gkeys = runtime.group_ids_from_keys([k1, k2], [1, 1])
    exprs, aggs, cols = grouped_query()
    q = runtime.compile_query(exprs, aggs, cols)
    dev = [runtime.DeviceColumn(t, 15, 2) for t in (qty, price, disc, tax)]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    outs = q.launch(dev, gid, G, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    raws = [bytes(t.cpu().numpy().tobytes()) for t in (qty, price, disc, tax)]
    graw = bytes(gid.cpu().numpy().tobytes())
    exp = oracle.query(q.built, q.aggs, raws, graw, rows, G, threads=8)
    for k, (o, e) in enumerate(zip(outs, exp)):
        assert bytes(o.cpu().numpy().tobytes()) == e, f"aggregate {k}"
    # groups come out in key order, as the reference's sort-based grouping
    keys = gkeys.cpu().numpy().reshape(-1, 2)
    assert [bytes(r) for r in keys] == sorted(bytes(r) for r in keys)
    assert G == (4 if rows >= 1000 else G)


@pytest.mark.parametrize("p", [15, 38, 150])
def test_group_agg_plain_parity(p):
    rows, G = 50_000, 97
    vals = runtime.gen_digits(rows, p, 77 + p)
    gid = torch.randint(0, G, (rows,), dtype=torch.int32, device="cuda",
                        generator=torch.Generator(device="cuda").manual_seed(p))
    s = p // 3
    col = runtime.DeviceColumn(vals, p, s)
    outs = runtime.group_agg([col, col, col], [abi.UP_AGG_SUM, abi.UP_AGG_AVG, abi.UP_AGG_COUNT], gid, G + 2)
    torch.cuda.synchronize()
    raw = bytes(vals.cpu().numpy().tobytes())
    graw = bytes(gid.cpu().numpy().tobytes())
    for o, kind in zip(outs, [abi.UP_AGG_SUM, abi.UP_AGG_AVG, abi.UP_AGG_COUNT]):
        exp = oracle.group_agg(raw, codec.compact_bytes(p), s, kind, graw, rows, G + 2)
        assert bytes(o.cpu().numpy().tobytes()) == exp, kind


def test_aggregate_column_data_segments():
    """AggregateColumnData form: rows visited through `associated`, grouped
    by ascending segment starts."""
    lib = abi.load()
    rng = random.Random(4)
    rows, G = 10_000, 13
    vals = [(rng.randint(0, 1), rng.randint(0, 10 ** 20)) for _ in range(rows)]
    raw = codec.encode(vals, 25)
    assoc = list(range(rows))
    rng.shuffle(assoc)
    starts = sorted(rng.sample(range(1, rows), G - 1))
    starts = [0] + starts
    d = runtime.DeviceColumn.from_host(raw, 25, 5)
    ta = torch.tensor(assoc, dtype=torch.int32, device="cuda")
    ts = torch.tensor(starts, dtype=torch.int32, device="cuda")
    out = torch.empty(G * 133, dtype=torch.uint8, device="cuda")
    c = d.up_column()
    abi.check(lib.up_aggregate_column_data(C.byref(c), abi.UP_AGG_SUM, ta.data_ptr(),
                                           ts.data_ptr(), G, rows, out.data_ptr(), None,
                                           torch.cuda.current_stream().cuda_stream), "agg")
    torch.cuda.synchronize()
    B = codec.compact_bytes(25)
    gath = b"".join(raw[i * B:(i + 1) * B] for i in assoc)
    gids = np.zeros(rows, dtype=np.int32)
    for g in range(G):
        gids[starts[g]:(starts[g + 1] if g + 1 < G else rows)] = g
    exp = oracle.group_agg(gath, B, 5, abi.UP_AGG_SUM, gids.tobytes(), rows, G)
    assert bytes(out.cpu().numpy().tobytes()) == exp


def test_division_int64_matches_oracle():
    lib = abi.load()
    rng = random.Random(8)
    n = 300
    imgs = bytearray()
    counts = []
    for i in range(n):
        mag = rng.randint(0, 1 << rng.choice([10, 40, 51, 60, 64, 100, 300]))
        img = bytearray(133)
        img[0] = 1
        img[1] = rng.randint(0, 1)
        img[3] = rng.randint(0, 20)
        img[5:133] = mag.to_bytes(128, "little")
        imgs += img
        counts.append(rng.choice([0, 1, 3, 7, 1 << 20, (1 << 33) + 5, rng.randint(1, 1 << 40)]))
    ts = torch.frombuffer(bytearray(imgs), dtype=torch.uint8).cuda()
    tc = torch.tensor(counts, dtype=torch.int64, device="cuda")
    out = torch.empty(n * 133, dtype=torch.uint8, device="cuda")
    abi.check(lib.up_division_int64(ts.data_ptr(), tc.data_ptr(), n, out.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream), "div")
    torch.cuda.synchronize()
    got = bytes(out.cpu().numpy().tobytes())
    for i in range(n):
        exp = oracle.division_int64(bytes(imgs[i * 133:(i + 1) * 133]), counts[i])
        assert got[i * 133:(i + 1) * 133] == exp, i


@pytest.mark.parametrize("groups,rows,offset", [
    (1, 70_001, 0), (3, 5_000, 0), (4, 1_000_000, 0), (4, 100_003, 1), (5, 33_333, 0),
    (8, 20_000, 0), (9, 20_000, 0), (100, 200_000, 0), (150, 3000, 1), (1000, 50_000, 0),
    (5000, 300_000, 0), (5000, 7_777, 1)])
def test_query_accumulation_modes(groups, rows, offset):
    """Every accumulation strategy of the fused query (per-thread registers,
    per-CTA shared memory, global) over signed values of three widths; an
    offset of one row misaligns the columns and group ids, which moves every
    tile through the synchronous copy path."""
    cols = [E.ColType(15, 2), E.ColType(30, 5), E.ColType(15, 2)]
    a, b, c = E.col(0), E.col(1), E.col(2)
    exprs = [a, a * b, b - c, a * c + b]
    aggs = [(abi.UP_AGG_SUM, 0), (abi.UP_AGG_SUM, 1), (abi.UP_AGG_AVG, 2), (abi.UP_AGG_COUNT, 0),
            (abi.UP_AGG_AVG, 0), (abi.UP_AGG_SUM, 3)]
    q = runtime.compile_query(exprs, aggs, cols)
    n = rows + offset
    raw = [runtime.gen_digits(n, ct.precision, 31 * groups + i, signed=True) for i, ct in enumerate(cols)]
    g = torch.Generator(device="cuda").manual_seed(groups)
    gid_all = torch.randint(0, groups, (n,), dtype=torch.int32, device="cuda", generator=g)
    dev = [runtime.DeviceColumn(t[offset * codec.compact_bytes(ct.precision):], ct.precision, ct.scale)
           for t, ct in zip(raw, cols)]
    gid = gid_all[offset:]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    outs = q.launch(dev, gid, groups, err=err, rows=rows)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    hraw = [bytes(d.data.cpu().numpy().tobytes()) for d in dev]
    exp = oracle.query(q.built, q.aggs, hraw, bytes(gid.cpu().numpy().tobytes()), rows, groups, threads=8)
    for k, (o, e) in enumerate(zip(outs, exp)):
        assert bytes(o.cpu().numpy().tobytes()) == e, f"aggregate {k}"
