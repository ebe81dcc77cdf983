"""GPU parity of GROUP BY keys read by the query kernel: the key table
(up_group_table_from_keys) against numpy's sorted unique keys and the per-row
ids of up_group_ids_from_keys, and the fused key query
(up_query_launch_keys) against the oracle, byte for byte, in every key layout
and accumulation mode."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from ultraprecise_b200 import abi, codec, runtime
from ultraprecise_b200 import expr as E
from tests.test_gpu_agg import grouped_query_columns, grouped_query

pytestmark = pytest.mark.gpu


def _keys_host(keys, key_bytes, rows):
    """Each row's key as an int (key bytes in column order, most significant
    first) and the dense ids in ascending key order."""
    key = np.zeros(rows, dtype=np.int64)
    for k, b in zip(keys, key_bytes):
        h = k.cpu().numpy()[: rows * b].reshape(rows, b).astype(np.int64)
        for j in range(b):
            key = (key << 8) | h[:, j]
    uniq = np.unique(key)
    return key, uniq, np.searchsorted(uniq, key).astype(np.int32)


def _make_keys(layout, groups, n, seed):
    """`n` rows of keys in one of the three layouts with about `groups`
    distinct keys spread over the key space."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    if layout == "1x1":
        space = torch.randperm(256, generator=g, device="cuda")[:groups].to(torch.int64)
    else:
        space = torch.randperm(65536, generator=g, device="cuda")[:groups].to(torch.int64)
    pick = space[torch.randint(0, groups, (n,), generator=g, device="cuda")]
    if layout == "1x1":
        return [pick.to(torch.uint8).contiguous()], [1]
    hi, lo = (pick >> 8).to(torch.uint8), (pick & 255).to(torch.uint8)
    if layout == "2x1":
        return [hi.contiguous(), lo.contiguous()], [1, 1]
    return [torch.stack([hi, lo], dim=1).reshape(-1).contiguous()], [2]


@pytest.mark.parametrize("layout,groups,rows,offset", [
    ("2x1", 4, 1, 0), ("2x1", 4, 1_000_003, 0), ("2x1", 4, 100_000, 1), ("1x1", 256, 70_001, 0),
    ("1x1", 7, 4096, 3), ("1x2", 3000, 500_000, 0), ("1x2", 50, 33_333, 1), ("2x1", 20_000, 2_000_000, 0)])
def test_key_table_matches_numpy(layout, groups, rows, offset):
    keys_all, kb = _make_keys(layout, groups, rows + offset, seed=groups + rows)
    keys = [k[offset * b:] for k, b in zip(keys_all, kb)]
    table, G, gkeys = runtime.group_table_from_keys(keys, kb)
    key, uniq, ids = _keys_host(keys, kb, rows)
    assert G == len(uniq)
    t = table.cpu().numpy()
    assert np.array_equal(t[key], ids)
    absent = np.ones(65536, dtype=bool)
    absent[uniq] = False
    assert (t[:65536][absent] == -1).all()
    assert np.array_equal(t[65536:65536 + G], uniq)
    total = sum(kb)
    got_keys = gkeys.cpu().numpy().reshape(-1, total).astype(np.int64)
    k_int = np.zeros(len(got_keys), dtype=np.int64)
    for j in range(total):
        k_int = (k_int << 8) | got_keys[:, j]
    assert np.array_equal(k_int, uniq)
    gid, G2, _ = runtime.group_ids_from_keys(keys, kb)
    assert G2 == G and np.array_equal(gid.cpu().numpy(), ids)


@pytest.mark.parametrize("rows", [1, 1000, 100_003, 1_000_000])
def test_grouped_query_from_keys_matches_oracle(rows):
    qty, price, disc, tax, k1, k2 = grouped_query_columns(rows, 20261203)
    exprs, aggs, cols = grouped_query()
    q = runtime.compile_query(exprs, aggs, cols)
    table, G, _ = runtime.group_table_from_keys([k1, k2], [1, 1])
    dev = [runtime.DeviceColumn(t, 15, 2) for t in (qty, price, disc, tax)]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    outs = q.launch_keys(dev, [k1, k2], [1, 1], table, G, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    _, uniq, ids = _keys_host([k1, k2], [1, 1], rows)
    assert G == len(uniq)
    raws = [bytes(t.cpu().numpy().tobytes()) for t in (qty, price, disc, tax)]
    exp = oracle.query(q.built, q.aggs, raws, ids.tobytes(), rows, G, threads=8)
    for k, (o, e) in enumerate(zip(outs, exp)):
        assert bytes(o.cpu().numpy().tobytes()) == e, f"aggregate {k}"


@pytest.mark.parametrize("layout,groups,rows,offset", [
    ("2x1", 4, 1_000_000, 0), ("1x1", 5, 70_001, 1), ("1x1", 9, 20_000, 0), ("1x1", 200, 200_000, 0),
    ("1x2", 150, 3000, 1), ("2x1", 1000, 50_000, 0), ("1x2", 5000, 300_000, 0), ("2x1", 5000, 7_777, 1)])
def test_query_from_keys_every_mode(layout, groups, rows, offset):
    """Register, shared-memory and global accumulation with each key layout;
    an offset of one row misaligns the columns and keys, which moves every
    tile through the synchronous copy path."""
    cols = [E.ColType(15, 2), E.ColType(30, 5), E.ColType(15, 2)]
    a, b, c = E.col(0), E.col(1), E.col(2)
    exprs = [a, a * b, b - c, a * c + b]
    aggs = [(abi.UP_AGG_SUM, 0), (abi.UP_AGG_SUM, 1), (abi.UP_AGG_AVG, 2), (abi.UP_AGG_COUNT, 0),
            (abi.UP_AGG_AVG, 0), (abi.UP_AGG_SUM, 3)]
    q = runtime.compile_query(exprs, aggs, cols)
    n = rows + offset
    raw = [runtime.gen_digits(n, ct.precision, 17 * groups + i, signed=True) for i, ct in enumerate(cols)]
    dev = [runtime.DeviceColumn(t[offset * codec.compact_bytes(ct.precision):], ct.precision, ct.scale)
           for t, ct in zip(raw, cols)]
    keys_all, kb = _make_keys(layout, groups, n, seed=groups * 3 + rows)
    keys = [k[offset * w:] for k, w in zip(keys_all, kb)]
    table, G, _ = runtime.group_table_from_keys(keys, kb)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    outs = q.launch_keys(dev, keys, kb, table, G, err=err, rows=rows)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    _, uniq, ids = _keys_host(keys, kb, rows)
    hraw = [bytes(d.data.cpu().numpy().tobytes()) for d in dev]
    exp = oracle.query(q.built, q.aggs, hraw, ids.tobytes(), rows, G, threads=8)
    for k, (o, e) in enumerate(zip(outs, exp)):
        assert bytes(o.cpu().numpy().tobytes()) == e, f"aggregate {k}"


def test_key_launch_rejects_bad_layouts():
    lib = abi.load()
    exprs, aggs, cols = grouped_query()
    q = runtime.compile_query(exprs, aggs, cols)
    k = torch.zeros(16, dtype=torch.uint8, device="cuda")
    table = torch.zeros(abi.UP_KEY_TABLE_ENTRIES, dtype=torch.int32, device="cuda")
    import ctypes as C
    kp = (C.c_void_p * 3)(k.data_ptr(), k.data_ptr(), k.data_ptr())
    for kb in ([3], [2, 1], [1, 1, 1]):
        arr = (C.c_int32 * len(kb))(*kb)
        assert lib.up_query_launch_keys(q._h, None, 0, 0, kp, arr, len(kb), table.data_ptr(), 1, None, None,
                                        None) == abi.UP_ERR_UNSUPPORTED
    n = C.c_int32()
    arr = (C.c_int32 * 2)(2, 1)
    assert lib.up_group_table_from_keys(kp, arr, 2, 16, table.data_ptr(), C.byref(n), None,
                                        None) == abi.UP_ERR_UNSUPPORTED


@pytest.mark.parametrize("groups", [2, 40])
def test_key_outside_the_table_is_a_domain_error(groups):
    """A table built from other rows than the launch's: rows whose key it
    lacks are flagged (register mode by the match count, the other modes by
    the table's -1)."""
    exprs, aggs, cols = grouped_query()
    q = runtime.compile_query(exprs, aggs, cols)
    rows = 50_000
    qty, price, disc, tax, _, _ = grouped_query_columns(rows, 5)
    k = (torch.arange(rows, device="cuda") % groups).to(torch.uint8)
    k[rows // 2:] = torch.where(k[rows // 2:] == 0, torch.full_like(k[rows // 2:], 200), k[rows // 2:])
    table, G, _ = runtime.group_table_from_keys([k[: rows // 2].contiguous()], [1])
    assert G == groups
    dev = [runtime.DeviceColumn(t, 15, 2) for t in (qty, price, disc, tax)]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    q.launch_keys(dev, [k], [1], table, G, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) & abi.UP_ROWERR_DOMAIN


def _mode_query():
    cols = [E.ColType(15, 2), E.ColType(30, 5), E.ColType(15, 2)]
    a, b, c = E.col(0), E.col(1), E.col(2)
    exprs = [a, a * b, b - c, a * c + b]
    aggs = [(abi.UP_AGG_SUM, 0), (abi.UP_AGG_SUM, 1), (abi.UP_AGG_AVG, 2), (abi.UP_AGG_COUNT, 0),
            (abi.UP_AGG_AVG, 0), (abi.UP_AGG_SUM, 3)]
    return runtime.compile_query(exprs, aggs, cols), cols


@pytest.mark.parametrize("layout,groups,rows,offset,cap", [
    ("2x1", 4, 1_000_000, 0, 4), ("2x1", 4, 100_000, 0, 64), ("1x1", 9, 20_000, 1, 256),
    ("1x1", 200, 200_000, 0, 256), ("1x2", 5000, 300_000, 0, 8192), ("2x1", 3000, 7_777, 1, 65536)])
def test_async_pair_matches_sync(layout, groups, rows, offset, cap):
    """Key table and query without a host round trip (the group count stays on
    the device and picks the accumulation mode there) give the same bytes as
    the synchronous pair, whatever the output capacity."""
    q, cols = _mode_query()
    n = rows + offset
    raw = [runtime.gen_digits(n, ct.precision, 5 * groups + i, signed=True) for i, ct in enumerate(cols)]
    dev = [runtime.DeviceColumn(t[offset * codec.compact_bytes(ct.precision):], ct.precision, ct.scale)
           for t, ct in zip(raw, cols)]
    keys_all, kb = _make_keys(layout, groups, n, seed=groups + 11 * rows)
    keys = [k[offset * w:] for k, w in zip(keys_all, kb)]
    table, G, _ = runtime.group_table_from_keys(keys, kb)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    exp = q.launch_keys(dev, keys, kb, table, G, err=err, rows=rows)
    table2 = torch.full((abi.UP_KEY_TABLE_ENTRIES,), -7, dtype=torch.int32, device="cuda")
    runtime.group_table_from_keys_async(keys, kb, table2)
    err2 = torch.zeros(1, dtype=torch.int32, device="cuda")
    got = q.launch_keys_async(dev, keys, kb, table2, cap, err=err2, rows=rows)
    torch.cuda.synchronize()
    assert int(err.item()) == 0 and int(err2.item()) == 0
    assert int(table2[abi.UP_KEY_TABLE_COUNT].item()) == G
    assert torch.equal(table2[:65536 + G], table[:65536 + G])
    for k, (o, e) in enumerate(zip(got, exp)):
        assert torch.equal(o[: e.numel()], e), f"aggregate {k}"


def test_async_count_above_capacity_is_a_domain_error():
    q, cols = _mode_query()
    rows = 10_000
    raw = [runtime.gen_digits(rows, ct.precision, 3 + i) for i, ct in enumerate(cols)]
    dev = [runtime.DeviceColumn(t, ct.precision, ct.scale) for t, ct in zip(raw, cols)]
    keys, kb = _make_keys("1x1", 20, rows, seed=4)
    table = torch.empty(abi.UP_KEY_TABLE_ENTRIES, dtype=torch.int32, device="cuda")
    runtime.group_table_from_keys_async(keys, kb, table)
    outs = [torch.full((8 * (8 if k == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES),), 0xAB, dtype=torch.uint8,
                       device="cuda") for k, _ in q.aggs]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    q.launch_keys_async(dev, keys, kb, table, 8, outs=outs, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) & abi.UP_ROWERR_DOMAIN
    assert all(bool((o == 0xAB).all()) for o in outs)


def test_async_pair_replays_in_a_cuda_graph():
    """The whole grouped query (key table + fused query) captured once and
    replayed over new key and value data gives the synchronous pair's bytes."""
    exprs, aggs, cols = grouped_query()
    q = runtime.compile_query(exprs, aggs, cols)
    rows, cap = 200_000, 16
    qty, price, disc, tax, k1, k2 = grouped_query_columns(rows, 1)
    dev = [runtime.DeviceColumn(t, 15, 2) for t in (qty, price, disc, tax)]
    table = torch.empty(abi.UP_KEY_TABLE_ENTRIES, dtype=torch.int32, device="cuda")
    outs = [torch.empty(cap * (8 if k == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES), dtype=torch.uint8,
                        device="cuda") for k, _ in q.aggs]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):  # load the modules outside the capture
        runtime.group_table_from_keys_async([k1, k2], [1, 1], table, stream=side)
        q.launch_keys_async(dev, [k1, k2], [1, 1], table, cap, outs=outs, err=err, stream=side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        s = torch.cuda.current_stream()
        runtime.group_table_from_keys_async([k1, k2], [1, 1], table, stream=s)
        q.launch_keys_async(dev, [k1, k2], [1, 1], table, cap, outs=outs, err=err, stream=s)
    for seed in (2, 3):
        new = grouped_query_columns(rows, seed)
        for dst, src in zip((qty, price, disc, tax, k1, k2), new):
            dst.copy_(src)
        err.zero_()
        graph.replay()
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        t2, G, _ = runtime.group_table_from_keys([k1, k2], [1, 1])
        exp = q.launch_keys(dev, [k1, k2], [1, 1], t2, G)
        torch.cuda.synchronize()
        for k, (o, e) in enumerate(zip(outs, exp)):
            assert torch.equal(o[: e.numel()], e), f"seed {seed} aggregate {k}"
    del graph
