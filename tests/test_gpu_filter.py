"""GPU parity of predicates (comparisons joined by AND / OR) against the
oracle, and of row selection (up_filter_flags) against numpy's nonzero: the
selected row indices in row order and their count."""
import random

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from tests.helpers import edge_values
from ultraprecise_b200 import abi, codec, runtime
from ultraprecise_b200 import expr as E

pytestmark = pytest.mark.gpu


def _oracle(e, types, raws, rows):
    b = E.build([e], types)
    E.derive_types(b)
    return oracle.eval_expr(b, b.roots[0], raws, rows, 1, threads=8)


def _device(e, types, raws, rows, tpv=0):
    m = runtime.compile_expr(e, types, threads_per_value=tpv) if tpv else runtime.compile_expr(e, types)
    dev = [runtime.DeviceColumn.from_host(r, t.precision, t.scale) for r, t in zip(raws, types)]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = m.launch(dev, rows, err=err)
    torch.cuda.synchronize()
    return out, int(err.item())


@pytest.mark.parametrize("p", [15, 38, 150])
def test_and_or_predicates_match_oracle(p):
    s = p // 4
    types = [E.ColType(p, s), E.ColType(p, s // 2), E.ColType(p, s)]
    a, b, c = E.col(0), E.col(1), E.col(2)
    rows = 4001
    rng = random.Random(p)
    vals = [edge_values(p, rng, rows) for _ in types]
    raws = [codec.encode(v, t.precision) for v, t in zip(vals, types)]
    for e in (a.lt(b).and_(c.ge(a)), a.eq(c).or_(b.ne(0)), a.gt(b).and_(b.gt(c).or_((a * b).le(c))),
              (a / b).lt(c).or_(a.eq(b))):
        exp, exp_err = _oracle(e, types, raws, rows)
        out, err = _device(e, types, raws, rows)
        assert bytes(out.cpu().numpy().tobytes()) == exp
        assert err == exp_err


def test_and_or_cooperative_matches_oracle():
    p, s = 300, 60
    types = [E.ColType(p, s), E.ColType(p, s)]
    a, b = E.col(0), E.col(1)
    rows = 2000
    rng = random.Random(5)
    raws = [codec.encode(edge_values(p, rng, rows), p) for _ in types]
    e = (a * b).ge(a + b).and_(a.ne(b)).or_(a.eq(0))
    exp, exp_err = _oracle(e, types, raws, rows)
    for tpv in (1, 8, 16):
        out, err = _device(e, types, raws, rows, tpv)
        assert bytes(out.cpu().numpy().tobytes()) == exp, f"threads_per_value={tpv}"
        assert err == exp_err


@pytest.mark.parametrize("rows,density,offset", [(1, 1.0, 0), (4095, 0.5, 0), (4096, 0.0, 0), (4097, 1.0, 0),
                                                 (100_003, 0.3, 0), (100_003, 0.3, 5), (5_000_000, 0.01, 0),
                                                 (5_000_000, 0.999, 0), (70_000, 0.5, 3)])
def test_filter_flags_matches_nonzero(rows, density, offset):
    """Flag bytes of any nonzero value; an offset misaligns the flags, which
    takes the byte-wise path."""
    g = torch.Generator(device="cuda").manual_seed(rows + offset)
    flags = (torch.rand(rows + offset, device="cuda", generator=g) < density).to(torch.uint8)
    flags[flags == 1] = torch.randint(1, 256, (int(flags.sum()),), device="cuda", dtype=torch.int32).to(torch.uint8)
    flags = flags[offset:]
    idx = runtime.filter_flags(flags, rows)
    exp = np.nonzero(flags.cpu().numpy())[0].astype(np.int32)
    assert np.array_equal(idx.cpu().numpy(), exp)


def test_filter_flags_empty_and_errors():
    cnt = torch.full((1,), 7, dtype=torch.int64, device="cuda")
    lib = abi.load()
    assert lib.up_filter_flags(None, 0, None, cnt.data_ptr(), None) == abi.UP_OK
    torch.cuda.synchronize()
    assert int(cnt.item()) == 0
    assert lib.up_filter_flags(None, -1, None, cnt.data_ptr(), None) == abi.UP_ERR_INVALID_ARG
    assert lib.up_filter_flags(None, 10, None, cnt.data_ptr(), None) == abi.UP_ERR_INVALID_ARG


def test_predicate_then_filter_selects_rows():
    """WHERE a*b >= c AND a <> 0: the predicate module's flags select the same
    rows as the oracle's."""
    p, s = 38, 6
    types = [E.ColType(p, s)] * 3
    a, b, c = E.col(0), E.col(1), E.col(2)
    rows = 300_000
    cols = [runtime.gen_digits(rows, p, 10 + i) for i in range(3)]
    e = (a * b).ge(c).and_(a.ne(0))
    m = runtime.compile_expr(e, types)
    dev = [runtime.DeviceColumn(t, p, s) for t in cols]
    flags = m.launch(dev, rows)
    idx = runtime.filter_flags(flags, rows)
    raws = [bytes(t.cpu().numpy().tobytes()) for t in cols]
    exp, _ = _oracle(e, types, raws, rows)
    exp_idx = np.nonzero(np.frombuffer(exp, dtype=np.uint8))[0].astype(np.int32)
    assert 0 < len(exp_idx) < rows
    assert np.array_equal(idx.cpu().numpy(), exp_idx)


def test_selected_rows_feed_the_next_expression():
    """The selected indices become the row indirection of the next launch
    (the reference's associated-column filter): a*b over the kept rows equals
    the oracle's a*b over the gathered values."""
    p, s = 38, 6
    types = [E.ColType(p, s)] * 2
    a, b = E.col(0), E.col(1)
    rows = 200_000
    B = codec.compact_bytes(p)
    cols = [runtime.gen_digits(rows, p, 20 + i) for i in range(2)]
    flags = runtime.compile_expr(a.lt(b), types).launch([runtime.DeviceColumn(t, p, s) for t in cols], rows)
    idx = runtime.filter_flags(flags, rows)
    kept = idx.numel()
    assert 0 < kept < rows
    dev = [runtime.DeviceColumn(t, p, s, indices=idx) for t in cols]
    out = runtime.compile_expr(a * b, types).launch(dev, kept)
    sel = idx.cpu().numpy().astype(np.int64)
    raws = []
    for t in cols:
        h = t.cpu().numpy().reshape(rows, B)
        raws.append(bytes(h[sel].tobytes()))
    bb = E.build([a * b], types)
    E.derive_types(bb)
    exp, _ = oracle.eval_expr(bb, bb.roots[0], raws, kept, codec.compact_bytes(bb.nodes[bb.roots[0]].precision),
                              threads=8)
    assert bytes(out.cpu().numpy().tobytes()) == exp
