"""CPU: the C oracle against the independent Python-int restatement and
against known answers taken from the reference's own tests and semantics."""
import random

import pytest

from oracle import oracle, pyref
from ultraprecise_b200 import abi, codec
from ultraprecise_b200 import expr as E
from tests.helpers import edge_values


def run_both(root_expr, cols_t, cols_vals, rows):
    b = E.build([root_expr], cols_t)
    E.derive_types(b)
    r = b.roots[0]
    nd = b.nodes[r]
    is_cmp = nd.kind in abi.COMPARE_KINDS
    ob = 1 if is_cmp else codec.compact_bytes(nd.precision)
    raw = [codec.encode(v, t.precision) for v, t in zip(cols_vals, cols_t)]
    got, err, rerr = oracle.eval_expr(b, r, raw, rows, ob, row_errors=True)
    for i in range(rows):
        row = [raw[c][i * codec.compact_bytes(t.precision):(i + 1) * codec.compact_bytes(t.precision)]
               for c, t in enumerate(cols_t)]
        v, z = pyref.eval_nodes(b.nodes, r, cols_t, row)
        if is_cmp:
            exp = bytes([v])
            ovf = False
        else:
            exp, ovf = pyref.encode(v, ob)
        assert got[i * ob:(i + 1) * ob] == exp, (i, row, v)
        assert bool(rerr[i] & abi.UP_ROWERR_DIV_BY_ZERO) == z
        assert bool(rerr[i] & abi.UP_ROWERR_OVERFLOW) == ovf
    return got, err


@pytest.mark.parametrize("p,s", [(15, 2), (18, 4), (38, 9), (20, 0), (9, 9), (76, 19)])
@pytest.mark.parametrize("op", ["add", "sub", "mul", "div", "mod", "cmp"])
def test_oracle_matches_pyref_binary(p, s, op):
    rng = random.Random(hash((p, s, op)) & 0xFFFF)
    n = 120
    s2 = max(0, min(p, s + rng.choice([-2, 0, 3])))
    cols = [E.ColType(p, s), E.ColType(p, s2)]
    a, b = E.col(0), E.col(1)
    expr = {"add": a + b, "sub": a - b, "mul": a * b, "div": a / b, "mod": a % b, "cmp": a.lt(b)}[op]
    va = edge_values(p, rng, n)
    vb = edge_values(p, rng, n)
    run_both(expr, cols, [va, vb], n)


@pytest.mark.parametrize("cmp", ["lt", "le", "gt", "ge", "eq", "ne"])
def test_oracle_compare_ops(cmp):
    rng = random.Random(7)
    cols = [E.ColType(12, 3), E.ColType(10, 1)]
    a, b = E.col(0), E.col(1)
    expr = getattr(a, cmp)(b)
    va = edge_values(12, rng, 80) + [(1, 0), (0, 0)]
    vb = edge_values(10, rng, 80) + [(0, 0), (1, 0)]
    run_both(expr, cols, [va, vb], 82)


def test_oracle_nested_and_constants():
    rng = random.Random(11)
    cols = [E.ColType(15, 2)] * 3
    a, b, c = E.col(0), E.col(1), E.col(2)
    exprs = [(a * (E.dec("1.00") - b)) * (E.dec("1.00") + c), (a + b) / (c - E.dec("0.5")),
             -(a - b) * c + E.lit(3), E.rescale(a * b, 20, 1), (a / b) / c]
    vals = [edge_values(15, rng, 60) for _ in range(3)]
    for e in exprs:
        run_both(e, cols, vals, 60)


def _div(a, sa, b, sb):
    return pyref.div((1 if a < 0 else 0, abs(a), sa), (1 if b < 0 else 0, abs(b), sb))[0]


def test_known_answers_divide():
    # value checks re-derived from test/testcases/datatypes/test_decimal.cu:398-466
    # under the live rule (scale + 4, half-up)
    assert _div(100, 0, 10, 0) == (0, 100000, 4)            # 10.0000
    assert _div(-100, 0, 10, 0) == (1, 100000, 4)           # -10.0000
    assert _div(-100, 0, -10, 0) == (0, 100000, 4)          # 10.0000
    assert _div(-912345, 5, -39876, 4) == (0, 2287955161, 9)  # 2.287955161
    assert _div(0, 5, -39876, 4) == (0, 0, 9)               # +0, not -0
    # half-up: 1/3 -> 0.3333, 2/3 -> 0.6667
    assert _div(1, 0, 3, 0) == (0, 3333, 4)
    assert _div(2, 0, 3, 0) == (0, 6667, 4)
    # 64-bit branch wraps: |a|*10^shift taken mod 2^64 (AriesDecimal.hxx:581-596)
    a = (1 << 58) + 12345  # bitlen 59; shift 4 -> ref bits 14 -> 59+14-1 = 72 > 64: general branch
    q = _div(a, 0, 7, 0)
    assert q[1] == (a * 10 ** 4) // 7 + (1 if 2 * ((a * 10 ** 4) % 7) >= 7 else 0)
    a2 = (1 << 50) + 99  # bitlen 51 + 14 - 1 = 64 -> 64-bit branch, product >= 2^64 wraps
    q2 = _div(a2, 0, 3, 0)
    dvs = (a2 * 10 ** 4) & ((1 << 64) - 1)
    assert q2[1] == dvs // 3 + (1 if ((dvs % 3) << 1) >= 3 else 0)


def test_known_answers_mul_and_negative_zero():
    # test_decimal.cu:390-396: 709.87 * 4540 = 3222809.80
    r = pyref.mul((0, 70987, 2), (0, 4540, 0))
    assert r == (0, 322280980, 2)
    # sign XOR even for zero: -x * 0 = -0 (AriesDecimal.hxx:318)
    assert pyref.mul((1, 5, 0), (0, 0, 0)) == (1, 0, 0)
    # equal magnitudes of different signs add to +0 (AriesDecimal.hxx:214)
    assert pyref.add((1, 5, 1), (0, 50, 2)) == (0, 0, 2)
    # -0 < +0 (AriesDecimal.hxx:1023-1030)
    assert pyref.compare(0, (1, 0, 0), (0, 0, 0)) == 1


def test_oracle_group_agg_matches_python():
    rng = random.Random(5)
    rows, G = 500, 7
    vals = [(rng.randint(0, 1), rng.randint(0, 10 ** 15 - 1)) for _ in range(rows)]
    vals[3] = (1, 0)
    gids = [rng.randrange(G) for _ in range(rows)]
    raw = codec.encode(vals, 15)
    graw = b"".join(g.to_bytes(4, "little", signed=True) for g in gids)
    for kind in (abi.UP_AGG_SUM, abi.UP_AGG_AVG, abi.UP_AGG_COUNT):
        out = oracle.group_agg(raw, 7, 2, kind, graw, rows, G + 1)  # last group empty
        for g in range(G + 1):
            members = [v for v, gg in zip(vals, gids) if gg == g]
            tot = sum((-m if s else m) for s, m in members)
            if kind == abi.UP_AGG_COUNT:
                assert int.from_bytes(out[8 * g:8 * g + 8], "little") == len(members)
                continue
            img = codec.decode_agg(out[g * 133:(g + 1) * 133], 1)[0]
            if not members:
                assert img["flag"] == 0 and img["mag"] == 0
                continue
            if kind == abi.UP_AGG_SUM:
                assert (img["sign"], img["mag"], img["frac"]) == ((1 if tot < 0 else 0), abs(tot), 2)
            else:
                exp = pyref.div((1 if tot < 0 else 0, abs(tot), 2), (0, len(members), 0))[0]
                if exp[1] == 0:
                    exp = (exp[0], 0, exp[2])
                assert (img["sign"], img["mag"], img["frac"]) == exp


def test_tables_match_reference_values():
    # values quoted from src/datatypes/decimal.cu:92 at the workloads' precisions
    lib = abi.load()
    o = oracle.load()
    for p, b in [(15, 7), (16, 7), (18, 8), (31, 14), (37, 16), (38, 16), (47, 20), (76, 32), (77, 33), (100, 42),
                 (150, 63), (153, 64)]:
        assert lib.up_compact_bytes(p) == b == o.orc_compact_bytes(p)
    for p in range(1, 1100):
        assert lib.up_compact_bytes(p) == o.orc_compact_bytes(p)
        assert lib.up_precision_words(p) == o.orc_precision_words(p)
        # a compact field always holds every p-digit magnitude
        assert 8 * lib.up_compact_bytes(p) - 1 >= (10 ** p - 1).bit_length()


@pytest.mark.parametrize("conn", ["and_", "or_"])
def test_oracle_and_or(conn):
    """AND / OR of comparisons, nested, with a division under one side so the
    division-by-zero flag of either child is kept."""
    rng = random.Random(11)
    cols = [E.ColType(18, 4), E.ColType(15, 2), E.ColType(30, 10)]
    a, b, c = E.col(0), E.col(1), E.col(2)
    expr = getattr(a.lt(b), conn)(c.ge(a / b).or_(b.eq(0)))
    n = 150
    vals = [edge_values(18, rng, n), edge_values(15, rng, n), edge_values(30, rng, n)]
    run_both(expr, cols, vals, n)


def test_boolean_typing_rejects_mixed_children():
    from ultraprecise_b200 import abi as A
    a, b = E.col(0), E.col(1)
    cols = [E.ColType(10, 2), E.ColType(10, 2)]
    for bad in (a.and_(b), a.lt(b).or_(b), a.lt(b).lt(a.gt(b)), a + a.lt(b)):
        built = E.build([bad], cols)
        with pytest.raises(A.UpError):
            E.derive_types(built)


def test_oracle_null_semantics():
    """NULL handling of the oracle (the rules the GPU tests check the CUDA path
    against): a nullable value's flag byte 0 is NULL; an expression over a NULL
    is NULL (flag 0, zero value bytes, no row error); SUM/AVG skip NULL rows,
    a group without any non-NULL row has SUM and AVG flag 0, COUNT counts all
    rows of the group."""
    import numpy as np
    from oracle import oracle, pyref
    from ultraprecise_b200 import abi, codec
    from ultraprecise_b200 import expr as E
    nb = codec.compact_bytes(15)
    vals = [(0, 1234), (1, 50), (0, 7), (0, 0), (1, 999)]
    flags = [1, 0, 1, 0, 1]
    rx = b"".join(bytes([f]) + codec.encode([v], 15) for f, v in zip(flags, vals))
    ry = codec.encode([(0, 3), (0, 4), (0, 5), (0, 6), (0, 7)], 15)
    ct = [E.ColType(15, 2, nullable=True), E.ColType(15, 2)]
    x, y = E.col(0), E.col(1)
    b = E.build([x * y], ct)
    E.derive_types(b)
    ob = codec.compact_bytes(b.nodes[b.roots[0]].precision) + 1
    out, err = oracle.eval_expr(b, b.roots[0], [rx, ry], 5, ob)
    assert err == 0
    for i in range(5):
        row = out[i * ob:(i + 1) * ob]
        assert row[0] == flags[i]
        if flags[i]:
            (s, m, _) = pyref.mul(pyref.decode(codec.encode([vals[i]], 15), 2),
                                  pyref.decode(ry[i * nb:(i + 1) * nb], 2))
            assert row[1:] == pyref.encode((s, m, 4), ob - 1)[0]
        else:
            assert not any(row[1:])
    # grouped: groups 0,0,1,1,0 -> group 1 holds rows 2 (value) and 3 (NULL)
    q = E.build([x, x * y], ct)
    E.derive_types(q)
    gid = np.array([0, 0, 1, 1, 2], dtype=np.int32).tobytes()
    # group 2 gets only row 4 (a value); a group 3 has no rows at all
    aggs = [(abi.UP_AGG_SUM, q.roots[0]), (abi.UP_AGG_AVG, q.roots[1]), (abi.UP_AGG_COUNT, q.roots[0])]
    s_img, a_img, cnt = oracle.query(q, aggs, [rx, ry], gid, 5, 4)
    img = abi.UP_AGG_DECIMAL_BYTES
    counts = np.frombuffer(cnt, dtype=np.int64).tolist()
    assert counts == [2, 2, 1, 0]                              # COUNT(*): NULL rows counted
    assert int.from_bytes(s_img[5:img], "little") == 1234       # group 0: the NULL row is skipped
    assert s_img[img] == 1 and s_img[3 * img] == 0              # group 1 has a value, group 3 none
    g1_avg = a_img[img:2 * img]
    assert g1_avg[0] == 1 and int.from_bytes(g1_avg[5:], "little") == 7 * 5 * 10000  # AVG over 1 non-NULL row
