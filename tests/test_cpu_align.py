"""CPU: the AlignOptimize rewrite (AriesEngineShell.cpp:244-685)."""
import random
from fractions import Fraction

from oracle import oracle
from ultraprecise_b200 import abi, codec
from ultraprecise_b200 import expr as E
from tests.helpers import edge_values


def opt(root, cols):
    b = E.build([root], cols)
    return E.align_optimize(b)


def describe(b, k=None):
    k = b.roots[0] if k is None else k
    nd = b.nodes[k]
    names = {0: "col", 1: "dec", 2: "int", 3: "+", 4: "-", 5: "*", 6: "/", 7: "%"}
    if nd.kind == abi.UP_NODE_COLUMN:
        s = f"c{nd.column}"
    elif nd.kind == abi.UP_NODE_CONST:
        mag = sum(nd.const_limbs[i] << (32 * i) for i in range(nd.const_nlimbs))
        s = codec.to_str(nd.const_sign, mag, nd.scale)
    elif nd.kind == abi.UP_NODE_INT:
        s = str(nd.int_value)
    else:
        s = f"({describe(b, nd.left)} {names[nd.kind]} {describe(b, nd.right)})"
    return ("-" + s) if nd.reverse else s


def test_one_minus_disc_becomes_decimal_constant():
    cols = [E.ColType(15, 2)] * 4
    b = opt(E.lit(1) - E.col(2), cols)
    assert describe(b) == "(1.00 - c2)"
    assert E.node_type(b, b.roots[0]) == (16, 2)


def test_query_expression_typing():
    cols = [E.ColType(15, 2)] * 4
    price, disc, tax = E.col(1), E.col(2), E.col(3)
    b = opt(price * (E.lit(1) - disc) * (E.lit(1) + tax), cols)
    assert describe(b) == "((c1 * (1.00 - c2)) * (1.00 + c3))"
    assert E.node_type(b, b.roots[0]) == (47, 6)


def test_addends_ordered_by_scale():
    for p in (18, 38, 76):
        s = p // 4
        cols = [E.ColType(p, s)] * 3
        b = opt(E.col(0) * E.col(1) + E.col(2), cols)
        assert describe(b) == "(c2 + (c0 * c1))"
        assert E.node_type(b, b.roots[0]) == (2 * p + 1, 2 * s)


def test_reference_comment_example():
    # AriesEngineShell.cpp:107-108: 1+l_tax+l_discount*(0/l_extendedprice)+1
    # "result precision changes from (21,6) to (13,2)"
    cols = [E.ColType(12, 2), E.ColType(15, 2), E.ColType(15, 2)]
    tax, disc, ext = E.col(0), E.col(1), E.col(2)
    b = opt(E.lit(1) + tax + disc * (E.lit(0) / ext) + E.lit(1), cols)
    assert describe(b) == "(2.00 + c0)"
    assert E.node_type(b, b.roots[0]) == (13, 2)


def test_subtraction_and_negation_pushed_down():
    cols = [E.ColType(10, 2), E.ColType(10, 3), E.ColType(10, 1)]
    a, b_, c = E.col(0), E.col(1), E.col(2)
    b = opt(a - (b_ - c), cols)
    # a + (-(b - c)) = a + (-b) + c, addends by scale: c(1), a(2), -b(3)
    assert describe(b) == "((c2 + c0) - c1)"


def test_reference_value_defects_are_not_reproduced():
    # the reference folds a-2*b to a+2*b (MUL folding ignores the constant's
    # reversal) and x*1 to 0 (RemoveZeroNode zeroes any INTEGER under MUL)
    cols = [E.ColType(10, 2), E.ColType(10, 2)]
    b = opt(E.col(0) - E.lit(2) * E.col(1), cols)
    assert describe(b) == "(c0 + (c1 * -2))"
    b = opt(E.col(0) * E.lit(1), cols)
    assert describe(b) == "(c0 * 1)"


def _value(b, cols_t, raws, rows):
    # values are compared at a wide output width: the reference's typing gives
    # folded constants precision 0, so a rewritten root can be declared
    # narrower than its values (they would overflow the column, as there)
    nd = b.nodes[b.roots[0]]
    ob = codec.compact_bytes(80)
    out, _ = oracle.eval_expr(b, b.roots[0], raws, rows, ob)
    vals = []
    for i in range(rows):
        raw = bytearray(out[i * ob:(i + 1) * ob])
        sign = raw[-1] >> 7
        raw[-1] &= 0x7F
        m = int.from_bytes(raw, "little")
        vals.append(Fraction(-m if sign else m, 10 ** nd.scale))
    return vals


def test_rewrite_preserves_values_of_random_trees():
    rng = random.Random(42)
    cols = [E.ColType(12, 2), E.ColType(10, 4), E.ColType(14, 0)]
    for trial in range(40):
        def rand_tree(depth):
            if depth == 0 or rng.random() < 0.3:
                r = rng.random()
                if r < 0.6:
                    return E.col(rng.randrange(3))
                if r < 0.8:
                    return E.lit(rng.randint(-5, 9))
                return E.dec(f"{rng.randint(0, 99)}.{rng.randint(0, 99):02d}")
            op = rng.choice(["+", "-", "*"])
            a, b_ = rand_tree(depth - 1), rand_tree(depth - 1)
            return a + b_ if op == "+" else (a - b_ if op == "-" else a * b_)
        root = rand_tree(3)
        b0 = E.build([root], cols)
        E.derive_types(b0)
        b1 = E.align_optimize(b0)
        if b1.nodes[b1.roots[0]].kind == abi.UP_NODE_INT:
            continue  # folded to zero (includes the x*1 quirk)
        rows = 50
        raws = [codec.encode(edge_values(c.precision, rng, rows), c.precision) for c in cols]
        v0 = _value(b0, cols, raws, rows)
        v1 = _value(b1, cols, raws, rows)
        assert v0 == v1, (trial, describe(b0), describe(b1))
