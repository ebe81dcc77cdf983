"""The sin(x) series workload (DECIMAL(p, p-2), 20 Horner terms with RESCALE
truncation): the oracle against an exact Python-integer restatement of the
same rules, and the series against sin(x) itself."""
import decimal
import random

import pytest

from oracle import oracle
from ultraprecise_b200 import codec, workloads
from ultraprecise_b200 import expr as E


def _oracle_sin(p, vals):
    e, cols = workloads.sin_expr(p)
    b = E.build([e], cols)
    E.derive_types(b)
    root = b.nodes[b.roots[0]]
    assert (root.precision, root.scale) == (p, p - 2)
    ob = codec.compact_bytes(p)
    out, err = oracle.eval_expr(b, b.roots[0], [codec.encode(vals, p)], len(vals), ob)
    return codec.decode(out, ob), err


@pytest.mark.parametrize("p", [100, 300, 1000])
def test_oracle_matches_python_series(p):
    s = p - 2
    pi = workloads.pi_scaled(s)
    rng = random.Random(p)
    vals = [(rng.randint(0, 1), rng.randint(0, pi)) for _ in range(24)]
    vals += [(0, 0), (1, 0), (0, pi), (1, pi), (0, 1), (1, 1), (0, 10 ** s), (1, 10 ** s // 2)]
    got, err = _oracle_sin(p, vals)
    assert err == 0
    for v, g in zip(vals, got):
        assert tuple(g) == workloads.sin_python(v[0], v[1], p), v


@pytest.mark.parametrize("p", [100, 300])
def test_series_close_to_sin(p):
    """20 terms at x = +-pi leave a truncation error below 1e-28."""
    s = p - 2
    decimal.getcontext().prec = p + 20
    pi = workloads.pi_scaled(s)
    vals = [(0, pi), (1, pi // 3), (0, 12345 * 10 ** (s - 5))]
    got, _ = _oracle_sin(p, vals)
    for (xs, xm), (gs, gm) in zip(vals, got):
        x = decimal.Decimal(xm).scaleb(-s) * (-1 if xs else 1)
        tot, term, k = decimal.Decimal(0), x, 1
        while term != 0 and abs(term) > decimal.Decimal(10) ** (-(p + 5)):
            tot += term
            term = -term * x * x / ((2 * k) * (2 * k + 1))
            k += 1
        v = decimal.Decimal(gm).scaleb(-s) * (-1 if gs else 1)
        assert abs(v - tot) < decimal.Decimal("1e-28")


def test_inputs_in_range():
    raw = workloads.sin_inputs(100, 1000, 5)
    vals = codec.decode(raw, codec.compact_bytes(100))
    pi = workloads.pi_scaled(98)
    assert all(0 <= m <= pi for _, m in vals)
    assert 400 < sum(sg for sg, _ in vals) < 600
