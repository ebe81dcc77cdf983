"""GPU parity of the cooperative evaluation (several threads per value,
carries passed by warp shuffles) against the oracle and the one-thread path,
byte for byte, for every group size."""
import random

import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from tests.helpers import edge_values
from ultraprecise_b200 import abi, codec, runtime
from ultraprecise_b200 import expr as E

pytestmark = pytest.mark.gpu


def _columns(p, rows, seed):
    """Edge and random values; every 7th row of column 1 repeats column 0 so
    that sums of opposite signs cancel to +0."""
    rng = random.Random(seed)
    v0 = edge_values(p, rng, rows)
    v1 = [v0[i] if i % 7 == 0 else x for i, x in enumerate(edge_values(p, rng, rows))]
    v2 = edge_values(p, rng, rows)
    return [v0, v1, v2]


def _run(e, types, raws, rows, tpv):
    m = runtime.compile_expr(e, types, threads_per_value=tpv)
    dev = [runtime.DeviceColumn.from_host(r, t.precision, t.scale) for r, t in zip(raws, types)]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = m.launch(dev, rows, err=err)
    torch.cuda.synchronize()
    return bytes(out.cpu().numpy().tobytes()), int(err.item())


def _oracle(e, types, raws, rows):
    b = E.build([e], types)
    E.derive_types(b)
    root = b.nodes[b.roots[0]]
    ob = 1 if root.kind in abi.COMPARE_KINDS else codec.compact_bytes(root.precision)
    return oracle.eval_expr(b, b.roots[0], raws, rows, ob, threads=8)


def _cases(kind):
    from ultraprecise_b200 import workloads
    names = {"mul": ("mad", "msub", "addsub", "const"), "div": ("div", "mod", "divmix", "trunc"), "sin": ("sin",)}
    groups = {}
    for name, p, e, types, tpv in workloads.coop_cases():
        if name in names[kind]:
            groups.setdefault((name, p), (e, types, []))[2].append(tpv)
    return [(name, p, e, types, tpvs) for (name, p), (e, types, tpvs) in sorted(groups.items(),
                                                                            key=lambda x: (x[0][1], x[0][0]))]


@pytest.mark.parametrize("name,p,e,types,tpvs", _cases("mul"), ids=lambda x: str(x)[:12])
def test_cooperative_matches_oracle(name, p, e, types, tpvs):
    rows = 3001
    raws = [codec.encode(v, p) for v in _columns(p, rows, seed=p * 31 + len(name))]
    exp, exp_err = _oracle(e, types, raws, rows)
    for tpv in tpvs:
        got, err = _run(e, types, raws, rows, tpv)
        assert got == exp, f"threads_per_value={tpv}"
        assert err == exp_err


@pytest.mark.parametrize("p", [150, 300])
def test_cooperative_products_rescale_compare(p):
    s = p // 5
    a, b, c = E.col(0), E.col(1), E.col(2)
    types = [E.ColType(p, s), E.ColType(p // 2, s // 2), E.ColType(p, s)]
    rows = 2000
    vals = _columns(p // 2, rows, seed=p)  # every value fits the narrowest column
    raws = [codec.encode(v, t.precision) for v, t in zip(vals, types)]
    for e in (a * b * c, E.rescale(a * b, 3 * p, s + s // 2 + 5), E.Expr(abi.UP_NODE_GE, a * b, c),
              E.Expr(abi.UP_NODE_EQ, a, c)):
        exp, exp_err = _oracle(e, types, raws, rows)
        one, _ = _run(e, types, raws, rows, 1)
        assert one == exp
        for tpv in (4, 16, 32):
            got, err = _run(e, types, raws, rows, tpv)
            assert got == exp and err == exp_err, f"threads_per_value={tpv}"




@pytest.mark.parametrize("name,p,e,types,tpvs", _cases("div"), ids=lambda x: str(x)[:12])
def test_cooperative_division_matches_oracle(name, p, e, types, tpvs):
    """Division in every branch of the divide rule: zero dividends and
    divisors (edge values include zeros), small operands (the 64-bit branch),
    one-limb divisors (remainder doubled mod 2^32), and wide divisors."""
    rows = 3001
    vals = _columns(p, rows, seed=p * 7 + len(name))
    # small values on some rows: one-limb divisors and the 64-bit branch
    vals[0] = [(sg, m % 10 ** 12) if i % 5 == 1 else (sg, m) for i, (sg, m) in enumerate(vals[0])]
    vals[1] = [(sg, m % 10 ** 9) if i % 3 == 1 else (sg, m) for i, (sg, m) in enumerate(vals[1])]
    raws = [codec.encode(v, p) for v in vals]
    exp, exp_err = _oracle(e, types, raws, rows)
    for tpv in tpvs:
        got, err = _run(e, types, raws, rows, tpv)
        assert got == exp, f"threads_per_value={tpv}"
        assert err == exp_err


@pytest.mark.parametrize("name,p,e,types,tpvs", _cases("sin"), ids=lambda x: str(x)[:12])
def test_cooperative_sin_matches_oracle(name, p, e, types, tpvs):
    from ultraprecise_b200 import workloads
    rows = 1500
    pi = workloads.pi_scaled(p - 2)
    raw = codec.encode([(0, 0), (1, 0), (0, pi), (1, pi), (0, 1)], p) + workloads.sin_inputs(p, rows - 5, seed=p)
    exp, exp_err = _oracle(e, types, [raw], rows)
    for tpv in tpvs:
        got, err = _run(e, types, [raw], rows, tpv)
        assert got == exp
        assert err == exp_err
