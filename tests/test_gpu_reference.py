"""GPU: the CUDA path against the reference's own AriesDecimal<LEN> code
(oracle/_ref/libariesref.so, built from the reference sources by
oracle/ref/Makefile), run with a limb count large enough for exact
intermediates.  Byte-exact."""
import random

import pytest

torch = pytest.importorskip("torch")

from tests.golden import make_golden, refharness
from ultraprecise_b200 import codec, runtime
from ultraprecise_b200 import expr as E

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refharness.available(), reason="reference harness not built")]


def _ours(op, types, raws, rows):
    cols = [E.ColType(p, s) for p, s in types]
    m = runtime.compile_expr(make_golden.expr_for(op), cols)
    dev = [runtime.DeviceColumn.from_host(r, p, s) for r, (p, s) in zip(raws, types)]
    out = m.launch(dev, rows)
    torch.cuda.synchronize()
    return bytes(out.cpu().numpy().tobytes()), m.value_bytes


def _ref(op, types, raws, rows, ob):
    devs = [torch.frombuffer(bytearray(r), dtype=torch.uint8).cuda() for r in raws]
    out = torch.zeros(rows * ob, dtype=torch.uint8, device="cuda")
    c = devs[2].data_ptr() if len(devs) > 2 else None
    pc, sc = types[2] if len(types) > 2 else (0, 0)
    refharness.run(op, devs[0].data_ptr(), types[0][0], types[0][1], devs[1].data_ptr(), types[1][0], types[1][1],
                   rows, out.data_ptr(), ob, c_dev=c, pc=pc, sc=sc, b_host=raws[1])
    torch.cuda.synchronize()
    return bytes(out.cpu().numpy().tobytes())


@pytest.mark.parametrize("p", [18, 38, 76, 150])
@pytest.mark.parametrize("op", ["mad", "div"])
def test_sweep_shapes_match_reference(p, op):
    s = p // 4
    if op == "div" and s + 4 > 38:
        pytest.skip("outside the reference's 10^38 table")
    rng = random.Random(1000 * p + len(op))
    rows = 2048
    types = [(p, s)] * (3 if op == "mad" else 2)
    vals = [make_golden.digits_values(p, rng, rows, nonzero=(op == "div" and k == 1)) for k in range(len(types))]
    raws = [codec.encode(v, p) for v in vals]
    got, ob = _ours(op, types, raws, rows)
    assert got == _ref(op, types, raws, rows, ob)


@pytest.mark.parametrize("op", ["q_dp", "q_charge"])
def test_query_expressions_match_reference(op):
    rng = random.Random(17)
    rows = 20000
    case = {"op": op, "types": [[15, 2]] * 3, "rows": rows, "dist": "query"}
    vals = make_golden.gen_inputs(case, rng)
    raws = [codec.encode(v, 15) for v in vals]
    types = [(15, 2)] * 3
    got, ob = _ours(op, types, raws, rows)
    assert got == _ref(op, types, raws, rows, ob)


@pytest.mark.parametrize("pair", make_golden.OP_PAIRS, ids=lambda t: f"{t[0]}x{t[1]}")
def test_all_operators_match_reference_on_edge_values(pair):
    rng = random.Random(hash(pair) & 0xFFFF)
    (pa, sa), (pb, sb) = pair
    for op in make_golden.OPS:
        if op == "div" and sb + 4 > 38:
            continue
        case = {"op": op, "types": [[pa, sa], [pb, sb]], "rows": 300, "dist": "edge"}
        vals = make_golden.gen_inputs(case, rng)
        raws = [codec.encode(v, p) for v, (p, _) in zip(vals, case["types"])]
        types = [(pa, sa), (pb, sb)]
        got, ob = _ours(op, types, raws, 300)
        assert got == _ref(op, types, raws, 300, ob), op
