"""CPU: the oracle reproduces golden vectors produced by the reference's own
AriesDecimal<LEN> device code (tests/golden/make_golden.py, run on a GPU host
with the reference harness), byte for byte."""
import json
import os

import pytest

from oracle import oracle
from tests.golden import make_golden
from ultraprecise_b200 import expr as E

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.json")

pytestmark = pytest.mark.skipif(not os.path.exists(PATH), reason="golden vectors not generated yet")


def _cases():
    if not os.path.exists(PATH):
        return []
    return json.load(open(PATH))["cases"]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c["name"])
def test_oracle_reproduces_reference_vectors(case):
    types = [E.ColType(p, s) for p, s in case["types"]]
    b = E.build([make_golden.expr_for(case["op"])], types)
    E.derive_types(b)
    raws = [bytes.fromhex(h) for h in case["inputs"]]
    got, _ = oracle.eval_expr(b, b.roots[0], raws, case["rows"], case["out_bytes"])
    assert got.hex() == case["output"]
