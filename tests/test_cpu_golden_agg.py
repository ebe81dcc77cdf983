"""CPU: the oracle reproduces golden vectors made by the reference's own
32-limb Decimal code (tests/golden/make_agg_golden.py, run on a GPU host with
oracle/_ref/libariesref_agg.so): grouped SUM through the XMP segmented add,
AVG through nullable_type<Decimal> /= int64, text parse through the CSV
import's constructor, and GetDecimal text.

Rules of the comparison (the parity contract):
* SUM images are compared byte for byte, except that a zero sum may carry
  sign 1 in the reference (-0: equal magnitudes of opposite signs give the
  second operand's sign in operator_add, decimal.cu:3359-3369, so it depends
  on the reduction order); the oracle and the CUDA path give +0;
* AVG images are compared byte for byte;
* parsed values are compared byte for byte, and the reference's overflow
  error (ERR_OVER_FLOW) must come with UP_ROWERR_OVERFLOW.
"""
import json
import os

import pytest

from oracle import oracle, pyref
from ultraprecise_b200 import abi

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_agg_vectors.json")

pytestmark = pytest.mark.skipif(not os.path.exists(PATH), reason="aggregate golden vectors not generated yet")

IMG = abi.UP_AGG_DECIMAL_BYTES


def _load(kind):
    if not os.path.exists(PATH):
        return []
    return json.load(open(PATH))[kind]


def _segment_ids(starts, rows, assoc):
    """group id per row from the segments of visiting positions"""
    gid = [0] * rows
    ends = list(starts[1:]) + [rows]
    for g, (b, e) in enumerate(zip(starts, ends)):
        for i in range(b, e):
            gid[assoc[i] if assoc is not None else i] = g
    return gid


def _same_sum(exp: bytes, got: bytes) -> bool:
    if exp == got:
        return True
    mag_zero = not any(exp[5:IMG])
    return mag_zero and exp[1] == 1 and got[1] == 0 and exp[:1] + exp[2:] == got[:1] + got[2:]


@pytest.mark.parametrize("case", _load("sum"), ids=lambda c: c["name"])
def test_oracle_sum_matches_reference(case):
    import numpy as np
    rows, starts = case["rows"], case["starts"]
    nb = oracle.compact_bytes(case["p"])
    gid = np.array(_segment_ids(starts, rows, case["assoc"]), dtype=np.int32).tobytes()
    got = oracle.group_agg(bytes.fromhex(case["input"]), nb, case["s"], abi.UP_AGG_SUM, gid, rows, len(starts))
    exp = bytes.fromhex(case["output"])
    for g in range(len(starts)):
        assert _same_sum(exp[g * IMG:(g + 1) * IMG], got[g * IMG:(g + 1) * IMG]), f"group {g}"


@pytest.mark.parametrize("case", _load("avg"), ids=lambda c: c["name"])
def test_oracle_avg_matches_reference(case):
    sums = bytes.fromhex(case["sums"])
    exp = bytes.fromhex(case["output"])
    for k, cnt in enumerate(case["counts"]):
        got = oracle.division_int64(sums[k * IMG:(k + 1) * IMG], cnt)
        assert got == exp[k * IMG:(k + 1) * IMG], f"count {cnt} (entry {k})"


@pytest.mark.parametrize("case", _load("parse"), ids=lambda c: c["name"])
def test_restated_parse_matches_reference(case):
    nb = oracle.compact_bytes(case["p"])
    exp = bytes.fromhex(case["output"])
    for i, (txt, rerr) in enumerate(zip(case["fields"], case["errors"])):
        got, err = pyref.parse_decimal(txt.encode(), nb, case["s"])
        assert got == exp[i * nb:(i + 1) * nb], txt
        assert bool(err & abi.UP_ROWERR_OVERFLOW) == (rerr == 1), (txt, rerr, err)


@pytest.mark.parametrize("case", _load("format"), ids=lambda c: c["name"])
def test_restated_format_matches_reference(case):
    nb = oracle.compact_bytes(case["p"])
    raw = bytes.fromhex(case["input"])
    for i, exp in enumerate(case["output"]):
        assert pyref.format_decimal(raw[i * nb:(i + 1) * nb], case["s"], hex_image=True) == exp
