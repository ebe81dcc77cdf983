"""GPU: the CUDA path against the reference's own 32-limb Decimal code
(oracle/_ref/libariesref_agg.so, built from decimal.cu by oracle/ref/Makefile):

* grouped SUM (up_aggregate_column_data, the AggregateColumnData form, and
  the fused query kernels) against the XMP segmented-reduction add;
* AVG (up_division_int64 and the fused query's AVG) against
  nullable_type<Decimal> /= int64;
* up_parse_decimal against the CSV import's Decimal(p, s, STRICT, text);
* up_format_decimal (hex image) against Decimal::GetDecimal.

Byte-exact, except that a zero SUM may be -0 in the reference (its sign
depends on the reduction order there) where this path gives +0."""
import random

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tests.golden import make_agg_golden, make_golden, refharness
from tests.test_cpu_golden_agg import _same_sum
from ultraprecise_b200 import abi, codec, runtime, workloads
from ultraprecise_b200 import expr as E

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refharness.agg_available(), reason="aggregate reference harness not built")]

IMG = abi.UP_AGG_DECIMAL_BYTES


def _acd(raw: bytes, p: int, s: int, kind: int, assoc, starts, rows):
    """up_aggregate_column_data over a host column."""
    lib = abi.load()
    col = runtime.DeviceColumn.from_host(raw, p, s)
    a = torch.tensor(assoc, dtype=torch.int32, device="cuda")
    st = torch.tensor(starts, dtype=torch.int32, device="cuda")
    out = torch.zeros(len(starts) * IMG, dtype=torch.uint8, device="cuda")
    arr = runtime._columns_array([col])
    abi.check(lib.up_aggregate_column_data(arr, kind, a.data_ptr(), st.data_ptr(), len(starts), rows,
                                           out.data_ptr(), None, torch.cuda.current_stream().cuda_stream),
              "up_aggregate_column_data")
    torch.cuda.synchronize()
    return bytes(out.cpu().numpy().tobytes())


def _segments(rng, rows, n_groups):
    cuts = sorted(rng.sample(range(1, rows), n_groups - 1))
    return [0] + cuts


@pytest.mark.parametrize("p,s", [(15, 2), (18, 4), (38, 9), (76, 19), (150, 37)])
@pytest.mark.parametrize("dist", ["digits", "edge"])
def test_aggregate_column_sum_and_avg_match_reference(p, s, dist):
    rng = random.Random(p * 31 + len(dist))
    rows, G = 3000, 37
    vals = (make_golden.digits_values(p, rng, rows) if dist == "digits" else make_golden.edge_values(p, rng, rows))
    raw = codec.encode(vals, p)
    starts = _segments(rng, rows, G)
    assoc = list(range(rows))
    rng.shuffle(assoc)
    exp = refharness.sum_segments(raw, p, s, starts, rows, assoc)
    got = _acd(raw, p, s, abi.UP_AGG_SUM, assoc, starts, rows)
    for g in range(G):
        assert _same_sum(exp[g * IMG:(g + 1) * IMG], got[g * IMG:(g + 1) * IMG]), f"SUM group {g}"
    counts = [e - b for b, e in zip(starts, starts[1:] + [rows])]
    exp_avg = refharness.div_int64(exp, counts)
    got_avg = _acd(raw, p, s, abi.UP_AGG_AVG, assoc, starts, rows)
    for g in range(G):
        e_img = exp_avg[g * IMG:(g + 1) * IMG]
        if not any(exp[g * IMG + 5:(g + 1) * IMG]) and exp[g * IMG + 1] == 1:
            continue  # a -0 sum in the reference: its AVG sign follows that -0
        assert got_avg[g * IMG:(g + 1) * IMG] == e_img, f"AVG group {g}"


def test_division_int64_matches_reference_on_chosen_counts():
    rng = random.Random(5)
    case = make_agg_golden.sum_cases(rng)[3]  # a digits case of DECIMAL(18,4)
    raw = bytes.fromhex(case["input"])
    sums = refharness.sum_segments(raw, case["p"], case["s"], case["starts"], case["rows"], case["assoc"])
    n = len(case["starts"])
    counts = [1, 2, 3, 7, 10, 12345, (1 << 31) - 1, (1 << 32) - 1, (1 << 32) + 5, (1 << 40) + 3, 0]
    imgs = b"".join(sums[IMG * (k % n):IMG * (k % n) + IMG] for k in range(len(counts)))
    exp = refharness.div_int64(imgs, counts)
    lib = abi.load()
    s_dev = torch.frombuffer(bytearray(imgs), dtype=torch.uint8).cuda()
    c_dev = torch.tensor(counts, dtype=torch.int64, device="cuda")
    out = torch.zeros(len(counts) * IMG, dtype=torch.uint8, device="cuda")
    abi.check(lib.up_division_int64(s_dev.data_ptr(), c_dev.data_ptr(), len(counts), out.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream), "up_division_int64")
    torch.cuda.synchronize()
    got = bytes(out.cpu().numpy().tobytes())
    for k, c in enumerate(counts):
        assert got[k * IMG:(k + 1) * IMG] == exp[k * IMG:(k + 1) * IMG], f"count {c}"


def test_grouped_query_matches_reference_expression_and_sum():
    """The fused grouped query (SUM x4, AVG x3, COUNT over DECIMAL(15,2)
    columns) against the reference end to end: its expression values come
    from the reference's AriesDecimal<LEN> (ref_harness.cu), its SUM and AVG
    from the reference's XMP add and Decimal /= int64."""
    if not refharness.available():
        pytest.skip("element-wise reference harness not built")
    rng = random.Random(77)
    rows = 6000
    R = workloads.QUERY_RANGES
    vals = {n: [(0, rng.randrange(R[n][0], R[n][1] + 1, R[n][2])) for _ in range(rows)] for n in R}
    raws = {n: codec.encode(v, 15) for n, v in vals.items()}
    G = 4
    gid = np.array([rng.choices(range(G), weights=[25, 0.7, 49.3, 25])[0] for _ in range(rows)], dtype=np.int32)
    exprs, aggs, ct = workloads.query_exprs()
    q = runtime.compile_query(exprs, aggs, ct)
    dev = [runtime.DeviceColumn.from_host(raws[n], 15, 2) for n in ("qty", "price", "disc", "tax")]
    outs = q.launch(dev, torch.from_numpy(gid).cuda(), G)
    torch.cuda.synchronize()
    got = [bytes(o.cpu().numpy().tobytes()) for o in outs]
    # reference expression columns: price*(1-disc) (31,4) and *(1+tax) (47,6)
    ref_cols = {"qty": (raws["qty"], 15, 2), "price": (raws["price"], 15, 2), "disc": (raws["disc"], 15, 2)}
    for op, name, (p, s) in (("q_dp", "dp", (31, 4)), ("q_charge", "charge", (47, 6))):
        ob = codec.compact_bytes(p)
        devs = [torch.frombuffer(bytearray(raws[n]), dtype=torch.uint8).cuda() for n in ("price", "disc", "tax")]
        o = torch.zeros(rows * ob, dtype=torch.uint8, device="cuda")
        refharness.run(op, devs[0].data_ptr(), 15, 2, devs[1].data_ptr(), 15, 2, rows, o.data_ptr(), ob,
                       c_dev=devs[2].data_ptr(), pc=15, sc=2)
        torch.cuda.synchronize()
        ref_cols[name] = (bytes(o.cpu().numpy().tobytes()), p, s)
    order = np.argsort(gid, kind="stable")
    counts = np.bincount(gid, minlength=G)
    starts = [0] + list(np.cumsum(counts)[:-1])
    sources = ["qty", "price", "dp", "charge", "qty", "price", "disc"]
    for i, (kind, _) in enumerate(aggs):
        if kind == abi.UP_AGG_COUNT:
            assert np.frombuffer(got[i][:8 * G], dtype=np.int64).tolist() == counts.tolist()
            continue
        raw, p, s = ref_cols[sources[i]]
        sums = refharness.sum_segments(raw, p, s, [int(x) for x in starts], rows, [int(x) for x in order])
        exp = sums if kind == abi.UP_AGG_SUM else refharness.div_int64(sums, [int(c) for c in counts])
        assert got[i][:G * IMG] == exp, f"aggregate {i}"


@pytest.mark.parametrize("p,s", make_agg_golden.PARSE_TYPES)
def test_parse_matches_reference(p, s):
    rng = random.Random(p + 1000 * s)
    fields = make_agg_golden.parse_fields(rng, p, s, 2000)
    exp, errs = refharness.parse(fields, p, s)
    got, _ = runtime.parse_decimal(fields, p, s)
    torch.cuda.synchronize()
    got = bytes(got.cpu().numpy().tobytes())
    nb = codec.compact_bytes(p)
    for i, f in enumerate(fields):
        if errs[i] == 1:
            continue  # overflow rows: compared by the CPU golden test's error rule
        assert got[i * nb:(i + 1) * nb] == exp[i * nb:(i + 1) * nb], f


@pytest.mark.parametrize("p,s", make_agg_golden.FORMAT_TYPES)
def test_hex_format_matches_reference(p, s):
    rng = random.Random(3 * p + s)
    vals = make_golden.edge_values(p, rng, 500) + make_golden.digits_values(p, rng, 500)
    raw = codec.encode(vals, p)
    exp = refharness.format_hex(raw, len(vals), p, s)
    col = torch.frombuffer(bytearray(raw), dtype=torch.uint8).cuda()
    got = runtime.format_strings(col, len(vals), p, s, hex_image=True)
    assert got == exp
