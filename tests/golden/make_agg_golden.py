"""Generate golden vectors for grouped SUM, AVG and decimal text from the
reference's own 32-limb Decimal code.

Runs on a GPU host with oracle/_ref/libariesref_agg.so (decimal.cu and the
harness of oracle/ref/ref_agg_harness.cu, built by oracle/ref/Makefile):

* SUM: seeded compact columns cut into segments of many lengths, each segment
  summed by the reference's XMP segmented-reduction add; the 133-byte images;
* AVG: those images (and a few chosen ones) divided by int64 counts with the
  reference's nullable_type<Decimal> /= int64;
* parse: decimal text fields through the CSV import's Decimal(p, s, STRICT,
  text) + ToCompactDecimal, with the error code per field;
* format: compact values through Decimal::GetDecimal.

Writes tests/golden/reference_agg_vectors.json; tests/test_cpu_golden_agg.py
checks the CPU oracle against it on every run, without a GPU.

    python tests/golden/make_agg_golden.py [--out tests/golden/reference_agg_vectors.json]
"""
from __future__ import annotations

import argparse
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden import make_golden, refharness  # noqa: E402
from ultraprecise_b200 import codec  # noqa: E402

SUM_TYPES = [(15, 2), (18, 4), (38, 9), (47, 6), (76, 19)]
SEGMENTS = [1, 2, 3, 7, 31, 100, 257, 1000]
PARSE_TYPES = [(15, 2), (38, 9), (76, 19), (9, 0)]
FORMAT_TYPES = [(15, 2), (38, 9), (76, 19), (150, 37)]


def sum_cases(rng: random.Random):
    out = []
    for p, s in SUM_TYPES:
        for dist in ("edge", "digits", "cancel"):
            lens = list(SEGMENTS)
            rng.shuffle(lens)
            rows = sum(lens)
            if dist == "edge":
                vals = make_golden.edge_values(p, rng, rows)
            elif dist == "digits":
                vals = make_golden.digits_values(p, rng, rows)
            else:
                # every segment holds values and their negations (exact
                # cancellation), then one extra value for half the segments
                vals = []
                for n in lens:
                    half = [(rng.randint(0, 1), int("".join(rng.choice("0123456789") for _ in range(p))))
                            for _ in range(n // 2)]
                    seg = half + [(1 - sg, m) for sg, m in half]
                    if len(seg) < n:
                        seg.append((rng.randint(0, 1), rng.randint(0, 10 ** min(p, 18))))
                    rng.shuffle(seg)
                    vals += seg
            starts, a = [], 0
            for n in lens:
                starts.append(a)
                a += n
            assoc = None
            if dist == "digits":  # visit the rows through a permutation, as AggregateColumnData does
                assoc = list(range(rows))
                rng.shuffle(assoc)
            out.append({"name": f"sum_{dist}_{p}_{s}", "p": p, "s": s, "rows": rows, "starts": starts,
                        "assoc": assoc, "input": codec.encode(vals, p).hex()})
    return out


def avg_counts(rng: random.Random, starts, rows):
    ends = list(starts[1:]) + [rows]
    counts = [e - b for b, e in zip(starts, ends)]
    # a few other divisors: 1, odd, near 2^32, above 2^32 (64-bit divisor), 0
    extra = [1, 3, 7, 12345, (1 << 32) - 1, (1 << 32) + 5, (1 << 40) + 3, 0]
    return counts, extra


def parse_fields(rng: random.Random, p: int, s: int, n: int):
    out = [b"0", b"-0", b"1", b"-1", b"0.5", b"-0.25"]
    ip = p - s
    out.append(("9" * ip + ("." + "9" * s if s else "")).encode())            # largest value
    out.append(("-" + "9" * ip + ("." + "9" * s if s else "")).encode())
    out.append(("1" + "0" * (ip - 1) + ".5").encode())
    while len(out) < n:
        di = rng.randint(1, ip)
        df = rng.randint(0, s + 3)  # fewer, as many and more fraction digits than the scale keeps
        txt = "".join(rng.choice("0123456789") for _ in range(di))
        if df:
            txt += "." + "".join(rng.choice("0123456789") for _ in range(df))
        if rng.random() < 0.5:
            txt = "-" + txt
        out.append(txt.encode())
    return out[:n]


def main():
    import torch  # noqa: F401  (the harness wrapper moves buffers with torch)
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "reference_agg_vectors.json"))
    a = ap.parse_args()
    rng = random.Random(20261204)
    res = {"generator": "tests/golden/make_agg_golden.py (the reference's decimal.cu via "
                        "oracle/_ref/libariesref_agg.so)", "sum": [], "avg": [], "parse": [], "format": []}
    for case in sum_cases(rng):
        raw = bytes.fromhex(case["input"])
        imgs = refharness.sum_segments(raw, case["p"], case["s"], case["starts"], case["rows"], case["assoc"])
        case["output"] = imgs.hex()
        res["sum"].append(case)
        counts, extra = avg_counts(rng, case["starts"], case["rows"])
        n = len(counts)
        all_imgs = imgs + b"".join(imgs[133 * (k % n):133 * (k % n) + 133] for k in range(len(extra)))
        all_counts = counts + extra
        out = refharness.div_int64(all_imgs, all_counts)
        res["avg"].append({"name": "avg_of_" + case["name"], "sums": all_imgs.hex(), "counts": all_counts,
                           "output": out.hex()})
        print(case["name"], "groups", n, "rows", case["rows"])
    for p, s in PARSE_TYPES:
        fields = parse_fields(rng, p, s, 200)
        comp, err = refharness.parse(fields, p, s)
        res["parse"].append({"name": f"parse_{p}_{s}", "p": p, "s": s, "fields": [f.decode() for f in fields],
                             "output": comp.hex(), "errors": list(err)})
        print("parse", p, s)
    for p, s in FORMAT_TYPES:
        vals = make_golden.edge_values(p, rng, 100) + make_golden.digits_values(p, rng, 100)
        raw = codec.encode(vals, p)
        strs = refharness.format_hex(raw, len(vals), p, s)
        res["format"].append({"name": f"format_{p}_{s}", "p": p, "s": s, "input": raw.hex(), "output": strs})
        print("format", p, s)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=0)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
