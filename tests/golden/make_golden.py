"""Generate golden vectors from the reference's own decimal code.

Runs on a GPU host with oracle/_ref/libariesref.so (the reference's
AriesDecimal<LEN> compiled by oracle/ref/Makefile).  For every case it draws
seeded inputs, evaluates them with the reference at a limb count large enough
for exact intermediates, and writes inputs + reference outputs to
tests/golden/reference_vectors.json.  tests/test_cpu_golden.py then checks the
CPU oracle against these vectors on every run, without a GPU.

    python tests/golden/make_golden.py [--out tests/golden/reference_vectors.json]
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

from tests.golden import refharness  # noqa: E402
from ultraprecise_b200 import codec  # noqa: E402
from ultraprecise_b200 import expr as E  # noqa: E402

OP_PAIRS = [((15, 2), (15, 2)), ((18, 4), (18, 4)), ((9, 9), (12, 0)), ((38, 9), (38, 9)), ((38, 9), (20, 3)),
            ((76, 19), (76, 19)), ((30, 12), (5, 5)), ((150, 34), (40, 30))]
OPS = ["add", "sub", "mul", "div", "mod", "lt", "le", "gt", "ge", "eq", "ne"]


def edge_values(p: int, rng: random.Random, n: int):
    top = 10 ** p - 1
    base = [(0, 0), (1, 0), (0, 1), (1, 1), (0, top), (1, top), (0, top // 2), (1, 10 ** (p - 1))]
    for k in (31, 32, 33, 63, 64, 65, 95, 96, 127, 128, 255, 256):
        v = (1 << k) - 1
        if v <= top:
            base += [(0, v), (1, min(v + 1, top))]
    out = base[:n]
    while len(out) < n:
        d = rng.randint(1, p)
        mag = int("".join(rng.choice("0123456789") for _ in range(d)))
        out.append((rng.randint(0, 1), mag))
    rng.shuffle(out)
    return out


def digits_values(p: int, rng: random.Random, n: int, nonzero=False):
    out = []
    for _ in range(n):
        while True:
            mag = int("".join(rng.choice("0123456789") for _ in range(p)))
            if mag or not nonzero:
                break
        out.append((rng.randint(0, 1), mag))
    return out


def expr_for(op: str):
    a, b, c = E.col(0), E.col(1), E.col(2)
    if op == "mad":
        return c + a * b
    if op == "q_dp":
        return a * (E.dec("1.00") - b)
    if op == "q_charge":
        return a * (E.dec("1.00") - b) * (E.dec("1.00") + c)
    return {"add": a + b, "sub": a - b, "mul": a * b, "div": a / b, "mod": a % b, "lt": a.lt(b), "le": a.le(b),
            "gt": a.gt(b), "ge": a.ge(b), "eq": a.eq(b), "ne": a.ne(b)}[op]


def out_bytes_for(op: str, types):
    cols = [E.ColType(p, s) for p, s in types]
    b = E.build([expr_for(op)], cols)
    E.derive_types(b)
    nd = b.nodes[b.roots[0]]
    if op in ("lt", "le", "gt", "ge", "eq", "ne"):
        return 1
    return codec.compact_bytes(nd.precision)


def cases():
    out = []
    for (pa, sa), (pb, sb) in OP_PAIRS:
        for op in OPS:
            if op == "div" and sb + 4 > 38:
                continue
            out.append({"name": f"{op}_{pa}_{sa}_{pb}_{sb}", "op": op, "types": [[pa, sa], [pb, sb]],
                        "rows": 64, "dist": "edge"})
    for p in (18, 38, 76, 150):
        s = p // 4
        out.append({"name": f"sweep_mad_{p}", "op": "mad", "types": [[p, s]] * 3, "rows": 256, "dist": "digits"})
        if s + 4 <= 38:
            out.append({"name": f"sweep_div_{p}", "op": "div", "types": [[p, s]] * 2, "rows": 256,
                        "dist": "digits"})
    for op in ("q_dp", "q_charge"):
        out.append({"name": f"query_{op}", "op": op, "types": [[15, 2]] * 3, "rows": 256, "dist": "query"})
    return out


def gen_inputs(case, rng):
    types = case["types"]
    n = case["rows"]
    if case["dist"] == "edge":
        vals = [edge_values(p, rng, n) for p, _ in types]
        if case["op"] == "mod":
            # the reference's ModCalc has no zero-divisor check (its top-limb
            # scan underflows, AriesDecimal.hxx:970-973): never give it one
            vals[1] = [(s, m) if m else (s, 1) for s, m in vals[1]]
        return vals
    if case["dist"] == "digits":
        return [digits_values(p, rng, n, nonzero=(case["op"] == "div" and k == 1)) for k, (p, _) in enumerate(types)]
    price = [(0, rng.randint(90000, 10494950)) for _ in range(n)]
    disc = [(0, rng.randint(0, 10)) for _ in range(n)]
    tax = [(0, rng.randint(0, 8)) for _ in range(n)]
    return [price, disc, tax]


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "reference_vectors.json"))
    a = ap.parse_args()
    rng = random.Random(20261203)
    result = {"generator": "tests/golden/make_golden.py (reference AriesDecimal<LEN> via oracle/_ref/libariesref.so)",
              "cases": []}
    for case in cases():
        vals = gen_inputs(case, rng)
        raws = [codec.encode(v, p) for v, (p, _) in zip(vals, case["types"])]
        devs = [torch.frombuffer(bytearray(r), dtype=torch.uint8).cuda() for r in raws]
        ob = out_bytes_for(case["op"], case["types"])
        out = torch.zeros(case["rows"] * ob, dtype=torch.uint8, device="cuda")
        t = case["types"]
        c_dev = devs[2].data_ptr() if len(devs) > 2 else None
        pc, sc = (t[2] if len(t) > 2 else (0, 0))
        L = refharness.run(case["op"], devs[0].data_ptr(), t[0][0], t[0][1], devs[1].data_ptr(), t[1][0], t[1][1],
                           case["rows"], out.data_ptr(), ob, c_dev=c_dev, pc=pc, sc=sc, b_host=raws[1])
        torch.cuda.synchronize()
        rec = dict(case)
        rec.update({"len": L, "out_bytes": ob, "inputs": [r.hex() for r in raws],
                    "output": bytes(out.cpu().numpy().tobytes()).hex()})
        result["cases"].append(rec)
        print(case["name"], "LEN", L, "rows", case["rows"])
    with open(a.out, "w") as f:
        json.dump(result, f, indent=0)
    print("wrote", a.out, len(result["cases"]), "cases")


if __name__ == "__main__":
    main()
