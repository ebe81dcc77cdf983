"""The benchmark workloads (expression shapes and sizes), shared by bench.py,
the tests and the build-time JIT prewarm.

Seeded synthetic inputs stand in for the reference's experiment data (TPC-H
lineitem and the paper's generated columns, not shipped with the reference).
"""
from __future__ import annotations

from . import abi
from . import expr as E

# precision sweep: (p, rows); s = p // 4; a*b+c and a/b
SWEEP = [(18, 16 << 20), (38, 16 << 20), (76, 8 << 20), (150, 4 << 20), (300, 2 << 20), (600, 1 << 20)]
SWEEP_OPS = ("mad", "div")


def sweep_expr(p: int, op: str):
    s = p // 4
    n = 3 if op == "mad" else 2
    cols = [E.ColType(p, s)] * n
    a, b = E.col(0), E.col(1)
    return (a * b + E.col(2) if op == "mad" else a / b), cols


# grouped-aggregate query: qty, price, disc, tax DECIMAL(15,2); keys l_returnflag, l_linestatus
QUERY_KEYS = [(b"A", b"F", 0.25), (b"N", b"F", 0.007), (b"N", b"O", 0.493), (b"R", b"F", 0.25)]
QUERY_RANGES = {"qty": (100, 5000, 100), "price": (90000, 10494950, 1), "disc": (0, 10, 1), "tax": (0, 8, 1)}


def query_exprs():
    """SUM(qty), SUM(price), SUM(price*(1-disc)), SUM(price*(1-disc)*(1+tax)),
    AVG(qty), AVG(price), AVG(disc), COUNT(*)."""
    cols = [E.ColType(15, 2)] * 4
    qty, price, disc, tax = [E.col(i) for i in range(4)]
    disc_price = price * (E.dec("1.00") - disc)
    charge = disc_price * (E.dec("1.00") + tax)
    exprs = [qty, price, disc_price, charge, disc]
    aggs = [(abi.UP_AGG_SUM, 0), (abi.UP_AGG_SUM, 1), (abi.UP_AGG_SUM, 2), (abi.UP_AGG_SUM, 3),
            (abi.UP_AGG_AVG, 0), (abi.UP_AGG_AVG, 1), (abi.UP_AGG_AVG, 4), (abi.UP_AGG_COUNT, 0)]
    return exprs, aggs, cols


# Batched mixed precision: 64 tasks, random trees of depth 3-5 over +,-,*,/ on
# 2-4 columns; p log-uniform in [10,400], s uniform in [0,p/2], rows
# log-uniform in [1e3,1e7]; half the tasks end in a grouped SUM over Zipf(1.1)
# int32 keys with 1..100k groups.  Every node of this path is exact (never
# truncated), so trees whose intermediates would exceed 4096 bits are redrawn.
BATCH_MAX_BITS = 4096


def _bits_bound(e, s: int, nbytes: int):
    """(bits, scale) bound of an expression over DECIMAL(p,s) columns, the
    same bound the library's node analysis computes."""
    if e.kind == abi.UP_NODE_COLUMN:
        return 8 * nbytes - 1, s
    a_bits, a_s = _bits_bound(e.left, s, nbytes)
    b_bits, b_s = _bits_bound(e.right, s, nbytes)
    if e.kind in (abi.UP_NODE_ADD, abi.UP_NODE_SUB):
        sc = max(a_s, b_s)
        ab = a_bits + ((10 ** (sc - a_s)).bit_length() if sc > a_s else 0)
        bb = b_bits + ((10 ** (sc - b_s)).bit_length() if sc > b_s else 0)
        return max(ab, bb) + 1, sc
    if e.kind == abi.UP_NODE_MUL:
        return a_bits + b_bits, a_s + b_s
    return max(64, a_bits + (10 ** (b_s + 4)).bit_length()), a_s + 4


def batch_tasks(seed: int = 20261203, n: int = 64, max_bits: int = BATCH_MAX_BITS, row_scale: float = 1.0):
    """Deterministic task list: dicts with expr, cols, p, s, rows, agg, groups."""
    import math
    import random
    from . import codec
    rng = random.Random(seed)
    ops = [abi.UP_NODE_ADD, abi.UP_NODE_SUB, abi.UP_NODE_MUL, abi.UP_NODE_DIV]
    out = []
    redraws = 0
    while len(out) < n:
        p = int(round(math.exp(rng.uniform(math.log(10), math.log(400)))))
        s = rng.randint(0, p // 2)
        rows = max(1, int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e7))) * row_scale)))
        ncols = rng.randint(2, 4)
        depth = rng.randint(3, 5)

        def tree(d, must):
            if d == 0 or (not must and rng.random() < 0.35):
                return E.col(rng.randrange(ncols))
            op = rng.choice(ops)
            deep = rng.randrange(2)
            return E.Expr(op, tree(d - 1, must and deep == 0), tree(d - 1, must and deep == 1))

        e = tree(depth, True)
        bits, _ = _bits_bound(e, s, codec.compact_bytes(p))
        if bits > max_bits:
            redraws += 1
            continue
        agg = abi.UP_AGG_SUM if len(out) % 2 == 0 else -1
        groups = max(1, int(round(math.exp(rng.uniform(0, math.log(1e5)))))) if agg >= 0 else 0
        out.append({"expr": e, "cols": [E.ColType(p, s)] * ncols, "p": p, "s": s, "rows": rows, "agg": agg,
                    "groups": groups, "ncols": ncols, "depth": depth})
    return out, redraws


def batch_specs(tasks):
    """TaskSpecs of batch_tasks() output."""
    from .batch import TaskSpec
    return [TaskSpec(t["expr"], t["cols"], t["agg"]) for t in tasks]


def batch_group_ids(rows: int, groups: int, seed: int):
    """int32 group ids in [0, groups) drawn from Zipf(1.1) over the group ranks
    (id 0 is the most frequent), as a numpy array."""
    import numpy as np
    rng = np.random.default_rng(seed)
    w = np.arange(1, groups + 1, dtype=np.float64) ** -1.1
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    ids = np.searchsorted(cdf, rng.random(rows), side="right")
    return np.minimum(ids, groups - 1).astype(np.int32)


def batch_columns(tasks, seed: int, row_cap: int | None = None):
    """Device columns and host group ids for batch_tasks() output: per task,
    its columns (every digit uniform, sign +/-, nonzero values so that leaf
    divisors are never zero) and, for SUM tasks, Zipf int32 keys.  Returns a
    list of (rows, [column tensors], group ids numpy array or None)."""
    from . import runtime
    out = []
    for k, t in enumerate(tasks):
        rows = t["rows"] if row_cap is None else min(t["rows"], row_cap)
        cols = [runtime.gen_digits(rows, t["p"], seed + 1000 * k + c, signed=True, nonzero=True)
                for c in range(t["ncols"])]
        gid = batch_group_ids(rows, t["groups"], seed + 1000 * k + 999) if t["agg"] >= 0 else None
        out.append((rows, cols, gid))
    return out


def _limbs(bits: int) -> int:
    return max(1, (bits + 31) // 32)


def expr_madds(e, s: int, nbytes: int):
    """(limb multiply-adds per row, bits, scale) of an expression over
    DECIMAL(p,s) columns of nbytes each: a*b costs La*Lb, aligning an operand
    by 10^d costs L*L(10^d), a/b costs the dividend scale-up plus the
    (m-n+1)*n long-division steps."""
    if e.kind == abi.UP_NODE_COLUMN:
        return 0, 8 * nbytes - 1, s
    am, ab, asc = expr_madds(e.left, s, nbytes)
    bm, bb, bsc = expr_madds(e.right, s, nbytes)
    m = am + bm
    if e.kind in (abi.UP_NODE_ADD, abi.UP_NODE_SUB):
        sc = max(asc, bsc)
        if sc > asc:
            m += _limbs(ab) * _limbs((10 ** (sc - asc)).bit_length())
        if sc > bsc:
            m += _limbs(bb) * _limbs((10 ** (sc - bsc)).bit_length())
    elif e.kind == abi.UP_NODE_MUL:
        m += _limbs(ab) * _limbs(bb)
    else:
        lp = _limbs((10 ** (bsc + 4)).bit_length())
        la, lb = _limbs(ab), _limbs(bb)
        m += la * lp + max(1, la + lp - lb + 1) * lb
    bits, sc = _bits_bound(e, s, nbytes)
    return m, bits, sc


# sin(x) series: 20 terms in Horner form on DECIMAL(p, p-2), x uniform in
# [-pi, pi] at full scale.  t_20 = 1; t_k = 1 - trunc(y * t_(k+1)) / (2k(2k+1))
# for k = 19..1 with y = trunc(x*x); sin x = trunc(x * t_1).  Every product and
# quotient is truncated toward zero to scale p-2 (RESCALE); the divisions by the
# exact integers 2k(2k+1) (ratios of consecutive factorials) follow the
# reference's divide rule (scale +4, half-up) before that truncation.
SIN = [(100, 1 << 20), (300, 1 << 19), (1000, 1 << 18)]
SIN_TERMS = 20


def sin_expr(p: int, terms: int = SIN_TERMS):
    s = p - 2
    x = E.col(0)
    y = E.rescale(x * x, p, s)
    t = E.dec(10 ** s, scale=s, precision=p)   # 1 at scale p-2
    one = t
    for k in range(terms - 1, 0, -1):
        m = E.rescale(y * t, p, s)
        d = E.rescale(m / E.lit(2 * k * (2 * k + 1)), p, s)
        t = E.rescale(one - d, p, s)
    return E.rescale(x * t, p, s), [E.ColType(p, s)]


def pi_scaled(s: int) -> int:
    """floor(pi * 10^s) by Machin's formula in integer arithmetic."""
    guard = 10
    unity = 10 ** (s + guard)

    def arctan_inv(n: int) -> int:
        total, term, k, sign = 0, unity // n, 1, 1
        n2 = n * n
        while term:
            total += sign * (term // k)
            term //= n2
            k += 2
            sign = -sign
        return total

    return (4 * (4 * arctan_inv(5) - arctan_inv(239))) // 10 ** guard


def sin_inputs(p: int, rows: int, seed: int) -> bytes:
    """Compact DECIMAL(p, p-2) column of x uniform over [-pi, pi] at full
    scale: magnitude floor(U * floor(pi * 10^(p-2))) with U uniform on [0,1)
    drawn to 64 bits beyond the magnitude's width, sign +/- with equal odds."""
    import random
    from . import codec
    rng = random.Random(seed)
    pi = pi_scaled(p - 2)
    nb = pi.bit_length() + 64
    vals = [(rng.getrandbits(1), (rng.getrandbits(nb) * pi) >> nb) for _ in range(rows)]
    return codec.encode(vals, p)


def sin_python(sign: int, mag: int, p: int, terms: int = SIN_TERMS):
    """The same series in exact Python integers with the decimal path's rules
    (sign-magnitude values; products and quotients truncated toward zero to
    scale p-2; division by the integer 2k(2k+1) at scale +4 rounded half up on
    the magnitude, then truncated): an independent restatement that checks the
    oracle.  Returns (sign, magnitude) with the sign of zero as computed."""
    s = p - 2
    S = 10 ** s

    def mul_trunc(a, b):  # (sign, mag) * (sign, mag), truncated to scale s
        return (a[0] ^ b[0], (a[1] * b[1]) // S)

    def sub(a, b):  # a - b in sign-magnitude (equal magnitudes give +0)
        av = -a[1] if a[0] else a[1]
        bv = -b[1] if b[0] else b[1]
        v = av - bv
        return (1 if v < 0 else 0, abs(v))

    x = (sign, mag)
    y = mul_trunc(x, x)
    one = (0, S)
    t = one
    for k in range(terms - 1, 0, -1):
        m = mul_trunc(y, t)
        D = 2 * k * (2 * k + 1)
        if m[1] == 0:
            d = (0, 0)  # dividend 0 gives +0
        else:
            q, r = divmod(m[1] * 10 ** 4, D)
            q += 1 if 2 * r >= D else 0
            d = (m[0], q // 10 ** 4)
        t = sub(one, d)
    return mul_trunc(x, t)


# Served stream: open-loop Poisson arrivals; each query is drawn 40/30/20/10
# from the grouped query, the precision-sweep expressions, the batched-set
# tasks and the sin series, all at 1/10 of their row counts, over columns
# kept resident in HBM.
SERVE_RATES = (100, 500, 2000, 5000)
SERVE_MIX = (0.4, 0.3, 0.2, 0.1)


def poisson_arrivals(rate: float, seconds: float, seed: int):
    """Arrival times in ms of an open-loop Poisson stream (exponential gaps)."""
    import random
    rng = random.Random(seed)
    t, out = 0.0, []
    while True:
        t += rng.expovariate(rate) * 1000.0
        if t >= seconds * 1000.0:
            return out
        out.append(t)


def serve_kinds(n: int, seed: int, mix=SERVE_MIX):
    """Request kind (0 query, 1 sweep, 2 batch task, 3 sin) per arrival."""
    import random
    rng = random.Random(seed)
    return [rng.choices(range(len(mix)), weights=mix)[0] for _ in range(n)]


# Cooperative-evaluation parity cases (the GPU tests run them; the prewarm
# compiles them): (name, p, expression, column types, threads per value).
def coop_cases():
    a, b, c = E.col(0), E.col(1), E.col(2)
    out = []
    for p in (76, 150, 600):
        s = p // 4
        types = [E.ColType(p, s)] * 3
        exprs = {"mad": a * b + c, "msub": a - b * c, "addsub": (a + b) - (c - a),
                 "const": a * E.dec("-12345678901234567890.123") + E.lit(7) * b}
        for name, e in exprs.items():
            for tpv in (0, 2, 8, 32):
                out.append((name, p, e, types, tpv))
    for p in (38, 150, 300):
        s = p // 4
        types = [E.ColType(p, s)] * 3
        exprs = {"div": a / b, "mod": a % b, "divmix": (a * c) / b + a,
                 "trunc": E.rescale(a * b, 2 * p + 1, s)}
        for name, e in exprs.items():
            for tpv in (4, 8, 32):
                out.append((name, p, e, types, tpv))
    for p, tpv in ((100, 8), (300, 16)):
        e, types = sin_expr(p)
        out.append(("sin", p, e, types, tpv))
    return out


# Cost-model data: launches measured on the device to train the model
# (COSTMODEL_TRAIN) and held-out shapes it has never seen on which its choice
# of threads per value is compared with the width rule (COSTMODEL_EVAL).
# Columns are DECIMAL(p, p/4) with every digit uniform; rows 64K..1M.
COSTMODEL_TRAIN_P = (40, 80, 150, 300, 600)
COSTMODEL_EVAL_P = (60, 110, 220, 450)
COSTMODEL_ROWS = (1 << 16, 1 << 18, 1 << 20)


def _cm_cols(p: int, n: int):
    return [E.ColType(p, p // 4)] * n


def costmodel_train_shapes():
    """(name, expression, column types) of the training launches."""
    a, b, c = E.col(0), E.col(1), E.col(2)
    out = []
    for p in COSTMODEL_TRAIN_P:
        for name, e, n in (("mad", a * b + c, 3), ("mul", a * b, 2), ("div", a / b, 2),
                           ("sq", (a + b) * (a - b), 2), ("mix", a * b - c * a, 3),
                           ("addmul", (a + b) * c, 3), ("divmul", a / b * c, 3), ("twodiv", a / b + c / a, 3)):
            out.append((f"{name} p={p}", e, _cm_cols(p, n)))
    return out


def batch_pinned_tpv(tasks, sizes):
    """Threads per value pinned on the wide projection tasks (p > 120) of a
    batch, cycling through `sizes`; 1 elsewhere (the GPU test of cooperative
    band tasks and its prewarm share it)."""
    out, i = [], 0
    for t in tasks:
        if t["agg"] < 0 and t["p"] > 120:
            out.append(sizes[i % len(sizes)])
            i += 1
        else:
            out.append(1)
    return out


def costmodel_eval_shapes():
    """Held-out shapes: other precisions and other expressions."""
    a, b, c = E.col(0), E.col(1), E.col(2)
    out = []
    for p in COSTMODEL_EVAL_P:
        for name, e, n in (("abc", a * b * c, 3), ("msum", a * b + c * b, 3), ("dmix", (a - b) / c + a, 3)):
            out.append((f"{name} p={p}", e, _cm_cols(p, n)))
    return out
