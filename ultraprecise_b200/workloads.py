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
