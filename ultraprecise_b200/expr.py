"""Expression builder: Python objects -> up_expr_node arrays for the C ABI.

Mirrors the reference's typed expression trees (AriesCommonExpr with CALC,
COLUMN_ID, INTEGER and DECIMAL nodes; AriesCommonExpr.h) closely enough that a
tree built here feeds both the CUDA path and the CPU oracle unchanged.
Nodes may be shared (a DAG); each shared node is evaluated once per row.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

from . import abi


@dataclass(eq=False)
class Expr:
    kind: int
    left: "Expr | None" = None
    right: "Expr | None" = None
    column: int = 0
    precision: int = 0
    scale: int = 0
    reverse: bool = False
    const_sign: int = 0
    const_mag: int = 0
    int_value: int = 0

    # arithmetic -----------------------------------------------------
    def _bin(self, kind, other):
        return Expr(kind, self, _wrap(other))

    def __add__(self, o):
        return self._bin(abi.UP_NODE_ADD, o)

    def __radd__(self, o):
        return _wrap(o)._bin(abi.UP_NODE_ADD, self)

    def __sub__(self, o):
        return self._bin(abi.UP_NODE_SUB, o)

    def __rsub__(self, o):
        return _wrap(o)._bin(abi.UP_NODE_SUB, self)

    def __mul__(self, o):
        return self._bin(abi.UP_NODE_MUL, o)

    def __rmul__(self, o):
        return _wrap(o)._bin(abi.UP_NODE_MUL, self)

    def __truediv__(self, o):
        return self._bin(abi.UP_NODE_DIV, o)

    def __rtruediv__(self, o):
        return _wrap(o)._bin(abi.UP_NODE_DIV, self)

    def __mod__(self, o):
        return self._bin(abi.UP_NODE_MOD, o)

    def __neg__(self):
        e = Expr(self.kind, self.left, self.right, self.column, self.precision, self.scale, not self.reverse,
                 self.const_sign, self.const_mag, self.int_value)
        return e

    # comparisons (named, so Python equality keeps its meaning) -------
    def lt(self, o):
        return self._bin(abi.UP_NODE_LT, o)

    def le(self, o):
        return self._bin(abi.UP_NODE_LE, o)

    def gt(self, o):
        return self._bin(abi.UP_NODE_GT, o)

    def ge(self, o):
        return self._bin(abi.UP_NODE_GE, o)

    def eq(self, o):
        return self._bin(abi.UP_NODE_EQ, o)

    def ne(self, o):
        return self._bin(abi.UP_NODE_NE, o)

    # boolean connectives over comparisons -----------------------------
    def and_(self, o):
        return self._bin(abi.UP_NODE_AND, o)

    def or_(self, o):
        return self._bin(abi.UP_NODE_OR, o)


def _wrap(o) -> Expr:
    if isinstance(o, Expr):
        return o
    if isinstance(o, int):
        return lit(o)
    if isinstance(o, str):
        return dec(o)
    raise TypeError(f"cannot use {type(o).__name__} in a decimal expression")


def col(index: int) -> Expr:
    """Input column `index` (its precision/scale come from the column types)."""
    return Expr(abi.UP_NODE_COLUMN, column=index)


def lit(value: int) -> Expr:
    """Integer literal (the reference's INTEGER node)."""
    return Expr(abi.UP_NODE_INT, int_value=int(value))


def dec(text: str | int, scale: int | None = None, precision: int = 0) -> Expr:
    """Decimal constant.  dec("1.25") has scale 2; dec(125, scale=2) too."""
    if isinstance(text, int):
        mag = abs(text)
        sign = 1 if text < 0 else 0
        sc = scale or 0
    else:
        t = text.strip()
        sign = 1 if t.startswith("-") else 0
        t = t.lstrip("+-")
        if "." in t:
            ip, fp = t.split(".", 1)
        else:
            ip, fp = t, ""
        sc = len(fp) if scale is None else scale
        if scale is not None and scale < len(fp):
            raise ValueError("scale smaller than the literal's fraction digits")
        fp = fp.ljust(sc, "0")
        mag = int((ip or "0") + fp)
    if precision <= 0:
        precision = max(len(str(mag)), sc, 1)
    return Expr(abi.UP_NODE_CONST, precision=precision, scale=sc, const_sign=sign, const_mag=mag)


def rescale(e: Expr, precision: int, scale: int) -> Expr:
    """Change scale by truncation toward zero (extension node)."""
    return Expr(abi.UP_NODE_RESCALE, e, precision=precision, scale=scale)


@dataclass
class ColType:
    precision: int
    scale: int
    nullable: bool = False


@dataclass
class Built:
    nodes: C.Array
    n_nodes: int
    roots: list[int]
    col_types: C.Array
    n_cols: int
    exprs: list[Expr] = field(default_factory=list)


def _limbs(mag: int) -> list[int]:
    out = []
    while mag:
        out.append(mag & 0xFFFFFFFF)
        mag >>= 32
    return out


def build(roots: Sequence[Expr], cols: Sequence[ColType]) -> Built:
    """Flatten expression roots into a node array (post-order, shared nodes once)."""
    order: list[Expr] = []
    index: dict[int, int] = {}

    def visit(e: Expr):
        stack = [(e, False)]
        while stack:
            x, done = stack.pop()
            if id(x) in index:
                continue
            if done:
                index[id(x)] = len(order)
                order.append(x)
                continue
            stack.append((x, True))
            if x.right is not None:
                stack.append((x.right, False))
            if x.left is not None:
                stack.append((x.left, False))

    for r in roots:
        visit(r)
    arr = (abi.UpExprNode * len(order))()
    for i, x in enumerate(order):
        nd = arr[i]
        nd.kind = x.kind
        nd.left = index[id(x.left)] if x.left is not None else -1
        nd.right = index[id(x.right)] if x.right is not None else -1
        nd.column = x.column
        nd.precision = x.precision
        nd.scale = x.scale
        nd.reverse = 1 if x.reverse else 0
        nd.const_sign = x.const_sign
        nd.int_value = x.int_value
        if x.kind == abi.UP_NODE_CONST:
            limbs = _limbs(x.const_mag)
            if len(limbs) > abi.UP_CONST_MAX_LIMBS:
                raise ValueError("constant too wide")
            nd.const_nlimbs = len(limbs)
            for k, w in enumerate(limbs):
                nd.const_limbs[k] = w
        if x.kind == abi.UP_NODE_COLUMN:
            if x.column >= len(cols):
                raise ValueError(f"column {x.column} has no type")
            nd.precision = cols[x.column].precision
            nd.scale = cols[x.column].scale
    ct = (abi.UpColType * max(1, len(cols)))()
    for i, c in enumerate(cols):
        ct[i].precision = c.precision
        ct[i].scale = c.scale
        ct[i].nullable = 1 if c.nullable else 0
    return Built(arr, len(order), [index[id(r)] for r in roots], ct, len(cols), order)


def derive_types(b: Built, root: int | None = None) -> Built:
    """Run the reference typing rules over every root (in place)."""
    lib = abi.load()
    for r in ([root] if root is not None else b.roots):
        abi.check(lib.up_expr_derive_types(b.nodes, b.n_nodes, r, b.col_types, b.n_cols), "up_expr_derive_types")
    return b


def node_type(b: Built, k: int) -> tuple[int, int]:
    return b.nodes[k].precision, b.nodes[k].scale


def align_optimize(b: Built, root: int | None = None, cap: int = 4096) -> Built:
    """The reference's AlignOptimize rewrite (AriesEngineShell.cpp:244-685)
    on one root; returns a new Built whose single root is the rewritten tree."""
    lib = abi.load()
    r = b.roots[0] if root is None else root
    out = (abi.UpExprNode * cap)()
    n = C.c_int32()
    nr = C.c_int32()
    abi.check(lib.up_expr_align_optimize(b.nodes, b.n_nodes, r, b.col_types, b.n_cols, out, cap, C.byref(n),
                                         C.byref(nr)), "up_expr_align_optimize")
    arr = (abi.UpExprNode * max(1, n.value))()
    C.memmove(arr, out, C.sizeof(abi.UpExprNode) * n.value)
    return Built(arr, n.value, [nr.value], b.col_types, b.n_cols, [])
