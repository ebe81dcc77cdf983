"""CPU: the C-ABI library loads without a GPU, exports every symbol the
public headers declare, types expressions like the reference, and every
benchmark kernel compiles for sm_100a with NVRTC."""
import ctypes as C
import os
import re

import pytest

from ultraprecise_b200 import abi, abi_ext, workloads
from ultraprecise_b200 import expr as E

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(up_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = abi.load()
    declared = declared_symbols()
    assert len(declared) > 20
    for name in sorted(declared):
        assert hasattr(lib, name), f"{name} not exported"
        assert name in abi.SIGNATURES or name in abi_ext.SIGNATURES, f"{name} has no ctypes prototype"


def test_status_strings_and_tables():
    lib = abi.load()
    assert lib.up_abi_version() == 1
    assert lib.up_status_string(abi.UP_ERR_COMPILE) == b"compile error"
    assert lib.up_compact_bytes(0) == -1
    assert lib.up_compact_bytes(15) == 7 and lib.up_compact_bytes(299) == 125
    assert lib.up_precision_words(19) == 3  # the reference's table, not the tight value (2)


def _types(root, cols):
    b = E.build([root], cols)
    E.derive_types(b)
    return E.node_type(b, b.roots[0])


def test_reference_typing_rules():
    c15 = [E.ColType(15, 2)] * 4
    qty, price, disc, tax = [E.col(i) for i in range(4)]
    # price*(1-disc) -> (31,4); *(1+tax) -> (47,6)  (AriesEngineShell.cpp:90-144)
    one = E.dec("1.00", precision=0)
    assert _types(price * (one - disc), c15) == (31, 4)
    assert _types(price * (one - disc) * (one + tax), c15) == (47, 6)
    for p in (18, 38, 76, 150):
        s = p // 4
        cols = [E.ColType(p, s)] * 3
        a, b, c = E.col(0), E.col(1), E.col(2)
        assert _types(c + a * b, cols) == (2 * p + 1, 2 * s)
        assert _types(a / b, cols) == (s + 5, s + 4)
    # MOD: p = p2, s = 0
    assert _types(E.col(0) % E.col(1), [E.ColType(20, 3), E.ColType(12, 5)]) == (12, 0)


def test_invalid_trees_are_rejected():
    lib = abi.load()
    b = E.build([E.col(0) + E.col(1)], [E.ColType(15, 2)] * 2)
    st = lib.up_expr_derive_types(b.nodes, b.n_nodes, b.roots[0], b.col_types, 1)  # column 1 untyped
    assert st == abi.UP_ERR_INVALID_ARG


@pytest.mark.parametrize("p", [18, 38, 76])
def test_sweep_kernels_compile_for_sm100a(p):
    lib = abi.load()
    for op in workloads.SWEEP_OPS:
        e, cols = workloads.sweep_expr(p, op)
        b = E.build([e], cols)
        E.derive_types(b)
        st = lib.up_util_compile_only(b.nodes, b.n_nodes, b.roots[0], b.col_types, b.n_cols, 0, None, 0)
        assert st == abi.UP_OK, lib.up_last_error_message()


def test_query_kernel_compiles_for_sm100a():
    lib = abi.load()
    exprs, aggs, cols = workloads.query_exprs()
    b = E.build(exprs, cols)
    E.derive_types(b)
    qa = (abi.UpQueryAgg * len(aggs))()
    for i, (k, r) in enumerate(aggs):
        qa[i].kind = k
        qa[i].root = b.roots[r]
    assert lib.up_util_compile_only(b.nodes, b.n_nodes, 0, b.col_types, b.n_cols, 1, qa, len(aggs)) == abi.UP_OK


def test_launch_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = abi.load()
    info = abi.UpDeviceInfo()
    assert lib.up_device_query(0, C.byref(info)) != abi.UP_OK


def test_automatic_choice_of_cooperative_path():
    """The widest a*b+c sweep expression gets the cooperative kernel (16
    threads per value), narrower ones and divisions one thread per value;
    threads_per_value overrides the choice."""
    from ultraprecise_b200 import prewarm, workloads
    for p, op, coop in ((150, "mad", False), (300, "mad", False), (600, "mad", True), (600, "div", False)):
        e, cols = workloads.sweep_expr(p, op)
        src = prewarm.expr_source(e, cols)
        assert ("up_trow" in src) == coop, (p, op)
    e, cols = workloads.sweep_expr(600, "mad")
    assert "tpi_mul<16, 8" in prewarm.expr_source(e, cols)
    assert "up_trow" not in prewarm.expr_source(e, cols, threads_per_value=1)
    assert "tpi_div_round<8," in prewarm.expr_source(*workloads.sweep_expr(150, "div"), threads_per_value=8)
