"""GPU parity of the expression kernels against the CPU oracle (byte-exact)."""
import random

import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from ultraprecise_b200 import abi, codec, runtime
from ultraprecise_b200 import expr as E
from tests.helpers import edge_values

pytestmark = pytest.mark.gpu


def _check(mod, cols_t, raws, rows, expr_root_built=None, err_expected=None):
    dev = [runtime.DeviceColumn.from_host(r, t.precision, t.scale) for r, t in zip(raws, cols_t)]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = mod.launch(dev, rows, err=err)
    torch.cuda.synchronize()
    got = bytes(out.cpu().numpy().tobytes())
    exp, exp_err = oracle.eval_expr(mod.built, mod.root, raws, rows, mod.value_bytes)
    if got != exp:
        ob = mod.value_bytes
        bad = [i for i in range(rows) if got[i * ob:(i + 1) * ob] != exp[i * ob:(i + 1) * ob]]
        i = bad[0]
        raise AssertionError(f"{len(bad)} rows differ; first row {i}: got {got[i*ob:(i+1)*ob].hex()} "
                             f"exp {exp[i*ob:(i+1)*ob].hex()}")
    assert int(err.item()) == exp_err
    return got


# The precision sweep: element-wise a*b+c and a/b on DECIMAL(p, p/4), every digit
# uniform 0-9, signs +/-, zero divisors redrawn (small row counts here; the
# full sizes run in bench.py)
@pytest.mark.parametrize("p", [18, 38, 76, 150, 300, 600])
@pytest.mark.parametrize("op", ["mad", "div"])
def test_precision_sweep_parity(p, op):
    s = p // 4
    rows = {18: 4099, 38: 4099, 76: 2053, 150: 1031, 300: 517, 600: 263}[p]
    cols = [E.ColType(p, s)] * 3
    a, b, c = E.col(0), E.col(1), E.col(2)
    mod = runtime.compile_expr(a * b + c if op == "mad" else a / b, cols)
    seed = 1000 * p + (1 if op == "mad" else 2)
    raws = [bytes(runtime.gen_digits(rows, p, seed + k, nonzero=(op == "div" and k == 1)).cpu().numpy().tobytes())
            for k in range(3)]
    torch.cuda.synchronize()
    _check(mod, cols, raws, rows)


@pytest.mark.parametrize("p,s", [(15, 2), (18, 4), (9, 9), (38, 9), (20, 0), (65, 30)])
@pytest.mark.parametrize("op", ["add", "sub", "mul", "div", "mod", "lt", "ge", "eq"])
def test_edge_values_parity(p, s, op):
    rng = random.Random(hash((p, s, op)) & 0xFFFFF)
    n = 300
    s2 = max(0, min(p, s + 3))
    cols = [E.ColType(p, s), E.ColType(p, s2)]
    a, b = E.col(0), E.col(1)
    expr = {"add": a + b, "sub": a - b, "mul": a * b, "div": a / b, "mod": a % b, "lt": a.lt(b), "ge": a.ge(b),
            "eq": a.eq(b)}[op]
    mod = runtime.compile_expr(expr, cols)
    raws = [codec.encode(edge_values(p, rng, n), p), codec.encode(edge_values(p, rng, n), p)]
    _check(mod, cols, raws, n)


def test_nested_constants_parity():
    rng = random.Random(3)
    cols = [E.ColType(15, 2)] * 3
    a, b, c = E.col(0), E.col(1), E.col(2)
    exprs = [(a * (E.dec("1.00") - b)) * (E.dec("1.00") + c), (a + b) / (c - E.dec("0.5")),
             -(a - b) * c + E.lit(3), E.rescale(a * b, 20, 1), (a / b) / c, (a * b) % c]
    raws = [codec.encode(edge_values(15, rng, 500), 15) for _ in range(3)]
    for e in exprs:
        _check(runtime.compile_expr(e, cols), cols, raws, 500)


def test_division_by_zero_and_overflow_flags():
    cols = [E.ColType(18, 4), E.ColType(18, 4)]
    a, b = E.col(0), E.col(1)
    mod = runtime.compile_expr(a / b, cols)
    va = [(0, 12345), (1, 10 ** 17), (0, 0), (0, 999)]
    vb = [(0, 0), (0, 1), (1, 0), (0, 3)]
    got = _check(mod, cols, [codec.encode(va, 18), codec.encode(vb, 18)], 4)
    assert len(got) == 4 * mod.value_bytes


def test_empty_and_ragged_rows():
    cols = [E.ColType(15, 2)] * 2
    mod = runtime.compile_expr(E.col(0) * E.col(1), cols)
    for rows in (0, 1, 2, 15, 17, 255, 257, 1000):
        rng = random.Random(rows)
        raws = [codec.encode(edge_values(15, rng, max(rows, 1))[:rows], 15) for _ in range(2)]
        if rows == 0:
            dev = [runtime.DeviceColumn.from_host(b"", 15, 2) for _ in range(2)]
            out = mod.launch(dev, 0)
            assert out.numel() == 0
            continue
        _check(mod, cols, raws, rows)


def test_generic_path_indices_and_unaligned():
    """Row indirection (AriesColumnDataIterator indices) and unaligned bases
    take the generic kernel; results must equal the gathered oracle run."""
    rng = random.Random(9)
    rows = 777
    cols = [E.ColType(38, 9)] * 2
    mod = runtime.compile_expr(E.col(0) * E.col(1) - E.col(0), cols)
    va = edge_values(38, rng, rows)
    vb = edge_values(38, rng, rows)
    perm = list(range(rows))
    rng.shuffle(perm)
    ra, rb = codec.encode(va, 38), codec.encode(vb, 38)
    B = codec.compact_bytes(38)
    da = runtime.DeviceColumn.from_host(ra, 38, 9)
    da.indices = torch.tensor(perm, dtype=torch.int32, device="cuda")
    # unaligned base for b: shift by one byte
    tb = torch.frombuffer(bytearray(b"\x00" + rb), dtype=torch.uint8).cuda()
    db = runtime.DeviceColumn(tb[1:], 38, 9)
    db.indices = da.indices
    out = mod.launch([da, db], rows)
    torch.cuda.synchronize()
    gathered_a = b"".join(ra[i * B:(i + 1) * B] for i in perm)
    gathered_b = b"".join(rb[i * B:(i + 1) * B] for i in perm)
    exp, _ = oracle.eval_expr(mod.built, mod.root, [gathered_a, gathered_b], rows, mod.value_bytes)
    assert bytes(out.cpu().numpy().tobytes()) == exp


def test_module_cache_reuses_kernels():
    lib = abi.load()
    cols = [E.ColType(20, 3)] * 2
    m1 = runtime.compile_expr(E.col(0) + E.col(1), cols)
    n1 = lib.up_module_cache_size(0)
    m2 = runtime.compile_expr(E.col(0) + E.col(1), cols)
    assert lib.up_module_cache_size(0) == n1
    assert m1.source() == m2.source()


@pytest.mark.parametrize("p,op,rows,chunk", [(18, "mad", 100_003, 0), (38, "div", 50_001, 7_000),
                                             (150, "mad", 20_000, 3_001), (600, "mad", 5_000, 999)])
def test_host_launch_matches_device_launch(p, op, rows, chunk):
    """up_expr_launch_host (host columns, chunked and overlapped) gives the
    same bytes and error word as the device launch."""
    from ultraprecise_b200 import workloads
    e, cols = workloads.sweep_expr(p, op)
    m = runtime.compile_expr(e, cols)
    dev = [runtime.gen_digits(rows, p, 300 + k, nonzero=(op == "div" and k == 1)) for k in range(len(cols))]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    want = m.launch([runtime.DeviceColumn(d, p, p // 4) for d in dev], rows, err=err)
    torch.cuda.synchronize()
    host = [d.cpu().pin_memory() if i % 2 == 0 else d.cpu() for i, d in enumerate(dev)]  # pinned and pageable
    out = torch.empty(rows * m.value_bytes, dtype=torch.uint8).pin_memory()
    herr = m.launch_host(host, cols, rows, out, chunk_rows=chunk)
    assert bytes(out.numpy().tobytes()) == bytes(want.cpu().numpy().tobytes())
    assert herr == int(err.item())
