"""GPU parity of the sin(x) series workload (DECIMAL(p, p-2), 20 Horner terms
with RESCALE truncation) against the oracle, byte for byte."""
import random

import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from ultraprecise_b200 import codec, runtime, workloads
from ultraprecise_b200 import expr as E

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p,rows", [(100, 20_000), (300, 6_000), (1000, 2_048)])
def test_sin_matches_oracle(p, rows):
    s = p - 2
    pi = workloads.pi_scaled(s)
    raw = workloads.sin_inputs(p, rows, seed=p)
    edges = codec.encode([(0, 0), (1, 0), (0, pi), (1, pi), (0, 1), (1, 1), (0, 10 ** s)], p)
    raw = edges + raw[len(edges):]
    e, cols = workloads.sin_expr(p)
    m = runtime.compile_expr(e, cols)
    dev = runtime.DeviceColumn.from_host(raw, p, s)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = m.launch([dev], rows, err=err)
    torch.cuda.synchronize()
    b = E.build([e], cols)
    E.derive_types(b)
    exp, exp_err = oracle.eval_expr(b, b.roots[0], [raw], rows, codec.compact_bytes(p), threads=8)
    assert bytes(out.cpu().numpy().tobytes()) == exp
    assert int(err.item()) == exp_err == 0
