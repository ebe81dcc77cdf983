"""GPU: the bounded-wait path of the bulk-copy pipelines.  Every mbarrier wait
in the kernels gives up after a bounded number of polls and reports
UP_ROWERR_TIMEOUT instead of hanging; here that path is made to run out on
purpose (up_util_wait_timeout_probe: a barrier armed for bytes that no copy
delivers, a short poll limit), the status reaches the host, and the context
stays usable for the next launch."""
import pytest

torch = pytest.importorskip("torch")

from oracle import oracle
from ultraprecise_b200 import abi, codec, runtime
from ultraprecise_b200 import expr as E

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("polls", [1, 1000, 100_000])
def test_wait_runs_out_and_reports_timeout(polls):
    lib = abi.load()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    done = torch.zeros(1, dtype=torch.int32, device="cuda")
    abi.check(lib.up_util_wait_timeout_probe(polls, err.data_ptr(), done.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream), "probe")
    torch.cuda.synchronize()
    assert int(err.item()) & abi.UP_ROWERR_TIMEOUT
    assert int(done.item()) == 1
    # the context is still good: an ordinary launch right after is exact
    p, s, rows = 38, 9, 5000
    m = runtime.compile_expr(E.col(0) * E.col(1) + E.col(2), [E.ColType(p, s)] * 3)
    ins = [runtime.gen_digits(rows, p, 70 + k) for k in range(3)]
    out = m.launch([runtime.DeviceColumn(t, p, s) for t in ins], rows)
    torch.cuda.synchronize()
    exp, _ = oracle.eval_expr(m.built, m.root, [bytes(t.cpu().numpy().tobytes()) for t in ins], rows,
                              m.value_bytes)
    assert bytes(out.cpu().numpy().tobytes()) == exp


def test_probe_refuses_unbounded_polls():
    lib = abi.load()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.up_util_wait_timeout_probe(0, err.data_ptr(), err.data_ptr(), None) == abi.UP_ERR_INVALID_ARG
    assert lib.up_util_wait_timeout_probe((1 << 24) + 1, err.data_ptr(), err.data_ptr(),
                                          None) == abi.UP_ERR_INVALID_ARG
