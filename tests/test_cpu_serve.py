"""Host-side pieces of the serving loop: the open-loop arrival schedule, the
request mix, the percentile rule, and that a session fails loudly without a
GPU."""
import ctypes as C
import statistics

import pytest

from ultraprecise_b200 import abi, serve, workloads


def test_poisson_arrivals_rate_and_order():
    t = workloads.poisson_arrivals(500.0, 4.0, seed=3)
    assert t == sorted(t) and all(0 <= x < 4000.0 for x in t)
    assert 1800 < len(t) < 2200
    gaps = [b - a for a, b in zip(t, t[1:])]
    assert abs(statistics.mean(gaps) - 2.0) < 0.2  # 1/rate in ms


def test_request_mix():
    k = workloads.serve_kinds(20000, seed=1)
    frac = [k.count(i) / len(k) for i in range(4)]
    for f, w in zip(frac, workloads.SERVE_MIX):
        assert abs(f - w) < 0.02


def test_percentile_rule():
    v = list(range(1, 101))
    assert serve.percentiles(v) == (51, 95, 99)
    assert serve.percentiles([]) == (0.0, 0.0, 0.0)


def test_session_without_device_fails_loudly():
    lib = abi.load()
    h = C.c_void_p()
    st = lib.up_serve_create(None, C.byref(h))
    assert st == abi.UP_ERR_NO_DEVICE
    assert not h.value
