"""The N>1 path of bench.py on CPU: two ranks over gloo.  Every rank times its
own share, the job's time is the maximum over ranks, ranks meet at barriers,
and in the reference arm rank 0 alone measures and prints while the other
ranks exit without work."""
import os
import socket
import sys
import types

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        mx = bench.max_over_ranks(10.0 * (rank + 1), world)
        args = types.SimpleNamespace(workload="sweep", steps=1, warmup=0, cpu_seconds=0.2, ref_seconds=0.5)
        ref = bench.run_reference(args, rank, world)
        bench.barrier(world)
        out[rank] = (mx, ref is None, None if ref is None else (ref["impl"], ref["n_gpus"], ref["unit"]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0          # the maximum over ranks, on every rank
    assert res[0][1] is False and res[0][2] == ("reference", 2, "rows/s")
    assert res[1][1] is True                        # the other rank does no reference work
