"""Benchmark of the exact-decimal path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload sweep|batch|query]

Workload "sweep" (default) is the precision sweep: element-wise a*b+c and a/b
(scale s+4, half-up) on DECIMAL(p, p/4), p in {18,38,76,150,300,600}, every
digit uniform 0-9, signs +/-, zero divisors redrawn, 16M rows for p<=38,
halved per doubling of p.  One step = one pass over all twelve
(p, expression) launches; inputs are resident in HBM and every case's input
is larger than L2 (126 MB), so no L2 flush is needed between steps.

Workload "batch" is the batched mixed-precision set: 64 seeded tasks (random
+,-,*,/ trees of depth 3-5 on 2-4 DECIMAL(p,s) columns, p log-uniform in
[10,400], rows log-uniform in [1e3,1e7], half ending in a grouped SUM over
Zipf(1.1) keys) run as one captured graph of persistent band kernels, beside
the same 64 tasks launched one by one through the plain per-task path.  A
step is one pass over all 64 tasks; inputs total about 7.5 GB, larger than L2.

The reference arm (--impl reference) times the CPU restatement of the
reference's decimal path (oracle/, the reference has no CPU decimal path of
its own) on the host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from ultraprecise_b200.workloads import SWEEP, sweep_expr  # noqa: E402
METRIC = "decimal rows/s (precision sweep a*b+c and a/b, p=18..600), bit-exact"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sweep", choices=["sweep", "batch", "query"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time of the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--only", default="", help="comma list of p:op sweep cases (profiling a subset)")
    ap.add_argument("--rows-scale", type=float, default=1.0, help="scale every case's rows (profiling)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# -------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit())
        mx = max((float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, n in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(self.samples)}


# ------------------------------------------------------------ workloads
def limbs(nbytes: int) -> int:
    return (nbytes + 3) // 4


def sweep_cases(scale_rows: float = 1.0):
    from ultraprecise_b200 import codec
    cases = []
    for p, rows in SWEEP:
        s = p // 4
        B = codec.compact_bytes(p)
        for op in ("mad", "div"):
            r = max(1, int(rows * scale_rows))
            if op == "mad":
                ob = codec.compact_bytes(2 * p + 1)
                nin = 3
                # limb multiply-adds per row: the a*b product plus aligning c by 10^s
                la = limbs(B)
                madds = la * la + la * limbs(max(1, ((10 ** s).bit_length() + 7) // 8))
            else:
                ob = codec.compact_bytes(max(s + 5, 1))
                nin = 2
                sh = s + 4
                la = limbs(B)
                nx = la + limbs(((10 ** sh).bit_length() + 7) // 8)
                madds = la * limbs(((10 ** sh).bit_length() + 7) // 8) + (nx - la + 1) * la
            cases.append({"p": p, "s": s, "op": op, "rows": r, "in_bytes": B, "n_in": nin, "out_bytes": ob,
                          "bytes_per_row": nin * B + ob, "madds_per_row": madds})
    return cases


def build_expr(case):
    return sweep_expr(case["p"], case["op"])


# DRAM bytes per row (dram__bytes_read.sum + dram__bytes_write.sum of one ncu
# capture, divided by the rows of the captured launch) for the sweep cases
# profiled so far: profiles/up_expr_tile_p600_mad.md, up_expr_tile_p38_mad.md.
NCU_TRAFFIC_PER_ROW = {(600, "mad"): 334.6e6 / 262144, (38, "mad"): 301.58e6 / 4194304}


# ---------------------------------------------------------- our arm
def run_ours(args, rank, world):
    import torch
    from ultraprecise_b200 import abi, runtime
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = abi.load()
    stream = torch.cuda.Stream()
    cases = sweep_cases(args.rows_scale)
    if args.only:
        keep = {tuple(x.split(":")) for x in args.only.split(",")}
        cases = [c for c in cases if (str(c["p"]), c["op"]) in keep]
    hbm_peak, peak_kind = peaks()
    madd_peak = C.c_double(0)
    abi.check(lib.up_util_imad_peak(C.byref(madd_peak), stream.cuda_stream), "imad peak")

    mods, inputs, outs = [], [], []
    with torch.cuda.stream(stream):
        for i, c in enumerate(cases):
            e, cols = build_expr(c)
            m = runtime.compile_expr(e, cols)
            mods.append(m)
            ins = []
            for k in range(c["n_in"]):
                t = runtime.gen_digits(c["rows"], c["p"], seed=1_000_003 * (i + 1) + 7919 * k + rank,
                                       nonzero=(c["op"] == "div" and k == 1), stream=stream)
                ins.append(runtime.DeviceColumn(t, c["p"], c["s"]))
            inputs.append(ins)
            outs.append(torch.empty(c["rows"] * m.value_bytes, dtype=torch.uint8, device="cuda"))
    torch.cuda.synchronize()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")

    def step():
        for i, (m, ins, o) in enumerate(zip(mods, inputs, outs)):
            m.launch(ins, cases[i]["rows"], out=o, err=err, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    per_case = [0.0] * len(cases)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # per-kernel events on the launching stream, recorded inside the timed region
    evs = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in cases]
           for _ in range(args.steps)]
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        t0.record(stream)
        for k in range(args.steps):
            for i, (m, ins, o) in enumerate(zip(mods, inputs, outs)):
                evs[k][i][0].record(stream)
                m.launch(ins, cases[i]["rows"], out=o, err=err, stream=stream)
                evs[k][i][1].record(stream)
        t1.record(stream)
        torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    for k in range(args.steps):
        for i in range(len(cases)):
            per_case[i] += evs[k][i][0].elapsed_time(evs[k][i][1]) / args.steps
    total_ms = max_over_ranks(total_ms, world)
    rows_per_step = sum(c["rows"] for c in cases)
    ms_per_step = total_ms / args.steps
    value = rows_per_step * world / (ms_per_step * 1e-3)

    case_rep = []
    for c, ms in zip(cases, per_case):
        gbs = c["bytes_per_row"] * c["rows"] / (ms * 1e-3) / 1e9
        gmadds = c["madds_per_row"] * c["rows"] / (ms * 1e-3) / 1e9
        case_rep.append({"p": c["p"], "op": c["op"], "rows": c["rows"], "ms": round(ms, 4),
                         "rows_per_s": round(c["rows"] / (ms * 1e-3)),
                         "hbm_gbs": round(gbs, 1), "hbm_frac": round(gbs / hbm_peak, 4),
                         "int_gmadds": round(gmadds, 1), "int_frac": round(gmadds * 1e9 / madd_peak.value, 4)})
    dom = max(range(len(cases)), key=lambda i: per_case[i])
    dc, dr = cases[dom], case_rep[dom]
    tr = NCU_TRAFFIC_PER_ROW.get((dc["p"], dc["op"]))
    traffic = round(tr * dc["rows"]) if tr else None
    hbm_bound = dr["hbm_frac"] >= dr["int_frac"]
    if hbm_bound:
        roof = {"bound": "hbm", "achieved": dr["hbm_gbs"], "peak": hbm_peak, "unit": "GB/s",
                "frac": round(dr["hbm_gbs"] / hbm_peak, 4), "traffic": traffic,
                "kernel": f"up_expr_tile p={dc['p']} {dc['op']}", "peak_source": peak_kind,
                "algorithmic_bytes": dc["bytes_per_row"] * dc["rows"]}
    else:
        roof = {"bound": "int32", "achieved": dr["int_gmadds"], "peak": round(madd_peak.value / 1e9, 1),
                "unit": "G limb-madd/s", "frac": dr["int_frac"], "traffic": traffic,
                "kernel": f"up_expr_tile p={dc['p']} {dc['op']}",
                "algorithmic_bytes": dc["bytes_per_row"] * dc["rows"],
                "madds_per_row": dc["madds_per_row"],
                "peak_source": "measured (up_util_imad_peak)",
                "hbm_achieved_gbs": dr["hbm_gbs"], "hbm_frac": dr["hbm_frac"]}
    res = {"metric": METRIC, "value": round(value), "unit": "rows/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (exact decimal)", "data": "synthetic",
           "config": {"workload": "precision sweep (configs[1]): a*b+c and a/b on DECIMAL(p,p/4), "
                                  "p in 18,38,76,150,300,600; 16M rows p<=38 halved per doubling",
                      "rows_per_step_per_gpu": rows_per_step, "l2": "inputs larger than L2 (no flush)",
                      "parallelism": f"replicas x{world} (row shards, no collective)"},
           "roofline": roof, "cases": case_rep,
           "gpu_launches": len(cases) * args.steps,
           "imad_peak_gmadds": round(madd_peak.value / 1e9, 1)}
    res["clocks"] = clk.summary()
    if not args.no_e2e:
        res["e2e"] = e2e_ours(args, cases, mods, world, stream)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        res["cpu_baseline"] = cpu_baseline(cases, args.cpu_seconds)
    return res


def e2e_ours(args, cases, mods, world, stream):
    """Same metric through the C ABI with HOST buffers: per step, every input
    column is copied from pinned host memory, the kernel runs, and every
    result is copied back to pinned host memory."""
    import torch
    from ultraprecise_b200 import runtime
    host_in, host_out, dev_in, dev_out = [], [], [], []
    for i, (c, m) in enumerate(zip(cases, mods)):
        ins, dins = [], []
        for k in range(c["n_in"]):
            d = runtime.gen_digits(c["rows"], c["p"], seed=77 + 31 * i + k, nonzero=(c["op"] == "div" and k == 1))
            h = torch.empty(d.numel(), dtype=torch.uint8, pin_memory=True)
            h.copy_(d)
            ins.append(h)
            dins.append(torch.empty_like(d))
        host_in.append(ins)
        dev_in.append(dins)
        host_out.append(torch.empty(c["rows"] * m.value_bytes, dtype=torch.uint8, pin_memory=True))
        dev_out.append(torch.empty(c["rows"] * m.value_bytes, dtype=torch.uint8, device="cuda"))
    h2d = sum(t.numel() for ins in host_in for t in ins)
    d2h = sum(t.numel() for t in host_out)

    def step():
        with torch.cuda.stream(stream):
            for i, (c, m) in enumerate(zip(cases, mods)):
                cols = []
                for k in range(c["n_in"]):
                    dev_in[i][k].copy_(host_in[i][k], non_blocking=True)
                    cols.append(runtime.DeviceColumn(dev_in[i][k], c["p"], c["s"]))
                m.launch(cols, c["rows"], out=dev_out[i], stream=stream)
                host_out[i].copy_(dev_out[i], non_blocking=True)

    steps = max(1, min(args.steps, 3))
    for _ in range(max(1, min(args.warmup, 2))):
        step()
    torch.cuda.synchronize()
    barrier(world)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1), world) / steps
    rows = sum(c["rows"] for c in cases)
    del dev_in, dev_out
    return {"value": round(rows * world / (ms * 1e-3)), "unit": "rows/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": round(ms, 3), "steps": steps}


# ------------------------------------------------------------ batch workload
BATCH_METRIC = "queries/s (64-task batched mixed-precision set, graph-replayed persistent kernels), bit-exact"


def batch_setup(rank):
    from ultraprecise_b200 import codec, workloads
    tasks, redraws = workloads.batch_tasks()
    for t in tasks:
        nb = codec.compact_bytes(t["p"])
        t["madds_per_row"], _, _ = workloads.expr_madds(t["expr"], t["s"], nb)
        t["in_bytes_per_row"] = t["ncols"] * nb
    return tasks, redraws


def run_batch(args, rank, world):
    import torch
    from ultraprecise_b200 import abi, batch, runtime, workloads
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = abi.load()
    stream = torch.cuda.Stream()
    tasks, redraws = batch_setup(rank)
    hbm_peak, peak_kind = peaks()
    madd_peak = C.c_double(0)
    abi.check(lib.up_util_imad_peak(C.byref(madd_peak), stream.cuda_stream), "imad peak")
    specs = workloads.batch_specs(tasks)
    t_build = time.perf_counter()
    b = batch.Batch(specs, autotune=True, use_graph=True)
    build_s = time.perf_counter() - t_build
    with torch.cuda.stream(stream):
        data = workloads.batch_columns(tasks, seed=20261203 + 1000003 * rank)
    torch.cuda.synchronize()
    outs, gids, devcols = [], [], []
    out_bytes = 0
    for k, (t, (rows, cols, gid)) in enumerate(zip(tasks, data)):
        dc = [runtime.DeviceColumn(c, t["p"], t["s"]) for c in cols]
        devcols.append(dc)
        if t["agg"] < 0:
            vb = b.task_type(k)[2]
            t["out_bytes_per_row"] = vb
            o = torch.empty(max(1, rows * vb), dtype=torch.uint8, device="cuda")
            b.bind(k, dc, rows, o)
            gids.append(None)
        else:
            t["out_bytes_per_row"] = 4  # the group id read
            g = torch.from_numpy(gid).cuda()
            o = torch.empty(t["groups"] * abi.UP_AGG_DECIMAL_BYTES, dtype=torch.uint8, device="cuda")
            b.bind(k, dc, rows, o, g, t["groups"])
            gids.append(g)
        out_bytes += o.numel()
        outs.append(o)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    t_tune = time.perf_counter()
    b.launch(err, stream=stream)  # tunes (or loads the tuned shapes) and captures the graph
    torch.cuda.synchronize()
    tune_s = time.perf_counter() - t_tune

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), world) / steps

    with ClockSampler(dev) as clk:
        ms_batch = timed(lambda: b.launch(err, stream=stream), args.steps, args.warmup)
    clocks = clk.summary()

    # the same 64 tasks, one plain launch each (no synchronisation between them)
    plain = []
    for t in tasks:
        if t["agg"] < 0:
            plain.append(runtime.compile_expr(t["expr"], t["cols"]))
        else:
            plain.append(runtime.compile_query([t["expr"]], [(t["agg"], 0)], t["cols"]))
    plain_out = [torch.empty_like(o) for o in outs]

    def plain_step():
        for k, (t, m) in enumerate(zip(tasks, plain)):
            if t["agg"] < 0:
                m.launch(devcols[k], data[k][0], out=plain_out[k], err=err, stream=stream)
            else:
                m.launch(devcols[k], gids[k], t["groups"], outs=[plain_out[k]], err=err, stream=stream)

    ms_plain = timed(plain_step, max(1, min(args.steps, 5)), max(1, min(args.warmup, 3)))
    torch.cuda.synchronize()
    same = all(torch.equal(a, c) for a, c in zip(outs, plain_out))

    rows = sum(t["rows"] for t in tasks)
    bytes_step = sum(t["rows"] * (t["in_bytes_per_row"] + t["out_bytes_per_row"]) for t in tasks)
    madds_step = sum(t["rows"] * t["madds_per_row"] for t in tasks)
    gmadds = madds_step / (ms_batch * 1e-3) / 1e9
    gbs = bytes_step / (ms_batch * 1e-3) / 1e9
    n = len(tasks)
    shapes = {f"band{i}": b.shape(i) for i in range(3)}
    res = {"metric": BATCH_METRIC, "value": round(n * world / (ms_batch * 1e-3), 2), "unit": "queries/s",
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_batch, 4),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "u32 limbs (exact decimal)", "data": "synthetic",
           "config": {"workload": "64-task batched mixed precision (seeded trees, p 10-400, rows 1e3-1e7, half "
                                  "grouped SUM over Zipf(1.1) keys)", "rows_per_step_per_gpu": rows,
                      "tree_redraws": redraws, "l2": "inputs larger than L2 (no flush)",
                      "parallelism": f"replicas x{world} (no collective)"},
           "rows_per_s": round(rows * world / (ms_batch * 1e-3)),
           "plain": {"ms_per_step": round(ms_plain, 4), "queries_per_s": round(n * world / (ms_plain * 1e-3), 2),
                     "speedup_batched": round(ms_plain / ms_batch, 3), "byte_equal": same},
           "roofline": {"bound": "int32", "achieved": round(gmadds, 1), "peak": round(madd_peak.value / 1e9, 1),
                        "unit": "G limb-madd/s", "frac": round(gmadds * 1e9 / madd_peak.value, 4),
                        "traffic": None, "kernel": "up_batch band kernels (whole graph)",
                        "peak_source": "measured (up_util_imad_peak)", "hbm_achieved_gbs": round(gbs, 1),
                        "hbm_frac": round(gbs / hbm_peak, 4)},
           "shapes": shapes, "module_build_s": round(build_s, 2), "tune_and_capture_s": round(tune_s, 2),
           "gpu_launches": args.steps * (1 + sum(1 for i in range(3) if any(
               b.task_type(k)[3] == i for k in range(n)))), "clocks": clocks}
    if not args.no_e2e:
        res["e2e"] = e2e_batch(args, b, tasks, data, outs, gids, world, stream)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        res["cpu_baseline"] = cpu_baseline_batch(tasks, args.cpu_seconds)
    return res


def e2e_batch(args, b, tasks, data, outs, gids, world, stream):
    """The batch through its public API with HOST buffers: per step every
    task's columns and group ids are copied from pinned host memory into the
    bound device buffers, the graph runs, and every result is copied back."""
    import torch
    pairs_in, pairs_out = [], []
    for k, (rows, cols, _) in enumerate(data):
        for c in cols:
            h = torch.empty(c.numel(), dtype=torch.uint8, pin_memory=True)
            h.copy_(c)
            pairs_in.append((c, h))
        if gids[k] is not None:
            h = torch.empty(gids[k].numel(), dtype=torch.int32, pin_memory=True)
            h.copy_(gids[k])
            pairs_in.append((gids[k], h))
        pairs_out.append((torch.empty(outs[k].numel(), dtype=torch.uint8, pin_memory=True), outs[k]))
    h2d = sum(h.numel() * h.element_size() for _, h in pairs_in)
    d2h = sum(h.numel() for h, _ in pairs_out)

    def step():
        with torch.cuda.stream(stream):
            for d, h in pairs_in:
                d.copy_(h, non_blocking=True)
            b.launch(None, stream=stream)
            for h, d in pairs_out:
                h.copy_(d, non_blocking=True)

    steps = max(1, min(args.steps, 3))
    step()
    torch.cuda.synchronize()
    barrier(world)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1), world) / steps
    return {"value": round(len(tasks) * world / (ms * 1e-3), 2), "unit": "queries/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": round(ms, 3), "steps": steps}


def batch_cpu_rate(tasks, cpu_seconds, threads, seed=1):
    """Oracle time for the 64 tasks on the host cores, every task at one common
    fraction of its rows, extrapolated to full rows: (queries/s, fraction, rows)."""
    import numpy as np
    from oracle import gen, oracle
    from ultraprecise_b200 import codec, workloads
    from ultraprecise_b200 import expr as E

    def run(frac):
        secs, rows_tot = 0.0, 0
        for k, t in enumerate(tasks):
            r = max(4, int(t["rows"] * frac))
            nb = codec.compact_bytes(t["p"])
            cols = [gen.compact_digits(r, t["p"], nb, seed + 97 * k + c, nonzero=True) for c in range(t["ncols"])]
            bt = E.build([t["expr"]], t["cols"])
            E.derive_types(bt)
            if t["agg"] < 0:
                ob = codec.compact_bytes(bt.nodes[bt.roots[0]].precision)
                t0 = time.perf_counter()
                oracle.eval_expr(bt, bt.roots[0], cols, r, ob, threads=threads)
            else:
                g = workloads.batch_group_ids(r, t["groups"], seed + k).tobytes()
                t0 = time.perf_counter()
                oracle.query(bt, [(t["agg"], bt.roots[0])], cols, g, r, t["groups"], threads=threads)
            secs += time.perf_counter() - t0
            rows_tot += r
        return secs, rows_tot

    f0 = 1.0 / 4096
    s0, _ = run(f0)
    frac = min(1.0 / 8, f0 * cpu_seconds / max(s0, 1e-4))
    s1, rows = run(frac)
    return len(tasks) / (s1 / frac), frac, rows


def cpu_baseline_batch(tasks, cpu_seconds):
    threads = os.cpu_count() or 1
    rate, frac, rows = batch_cpu_rate(tasks, cpu_seconds, threads)
    return {"value": round(rate, 4), "unit": "queries/s", "cores": threads, "kind": "port",
            "sample": f"{rows} rows: every task at {frac:.2e} of its rows, time scaled to full rows; oracle on "
                      f"{threads} host threads"}


# ------------------------------------------------------------ query workload
QUERY_METRIC = "decimal rows/s (fused grouped SUM/AVG/COUNT query over DECIMAL(15,2)), bit-exact"
QUERY_BYTES_PER_ROW = 4 * 7 + 4  # four 7-byte decimal columns and the int32 group id


def query_inputs(rows, seed, stream=None):
    import torch
    from ultraprecise_b200 import runtime, workloads
    R = workloads.QUERY_RANGES
    cols = [runtime.gen_range(rows, 15, *R[n], seed + i, stream=stream) for i, n in enumerate(("qty", "price",
                                                                                                 "disc", "tax"))]
    g = torch.Generator(device="cuda").manual_seed(seed)
    w = torch.tensor([k[2] for k in workloads.QUERY_KEYS], device="cuda")
    pick = torch.multinomial(w, rows, replacement=True, generator=g) if rows <= (1 << 24) else torch.cat(
        [torch.multinomial(w, min(1 << 24, rows - o), replacement=True, generator=g) for o in range(0, rows, 1 << 24)])
    k1 = torch.tensor([k[0][0] for k in workloads.QUERY_KEYS], dtype=torch.uint8, device="cuda")[pick].contiguous()
    k2 = torch.tensor([k[1][0] for k in workloads.QUERY_KEYS], dtype=torch.uint8, device="cuda")[pick].contiguous()
    del pick
    return cols, k1, k2


def run_query(args, rank, world):
    import torch
    from ultraprecise_b200 import abi, runtime, workloads
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    hbm_peak, peak_kind = peaks()
    exprs, aggs, ctypes_ = workloads.query_exprs()
    q = runtime.compile_query(exprs, aggs, ctypes_)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    results = {}
    for label, rows in (("1M", 1 << 20), ("256M", max(1, int((256 << 20) * args.rows_scale)))):
        with torch.cuda.stream(stream):
            cols, k1, k2 = query_inputs(rows, 20261203 + 7 * rank, stream)
            torch.cuda.synchronize()
            gid, G, _ = runtime.group_ids_from_keys([k1, k2], [1, 1], stream=stream)  # warm (module load)
            gid_ms = 1e30
            for _ in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                gid, G, _ = runtime.group_ids_from_keys([k1, k2], [1, 1], stream=stream)
                e1.record(stream)
                torch.cuda.synchronize()
                gid_ms = min(gid_ms, e0.elapsed_time(e1))
        dc = [runtime.DeviceColumn(c, 15, 2) for c in cols]
        outs = [torch.empty(G * (8 if k == abi.UP_AGG_COUNT else abi.UP_AGG_DECIMAL_BYTES), dtype=torch.uint8,
                            device="cuda") for k, _ in aggs]

        def step():
            q.launch(dc, gid, G, outs=outs, err=err, stream=stream)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        barrier(world)
        steps = args.steps
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(dev) as clk:
            e0.record(stream)
            for _ in range(steps):
                step()
            e1.record(stream)
            torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world) / steps
        gbs = QUERY_BYTES_PER_ROW * rows / (ms * 1e-3) / 1e9
        results[label] = {"rows": rows, "groups": G, "ms_per_step": round(ms, 4),
                          "rows_per_s": round(rows * world / (ms * 1e-3)), "hbm_gbs": round(gbs, 1),
                          "hbm_frac": round(gbs / hbm_peak, 4), "group_ids_ms": round(gid_ms, 3),
                          "clocks": clk.summary()}
        if label == "256M":
            main = results[label]
            inputs = (cols, k1, k2, gid, G, outs)
        else:
            del cols, k1, k2, gid, dc, outs
    m = main
    res = {"metric": QUERY_METRIC, "value": m["rows_per_s"], "unit": "rows/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u32 limbs (exact decimal)", "data": "synthetic",
           "config": {"workload": f"grouped SUMx4/AVGx3/COUNT query, DECIMAL(15,2) x4, 2 CHAR(1) keys, "
                                  f"{m['rows']} rows (256M roofline run; 1M-row case in 'rows_1m')",
                      "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world} (no collective)"},
           "roofline": {"bound": "hbm", "achieved": m["hbm_gbs"], "peak": hbm_peak, "unit": "GB/s",
                        "frac": m["hbm_frac"], "traffic": None, "kernel": "up_query_acc + up_query_fin",
                        "peak_source": peak_kind, "bytes_per_row": QUERY_BYTES_PER_ROW},
           "rows_1m": results["1M"], "gpu_launches": 2 * args.steps, "clocks": m["clocks"]}
    if not args.no_e2e:
        res["e2e"] = e2e_query(args, q, aggs, inputs, world, stream)
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        rate, rows = query_cpu_rate(args.cpu_seconds, os.cpu_count() or 1)
        res["cpu_baseline"] = {"value": round(rate), "unit": "rows/s", "cores": os.cpu_count() or 1,
                               "kind": "port", "sample": f"{rows} rows of the same query, oracle on "
                                                         f"{os.cpu_count() or 1} host threads"}
    return res


def e2e_query(args, q, aggs, inputs, world, stream):
    """The query through the C ABI with HOST buffers: per step the four
    decimal columns and the group ids are copied from pinned host memory, the
    query runs, and the eight aggregate outputs are copied back."""
    import torch
    from ultraprecise_b200 import runtime
    cols, k1, k2, gid, G, outs = inputs
    pairs = []
    for d in list(cols) + [gid]:
        h = torch.empty(d.numel(), dtype=d.dtype, pin_memory=True)
        h.copy_(d)
        pairs.append((d, h))
    hout = [torch.empty(o.numel(), dtype=torch.uint8, pin_memory=True) for o in outs]
    dc = [runtime.DeviceColumn(c, 15, 2) for c in cols]
    h2d = sum(h.numel() * h.element_size() for _, h in pairs)
    d2h = sum(h.numel() for h in hout)

    def step():
        with torch.cuda.stream(stream):
            for d, h in pairs:
                d.copy_(h, non_blocking=True)
            q.launch(dc, gid, G, outs=outs, stream=stream)
            for h, o in zip(hout, outs):
                h.copy_(o, non_blocking=True)

    step()
    torch.cuda.synchronize()
    barrier(world)
    steps = max(1, min(args.steps, 3))
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(t0.elapsed_time(t1), world) / steps
    rows = gid.numel()
    return {"value": round(rows * world / (ms * 1e-3)), "unit": "rows/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": round(ms, 3), "steps": steps}


def query_cpu_rate(cpu_seconds, threads, seed=3):
    """Oracle rows/s for the query on the host cores, sized for ~cpu_seconds."""
    import numpy as np
    from oracle import gen, oracle
    from ultraprecise_b200 import workloads
    from ultraprecise_b200 import expr as E
    exprs, aggs, ctypes_ = workloads.query_exprs()
    b = E.build(exprs, ctypes_)
    E.derive_types(b)
    qa = [(k, b.roots[i]) for k, i in aggs]

    def run(rows):
        rng = np.random.default_rng(seed)
        R = workloads.QUERY_RANGES
        cols = []
        for n in ("qty", "price", "disc", "tax"):
            lo, hi, st = R[n]
            v = lo + st * rng.integers(0, (hi - lo) // st + 1, rows, dtype=np.int64)
            cols.append(gen.pack_unsigned(v, 7))
        w = np.array([k[2] for k in workloads.QUERY_KEYS])
        g = rng.choice(len(w), size=rows, p=w / w.sum()).astype(np.int32).tobytes()
        t = time.perf_counter()
        oracle.query(b, qa, cols, g, rows, len(w), threads=threads)
        return time.perf_counter() - t

    r0 = 1 << 16
    s0 = run(r0)
    rows = int(min(1 << 28, r0 * cpu_seconds / max(s0, 1e-4)))
    return rows / run(rows), rows


# ------------------------------------------------------ CPU baseline
def cpu_rate(cases, cpu_seconds, threads, seed=1):
    """Time the oracle on the host cores over the same sweep mix (every case
    scaled by one common fraction of its rows), sized for ~cpu_seconds."""
    from oracle import gen, oracle
    from ultraprecise_b200 import codec
    from ultraprecise_b200 import expr as E

    def run(frac):
        rows_tot, secs = 0, 0.0
        for i, c in enumerate(cases):
            r = max(8, int(c["rows"] * frac))
            cols = [gen.compact_digits(r, c["p"], c["in_bytes"], seed + 31 * i + k,
                                       nonzero=(c["op"] == "div" and k == 1)) for k in range(c["n_in"])]
            e, ct = build_expr(c)
            b = E.build([e], ct)
            E.derive_types(b)
            ob = codec.compact_bytes(b.nodes[b.roots[0]].precision)
            t = time.perf_counter()
            oracle.eval_expr(b, b.roots[0], cols, r, ob, threads=threads)
            secs += time.perf_counter() - t
            rows_tot += r
        return rows_tot, secs

    f0 = 1.0 / 65536
    r0, s0 = run(f0)
    frac = min(1.0 / 16, f0 * cpu_seconds / max(s0, 1e-4))
    r1, s1 = run(frac)
    return r1 / s1, frac, r1


def cpu_baseline(cases, cpu_seconds):
    threads = os.cpu_count() or 1
    rate, frac, rows = cpu_rate(cases, cpu_seconds, threads)
    return {"value": round(rate), "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": f"{rows} rows: every sweep case at {frac:.2e} of its rows (same mix), oracle on "
                      f"{threads} host threads"}


# ---------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    """The reference's decimal arithmetic has no CPU implementation (it is
    device-only PTX); its restatement in oracle/ runs on all host cores."""
    if rank != 0:
        return None
    threads = os.cpu_count() or 1
    if args.workload == "query":
        per = args.cpu_seconds / max(1, args.steps)
        rates, rows = [], 0
        for k in range(max(1, args.steps)):
            r, rows = query_cpu_rate(per, threads, seed=3 + k)
            rates.append(r)
        rate = sorted(rates)[len(rates) // 2]
        return {"metric": QUERY_METRIC, "value": round(rate), "unit": "rows/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round((256 << 20) / rate * 1e3, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (exact decimal)", "data": "synthetic",
                "impl": "reference", "config": {"workload": "grouped query on host cores, bounded sample",
                                                "parallelism": f"{threads} host threads"},
                "cpu_baseline": {"value": round(rate), "unit": "rows/s", "cores": threads, "kind": "port",
                                 "sample": f"{rows} rows per step"},
                "e2e": {"value": round(rate), "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "batch":
        tasks, _ = batch_setup(rank)
        per = args.cpu_seconds / max(1, args.steps)
        rates, rows, frac = [], 0, 0.0
        for k in range(max(1, args.steps)):
            r, frac, rows = batch_cpu_rate(tasks, per, threads, seed=1 + k)
            rates.append(r)
        rate = sorted(rates)[len(rates) // 2]
        return {"metric": BATCH_METRIC, "value": round(rate, 4), "unit": "queries/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(len(tasks) / rate * 1e3, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u32 limbs (exact decimal)", "data": "synthetic", "impl": "reference",
                "config": {"workload": "64-task batched mixed precision on host cores, bounded sample",
                           "parallelism": f"{threads} host threads"},
                "cpu_baseline": {"value": round(rate, 4), "unit": "queries/s", "cores": threads, "kind": "port",
                                 "sample": f"{rows} rows per step: every task at {frac:.2e} of its rows"},
                "e2e": {"value": round(rate, 4), "unit": "queries/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
    cases = sweep_cases()
    per = args.cpu_seconds / max(1, args.steps)
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_rate(cases, min(per, 2.0), threads, seed=99)
    rates, rows = [], 0
    for k in range(max(1, args.steps)):
        r, frac, rows = cpu_rate(cases, per, threads, seed=1 + k)
        rates.append(r)
    rate = sorted(rates)[len(rates) // 2]
    total_rows = sum(c["rows"] for c in cases)
    return {"metric": METRIC, "value": round(rate), "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_rows / rate * 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 limbs (exact decimal)", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "precision sweep (configs[1]) on host cores, bounded sample",
                       "parallelism": f"{threads} host threads"},
            "cpu_baseline": {"value": round(rate), "unit": "rows/s", "cores": threads, "kind": "port",
                             "sample": f"{rows} rows per step: every sweep case at {frac:.2e} of its rows"},
            "e2e": {"value": round(rate), "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------- distributed
def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        res = run_reference(args, rank, world)
        if res is not None:
            print(json.dumps(res))
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    run = {"batch": run_batch, "query": run_query}.get(args.workload, run_ours)
    res = run(args, rank, world)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


if __name__ == "__main__":
    main()
