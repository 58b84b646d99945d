"""Benchmark of the engine's headline workload: the two bandwidth-bound scans over a
60,000,000-row synthetic lineitem table (filtered sum Q6-like, 6-group aggregate Q1-like),
one step = one pass of each pipeline over the table.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). value = lineitem rows scanned per second by the whole job
(2 x rows x N per step), device-timed over K steps of async calls on the engine's stream;
`roofline` is the Q1 kernel's, its launch time from CUDA events around the calls of every
16th step of that timed region; e2e = the same metric through the C ABI with the table in pinned
host memory (chunked host->HBM streaming inside the timed region), one call per pipeline;
e2e_batched = the same two requests as one gpudb_batch_run call, which copies each chunk
once for both scans. For N > 1 (torchrun) every rank scans its own 60M-row shard of one
table (weak scaling, no collective on the data path); times are the max over ranks.

On one GPU the line also carries, under `pipelines`, the device time, rows/s and HBM
roofline fraction of every other configuration of the workload: the Q1 aggregate at 6M
rows, the Q3 join + top-10 at 1x and 10x in each join mode, the Q9 star join at 60M fact
rows and streamed at 600M, the join microbenchmark; under `serve`, the served mixed
stream against the plain one-query-per-launch form (queries/s, p50/p99, bit-exact flag);
and two CPU baselines: the reference's own kernels on all host cores (`cpu_baseline`) and
the single-threaded C oracle (`cpu_baseline_oracle`).

--impl reference times the reference's own kernels (kernels/q6.metal, kernels/q1.metal of
nd-tung/GPUDBMetalBenchmark) compiled for the host CPU (oracle/_ref), on all host cores.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "lineitem rows/s (Q6-like filtered sum + Q1-like 6-group aggregate over 60M rows)"
Q6_BYTES_PER_ROW = 20   # ship_date 4 + discount 4 + quantity 4 + ext_price 8
Q1_BYTES_PER_ROW = 26   # ship_date 4 + quantity 4 + ext_price 8 + discount 4 + tax 4 + flag 1 + status 1
TIME_EVERY = 16         # one step in TIME_EVERY has its two calls timed with CUDA events


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=60_000_000)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--skip-cpu", action="store_true", help="no CPU baselines (profiling runs)")
    ap.add_argument("--skip-extra", action="store_true",
                    help="only the config-1 step: no per-pipeline block, serving comparison or CPU baselines")
    ap.add_argument("--no-stream600m", action="store_true", help="leave out the 600M-row streamed Q9 case")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes per row of a kernel from a committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while the timed region runs."""

    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.15)
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == len(self.FIELDS):
                self.rows.append(parts)

    def __exit__(self, *a):
        time.sleep(0.15)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def physical_index(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",")]
        if local < len(ids) and ids[local].isdigit():
            return int(ids[local])
    return local


# ---------------------------------------------------------------------------------------
def cpu_baseline(rows_total, seed):
    """The reference's own Q6/Q1 kernels compiled for the host CPU (oracle/_ref), all host
    threads, on a bounded sample of the same workload."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np
    import oracle_py as orc
    threads = os.cpu_count() or 1
    sample = min(rows_total, 8_000_000)
    li = orc.lineitem(sample, seed)
    ref = orc.reference()
    cols = ("ship_date", "quantity", "ext_price", "discount", "tax", "flag", "status")
    if ref is not None:
        ref.ref_scan_prepare.restype = C.c_void_p
        ref.ref_scan_prepare.argtypes = [C.c_uint64] + [C.c_void_p] * 7
        ref.ref_q6_run.restype = C.c_float
        ref.ref_q6_run.argtypes = [C.c_void_p] + [C.c_int32] * 5 + [C.c_int, C.c_int]
        ref.ref_q1_run.restype = C.c_uint32
        ref.ref_q1_run.argtypes = [C.c_void_p, C.c_int32, C.c_int, C.c_int]
        ref.ref_scan_free.argtypes = [C.c_void_p]
        h = ref.ref_scan_prepare(sample, *(li[c].ctypes.data for c in cols))
        groups = threads * 8

        def step():
            ref.ref_q6_run(h, 365, 730, 5, 7, 24, groups, threads)
            ref.ref_q1_run(h, 2436, groups, threads)
        kind = "reference"
    else:
        h = None

        def step():
            orc.q6(li, threads=threads)
            orc.q1(li, threads=threads)
        kind = "port"
    step()
    times = []
    t_end = time.perf_counter() + 10.0
    while time.perf_counter() < t_end or len(times) < 3:
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
        if len(times) >= 50:
            break
    if h is not None:
        ref.ref_scan_free(h)
    del np
    t = statistics.median(times)
    return {"value": 2 * sample / t, "unit": "rows/s", "cores": threads, "kind": kind,
            "sample": "%d of the 60M rows (Q6 + Q1 per step), median of %d runs, float32 columns "
                      "prepared once outside the timing" % (sample, len(times)) if kind == "reference" else
                      "%d rows, oracle port, median of %d runs" % (sample, len(times)),
            "step_s": t}


def cpu_baseline_oracle(li_host, rows):
    """The project's single-threaded C oracle (exact int128 sums) over the same 60M-row table
    in host memory, Q6 + Q1 per step, median of 5 steps."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as orc
    times = []
    for _ in range(5):
        t0 = time.perf_counter()
        orc.q6(li_host)
        orc.q1(li_host)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"value": 2 * rows / t, "unit": "rows/s", "cores": 1, "kind": "port",
            "sample": "all %d rows of the workload (Q6 + Q1 per step), single-threaded C oracle, median of 5" % rows,
            "step_s": t}


def workload_config(rows, world):
    return {"workload": "config 1: Q6-like filtered sum (1a) + Q1-like 6-group aggregate (1b) over a "
                        "%d-row lineitem table per GPU" % rows,
            "rows_per_gpu": rows, "l2": "inputs %.2f GB per step > 126 MB L2, no flush needed" % (46 * rows / 1e9),
            "parallelism": "row shards, one per GPU" if world > 1 else "single GPU"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py as orc
    ref = orc.reference()
    threads = os.cpu_count() or 1
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libgpudbref.so (the reference's kernels "
                                                              "compiled for the CPU) is not built"}))
        return 0
    ref.ref_scan_prepare.restype = C.c_void_p
    ref.ref_scan_prepare.argtypes = [C.c_uint64] + [C.c_void_p] * 7
    ref.ref_q6_run.restype = C.c_float
    ref.ref_q6_run.argtypes = [C.c_void_p] + [C.c_int32] * 5 + [C.c_int, C.c_int]
    ref.ref_q1_run.restype = C.c_uint32
    ref.ref_q1_run.argtypes = [C.c_void_p, C.c_int32, C.c_int, C.c_int]
    ref.ref_scan_free.argtypes = [C.c_void_p]
    cols = ("ship_date", "quantity", "ext_price", "discount", "tax", "flag", "status")
    # size the per-step sample so that warmup + steps take about two minutes
    probe = 2_000_000
    li = orc.lineitem(probe, args.seed)
    h = ref.ref_scan_prepare(probe, *(li[c].ctypes.data for c in cols))
    groups = threads * 8
    t0 = time.perf_counter()
    ref.ref_q6_run(h, 365, 730, 5, 7, 24, groups, threads)
    ref.ref_q1_run(h, 2436, groups, threads)
    per_row = (time.perf_counter() - t0) / probe
    ref.ref_scan_free(h)
    budget = 120.0 / max(1, args.steps + args.warmup)
    sample = int(max(100_000, min(args.rows, budget / max(per_row, 1e-12))))
    li = orc.lineitem(sample, args.seed)
    h = ref.ref_scan_prepare(sample, *(li[c].ctypes.data for c in cols))
    for _ in range(args.warmup):
        ref.ref_q6_run(h, 365, 730, 5, 7, 24, groups, threads)
        ref.ref_q1_run(h, 2436, groups, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.ref_q6_run(h, 365, 730, 5, 7, 24, groups, threads)
        ref.ref_q1_run(h, 2436, groups, threads)
    dt = time.perf_counter() - t0
    ref.ref_scan_free(h)
    value = 2 * sample * args.steps / dt
    line = {"metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1000 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": workload_config(args.rows, world),
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "reference",
                             "sample": "%d of the %d rows per step (the reference's Q6 and Q1 kernels compiled for "
                                       "the host, float32 columns prepared once outside the timing)" % (sample, args.rows)},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------------
def h2d_probe(local, gb=1.0, reps=5):
    """Pinned host -> HBM copy bandwidth (GB/s), the bound of every streamed table."""
    import torch
    n = int(gb * 1e9)
    src = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    dst = torch.empty(n, dtype=torch.uint8, device="cuda:%d" % local)
    dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        dst.copy_(src, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    gbs = n * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9
    del src, dst
    torch.cuda.empty_cache()
    return gbs


def shared_pass(eng, li, steps, stream, ref6, ref1):
    """The same two requests as one gpudb_batch_run over the device-resident table: the Q1
    kernel evaluates the Q6 request on the rows it reads, so the union of the columns
    (26 B/row) is read once for both."""
    import torch
    from gpudbmetalbenchmark_b200 import capi
    reqs = (capi.Request * 2)()
    o6, o1 = capi.Q6Result(), capi.Q1Result()
    reqs[0].pipeline, reqs[0].li, reqs[0].q6 = capi.PIPE_Q6, C.pointer(li), capi.Q6Params(365, 730, 5, 7, 24)
    reqs[0].q6_out = C.pointer(o6)
    reqs[1].pipeline, reqs[1].li, reqs[1].q1 = capi.PIPE_Q1, C.pointer(li), capi.Q1Params(2436, 0)
    reqs[1].q1_out = C.pointer(o1)
    eng._check(eng.lib.gpudb_batch_run(eng.ctx, reqs, 2, None, None))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        eng._check(eng.lib.gpudb_batch_run(eng.ctx, reqs, 2, None, None))
    e1.record(stream)
    torch.cuda.synchronize()
    assert (o6.revenue, o6.rows_matched) == ref6 and bytes(o1) == ref1
    ms = e0.elapsed_time(e1) / steps
    rows = li.n_rows
    return {"ms": ms, "rows_per_s": 2 * rows / (ms * 1e-3), "gbs_algorithmic": 26 * rows / (ms * 1e-3) / 1e9,
            "call": "gpudb_batch_run with the Q6 and the Q1 request over the device-resident table (one read "
                    "of 26 B/row for both: the Q6 request rides on the Q1 kernel), synchronous per step"}


def pipelines_block(eng, reps, stream600m, h2d_gbs):
    """Every other configuration of the workload on this GPU (device time of the call's
    kernels, CUDA events on its stream, median of `reps` after a warm-up call)."""
    from gpudbmetalbenchmark_b200 import pipebench as pb
    quiet = pb.record
    out = {}
    r6, r1 = pb.scan_case(eng, 6_000_000, reps, out=quiet)
    out["q1_cfg0_6m"] = r1
    out["q6_6m"] = r6
    for label, key, sizes in (("config 2 (1x)", "q3_1x", (150_000, 1_500_000, 6_000_000)),
                              ("config 2 (10x)", "q3_10x", (1_500_000, 15_000_000, 60_000_000))):
        for mode, rec in pb.q3_case(eng, *sizes, reps, label, out=quiet).items():
            out["%s_%s" % (key, mode)] = rec
    q9 = pb.q9_case(eng, reps, stream600m, out=quiet)
    out["q9_60m"] = q9["resident"]
    if "streamed" in q9:
        rec = q9["streamed"]
        rec["h2d_probe_gbs"] = h2d_gbs
        rec["frac_of_h2d"] = rec["h2d_gbs"] / h2d_gbs if h2d_gbs else None
        out["q9_600m_streamed"] = rec
    for mode, rec in pb.join_count_case(eng, max(3, reps // 2), out=quiet).items():
        out["join_count_15m_60m_%s" % mode] = rec
    return out


def run_ours(args, rank, world, local):
    import torch
    from gpudbmetalbenchmark_b200 import Engine, capi
    from gpudbmetalbenchmark_b200.engine import Q1_COLS

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    eng = Engine(local)
    rows = args.rows
    # weak scaling: rank r scans rows [r*rows, (r+1)*rows) of one seeded table
    t = eng.generate("lineitem", rows, seed=args.seed, columns=Q1_COLS, row_offset=rank * rows)
    li = t.lineitem()
    stream = torch.cuda.ExternalStream(eng.lib.gpudb_stream(eng.ctx))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_ms(ms):
        if dist is None:
            return ms
        m = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        return float(m.item())

    r6, r1 = capi.Q6Result(), capi.Q1Result()
    for _ in range(args.warmup):
        eng.q6(li, async_=True, out=r6)
        eng.q1(li, async_=True, out=r1)
    eng.sync()

    K = args.steps
    # kernel durations: CUDA events around both calls of every TIME_EVERY-th step (events
    # between two launches hold the stream a few microseconds; on every call they would add
    # about 5% to the step)
    sampled = list(range(0, K, TIME_EVERY))
    t6 = {k: capi.Timing() for k in sampled}
    t1 = {k: capi.Timing() for k in sampled}
    o6 = [capi.Q6Result() for _ in range(K)]
    o1 = [capi.Q1Result() for _ in range(K)]
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with Clocks(physical_index(local)) as clk:
        launches0 = eng.launches()
        ev0.record(stream)
        for k in range(K):
            eng.q6(li, async_=True, out=o6[k], timing=t6.get(k))
            eng.q1(li, async_=True, out=o1[k], timing=t1.get(k))
        ev1.record(stream)
        eng.sync()
        launches = eng.launches() - launches0
        barrier()
    ms = max_ms(ev0.elapsed_time(ev1))
    # every step's result equals the first (same input): a cheap live consistency check
    assert all(o.revenue == o6[0].revenue for o in o6) and all(bytes(o) == bytes(o1[0]) for o in o1)
    ref6, ref1 = (o6[0].revenue, o6[0].rows_matched), bytes(o1[0])

    # the shards' results, merged with the engine's exact merge (one small all-gather after
    # the timed region): the whole job's answer
    merged = None
    if dist is not None:
        parts = [None] * world
        dist.all_gather_object(parts, (bytes(o6[0]), bytes(o1[0])))
        p6 = [capi.Q6Result.from_buffer_copy(x[0]) for x in parts]
        p1 = [capi.Q1Result.from_buffer_copy(x[1]) for x in parts]
        m6, m1 = capi.merge_q6(p6), capi.merge_q1(p1)
        assert bytes(capi.merge_q1(p1[::-1])) == bytes(m1)   # order-independent
        assert m6.rows_matched == sum(x.rows_matched for x in p6)
        merged = {"q6_revenue": m6.revenue, "q6_rows": m6.rows_matched,
                  "q1_rows": sum(g.count for g in m1.groups[:m1.n_groups]), "q1_groups": m1.n_groups,
                  "how": "all_gather of each rank's result structs, gpudb_q6/q1_result_merge on every rank"}
    q6_ms = statistics.mean(x.gpu_ms for x in t6.values())
    q1_ms = statistics.mean(x.gpu_ms for x in t1.values())
    peak, peak_kind = peaks()
    q1_gbs = Q1_BYTES_PER_ROW * rows / (q1_ms * 1e-3) / 1e9
    q6_gbs = Q6_BYTES_PER_ROW * rows / (q6_ms * 1e-3) / 1e9
    tr = ncu_traffic("q1_vec_smem_kernel")
    shared = None
    if world == 1 and not args.skip_extra:
        shared = shared_pass(eng, li, K, stream, ref6, ref1)
    eng.free(t)

    # ---- end to end: the same step through the C ABI from pinned host memory -------------
    e2e = e2e_b = None
    cpu_oracle = None
    if args.e2e_steps > 0:
        th = eng.generate("lineitem", rows, seed=args.seed, columns=Q1_COLS, row_offset=rank * rows,
                          location=capi.MEM_HOST)
        lh = th.lineitem()

        def timed_e2e(step):
            step()   # warm-up: sizes the streaming ring
            h2d = d2h = 0
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            barrier()
            e0.record(stream)
            for _ in range(args.e2e_steps):
                a, b = step()
                h2d += a
                d2h += b
            e1.record(stream)
            barrier()
            ems = max_ms(e0.elapsed_time(e1))
            return {"value": 2 * rows * world * args.e2e_steps / (ems * 1e-3), "unit": "rows/s",
                    "h2d_bytes_per_step": h2d // args.e2e_steps, "d2h_bytes_per_step": d2h // args.e2e_steps,
                    "ms_per_step": ems / args.e2e_steps, "h2d_gbs": h2d / (ems * 1e-3) / 1e9}

        def plain_step():
            a, b = capi.Timing(), capi.Timing()
            out1 = capi.Q1Result()
            got6 = eng.q6(lh, timing=a)
            eng.q1(lh, timing=b, out=out1)
            assert got6 == ref6 and bytes(out1) == ref1
            return a.h2d_bytes + b.h2d_bytes, a.d2h_bytes + b.d2h_bytes

        reqs = (capi.Request * 2)()
        q6o, q1o = capi.Q6Result(), capi.Q1Result()
        reqs[0].pipeline, reqs[0].li, reqs[0].q6 = capi.PIPE_Q6, C.pointer(lh), capi.Q6Params(365, 730, 5, 7, 24)
        reqs[0].q6_out = C.pointer(q6o)
        reqs[1].pipeline, reqs[1].li, reqs[1].q1 = capi.PIPE_Q1, C.pointer(lh), capi.Q1Params(2436, 0)
        reqs[1].q1_out = C.pointer(q1o)

        def batched_step():
            tm = capi.Timing()
            eng._check(eng.lib.gpudb_batch_run(eng.ctx, reqs, 2, C.byref(tm), None))
            assert reqs[0].status == capi.OK and reqs[1].status == capi.OK
            assert (q6o.revenue, q6o.rows_matched) == ref6 and bytes(q1o) == ref1
            return tm.h2d_bytes, tm.d2h_bytes

        e2e = timed_e2e(plain_step)
        e2e_b = timed_e2e(batched_step)
        e2e_b["call"] = "gpudb_batch_run with the Q6 and the Q1 request: each chunk copied once for both"
        if rank == 0 and world == 1 and not (args.skip_cpu or args.skip_extra):
            cpu_oracle = cpu_baseline_oracle({c: th.host_view(c) for c in Q1_COLS}, rows)
        eng.free(th)

    extra = {}
    if world == 1 and not args.skip_extra:
        h2d = h2d_probe(local)
        extra["h2d_probe_gbs"] = h2d
        extra["pipelines"] = pipelines_block(eng, 10, not args.no_stream600m, h2d)
        from gpudbmetalbenchmark_b200 import serve
        extra["serve"] = serve.compare(eng, seconds=args.serve_seconds)

    cpu = cpu_baseline(rows, args.seed) if (rank == 0 and world == 1 and not (args.skip_cpu or args.skip_extra)) \
        else None
    if rank == 0:
        pipes = {
            "q1_cfg1b_60m": {"ms": q1_ms, "rows_per_s": rows / (q1_ms * 1e-3), "gbs_algorithmic": q1_gbs,
                             "frac": q1_gbs / peak, "peak_kind": peak_kind},
            "q6_cfg1a_60m": {"ms": q6_ms, "rows_per_s": rows / (q6_ms * 1e-3), "gbs_algorithmic": q6_gbs,
                             "frac": q6_gbs / peak, "peak_kind": peak_kind,
                             "traffic": (ncu_traffic("q6_vec_kernel") * rows if ncu_traffic("q6_vec_kernel") else None)},
        }
        if shared is not None:
            shared["frac"] = shared["gbs_algorithmic"] / peak
            pipes["q6_q1_shared_pass_60m"] = shared
        pipes.update(extra.pop("pipelines", {}))
        line = {
            "metric": METRIC, "value": 2 * rows * world * K / (ms * 1e-3), "unit": "rows/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded generator, inputs larger than L2)",
            "config": workload_config(rows, world),
            "roofline": {"bound": "hbm", "kernel": "q1_vec_smem_kernel", "achieved": q1_gbs, "peak": peak,
                         "unit": "GB/s", "frac": q1_gbs / peak, "peak_kind": peak_kind,
                         "traffic": (tr * rows if tr else None),
                         "algorithmic_bytes": Q1_BYTES_PER_ROW * rows, "ms_per_launch": q1_ms,
                         "launches_timed": len(t1), "timed": "CUDA events around every %dth step's calls "
                                                              "inside the timed region" % TIME_EVERY},
            "pipelines": pipes,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "e2e": e2e,
            "e2e_batched": e2e_b,
            "cpu_baseline": cpu,
            "cpu_baseline_oracle": cpu_oracle,
        }
        if merged is not None:
            line["merged_result"] = merged
        line.update(extra)
        print(json.dumps(line))
    eng.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
