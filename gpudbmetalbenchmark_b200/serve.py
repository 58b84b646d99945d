"""Serving front end: resident tables, a mixed request stream, and the served-vs-plain
benchmark of BASELINE config 4.

    python -m gpudbmetalbenchmark_b200.serve [--rates 2000 5000 ...] [--seconds S]

Tables of configs 0-3 stay in HBM (lineitem at 1M, 6M and 60M rows, the Q3 tables at 1x,
a Q9 star at 6M fact rows). Each request is a pipeline drawn uniformly from Q6/Q1/Q3/Q9
with randomised constants (date bounds uniform over the date domain, segment uniform,
discount and quantity bounds spanning ~0.5%-98% selectivity). Arrivals are Poisson (open
loop, seeded). Each request's latency runs from submission to completion; every result is
checked against the same request executed alone through the single-request API.

Plain form: one lane, one request per batch (each query runs by itself, in arrival order).
Served form: several lanes with continuous batching (gpudb_serve_*).
"""
import argparse
import ctypes as C
import json
import random
import sys
import threading
import time

from . import capi
from .engine import Engine, Q1_COLS


class Server:
    def __init__(self, device=0, lanes=2, max_batch=64, memory_budget=0, heavy_lanes=0):
        self.lib = capi.load()
        cfg = capi.ServeConfig(device=device, lanes=lanes, max_batch=max_batch, memory_budget=memory_budget,
                               heavy_lanes=heavy_lanes)
        h = C.c_void_p()
        rc = self.lib.gpudb_serve_open(C.byref(cfg), C.byref(h))
        if rc != capi.OK:
            raise capi.GpudbError(rc, "gpudb_serve_open failed")
        self.h = h

    def submit(self, req):
        t = C.c_uint64()
        rc = self.lib.gpudb_serve_submit(self.h, C.byref(req), C.byref(t))
        if rc != capi.OK:
            raise capi.GpudbError(rc, "gpudb_serve_submit failed")
        return t.value

    def wait(self, ticket, timeout_ms=120000.0):
        lat = C.c_double()
        rc = self.lib.gpudb_serve_wait(self.h, ticket, timeout_ms, C.byref(lat))
        return rc, lat.value

    def warmup(self, jobs):
        """Runs the jobs once on every lane before traffic (sizes each lane's scratch)."""
        arr = (capi.Request * len(jobs))(*[j.req for j in jobs])
        rc = self.lib.gpudb_serve_warmup(self.h, arr, len(jobs))
        for j, a in zip(jobs, arr):   # the array holds copies of the request structs
            j.req.status, j.req.q9_groups = a.status, a.q9_groups
        if rc != capi.OK:
            raise capi.GpudbError(rc, "gpudb_serve_warmup failed")

    def stats(self):
        s = capi.ServeStats()
        self.lib.gpudb_serve_stats_get(self.h, C.byref(s))
        return {f: getattr(s, f) for f, _ in capi.ServeStats._fields_}

    def close(self):
        if self.h:
            self.lib.gpudb_serve_close(self.h)
            self.h = None


class Job:
    """One request plus the result storage it writes into."""

    def __init__(self, kind, req, out):
        self.kind, self.req, self.out = kind, req, out

    def result(self):
        r = self.out
        if self.kind == capi.PIPE_Q6:
            return (r.revenue, r.rows_matched)
        if self.kind == capi.PIPE_Q1:
            return bytes(r)
        if self.kind == capi.PIPE_Q3:
            return (r.n_groups, r.n_rows, bytes(r.rows))
        return (self.req.q9_groups, bytes(r))


class Workload:
    """HBM-resident tables of configs 0-3 and a seeded generator of mixed requests."""

    def __init__(self, engine, scan_rows=(1_000_000, 6_000_000, 60_000_000), q3=(150_000, 1_500_000, 6_000_000),
                 q9=(200_000, 10_000, 1_500_000, 6_000_000)):
        e = self.engine = engine
        self.scans = [e.generate("lineitem", n, seed=42, columns=Q1_COLS) for n in scan_rows]
        self.scan_structs = [t.lineitem() for t in self.scans]
        n_cu, n_or, n_li = q3
        cu = e.generate("customer", n_cu, seed=7)
        od = e.generate("orders", n_or, seed=7, n_cust=n_cu)
        li = e.generate("lineitem", n_li, seed=7, columns=("order_key", "ship_date", "ext_price", "discount"),
                        n_orders=n_or, order_mode=capi.ORDERS_CLUSTERED)
        self.q3 = capi.Q3Tables(cu.struct(), od.struct(), li.lineitem())
        n_pa, n_su, n_or9, n_li9 = q9
        pa = e.generate("part", n_pa, seed=9)
        su = e.generate("supplier", n_su, seed=9)
        ps = e.generate("partsupp", 4 * n_pa, seed=9, n_supp=n_su)
        od9 = e.generate("orders", n_or9, seed=9, columns=("order_key", "order_date"))
        li9 = e.generate("lineitem", n_li9, seed=9,
                         columns=("part_key", "supp_key", "order_key", "ext_price", "discount", "quantity"),
                         n_orders=n_or9, n_parts=n_pa, n_supp=n_su, order_mode=capi.ORDERS_UNIFORM)
        self.q9 = capi.Q9Tables(pa.struct(), su.struct(), ps.struct(), od9.struct(), li9.lineitem())

    def make(self, rng):
        kind = rng.choice((capi.PIPE_Q6, capi.PIPE_Q1, capi.PIPE_Q3, capi.PIPE_Q9))
        r = capi.Request(pipeline=kind)
        if kind == capi.PIPE_Q6:
            r.li = C.pointer(rng.choice(self.scan_structs))
            lo = rng.randrange(0, 2527)
            d = rng.randrange(0, 11)
            r.q6 = capi.Q6Params(lo, lo + rng.randrange(1, 731), d, min(10, d + rng.randrange(0, 4)),
                                 rng.randrange(1, 52))
            out = capi.Q6Result()
            r.q6_out = C.pointer(out)
        elif kind == capi.PIPE_Q1:
            r.li = C.pointer(rng.choice(self.scan_structs))
            r.q1 = capi.Q1Params(rng.randrange(0, 2527), 0)
            out = capi.Q1Result()
            r.q1_out = C.pointer(out)
        elif kind == capi.PIPE_Q3:
            r.q3 = C.pointer(self.q3)
            r.q3p = capi.Q3Params(rng.randrange(0, 5), rng.randrange(0, 2406), rng.randrange(0, 2527), 10,
                                  capi.JOIN_GLOBAL, 0)
            out = capi.Q3Result()
            r.q3_out = C.pointer(out)
        else:
            r.q9 = C.pointer(self.q9)
            out = (capi.Q9Group * 256)()
            r.q9_out = C.cast(out, C.POINTER(capi.Q9Group))
            r.q9_capacity = 256
        return Job(kind, r, out)

    def make_like(self, job):
        """A new job with the same request as `job` and its own result storage."""
        r = capi.Request()
        C.pointer(r)[0] = job.req
        if job.kind == capi.PIPE_Q6:
            out = capi.Q6Result()
            r.q6_out = C.pointer(out)
        elif job.kind == capi.PIPE_Q1:
            out = capi.Q1Result()
            r.q1_out = C.pointer(out)
        elif job.kind == capi.PIPE_Q3:
            out = capi.Q3Result()
            r.q3_out = C.pointer(out)
        else:
            out = (capi.Q9Group * job.req.q9_capacity)()
            r.q9_out = C.cast(out, C.POINTER(capi.Q9Group))
        return Job(job.kind, r, out)

    def jobs(self, n, seed):
        rng = random.Random(seed)
        return [self.make(rng) for _ in range(n)]

    def solo_results(self, jobs):
        """Each request alone through gpudb_batch_run with one request (synchronous)."""
        out = []
        for j in jobs:
            self.engine._check(self.engine.lib.gpudb_batch_run(self.engine.ctx, C.byref(j.req), 1, None, None))
            assert j.req.status == capi.OK, j.req.status
            out.append(j.result())
        return out


def pct(xs, p):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(round(p / 100.0 * (len(xs) - 1))))]


def job_class(job):
    """Pipeline and, for the scans, the table size: "q6_60m", "q1_6m", "q3", "q9"."""
    if job.kind in (capi.PIPE_Q6, capi.PIPE_Q1):
        rows = job.req.li.contents.n_rows
        return "%s_%dm" % ("q6" if job.kind == capi.PIPE_Q6 else "q1", rows // 1_000_000)
    return "q3" if job.kind == capi.PIPE_Q3 else "q9"


def latency_by_class(jobs, lat):
    """Per request class: count, p50 and p99 (ms), and its share of the requests above the
    run's p99 (which classes make the tail)."""
    cut = pct(lat, 99)
    groups = {}
    for j, x in zip(jobs, lat):
        groups.setdefault(job_class(j), []).append(x)
    tail = sum(1 for x in lat if x > cut) or 1
    return {c: {"n": len(v), "p50_ms": pct(v, 50), "p99_ms": pct(v, 99),
                "tail_share": sum(1 for x in v if x > cut) / tail} for c, v in sorted(groups.items())}


def open_loop(server, jobs, rate, seed):
    """Submits jobs at Poisson arrival times (rate per second); returns latencies (ms) and wall time."""
    rng = random.Random(seed)
    tickets = [None] * len(jobs)
    lat = [None] * len(jobs)
    status = [None] * len(jobs)
    t0 = time.perf_counter()

    def collect():
        for i in range(len(jobs)):
            while tickets[i] is None:
                time.sleep(0.0001)
            status[i], lat[i] = server.wait(tickets[i])

    th = threading.Thread(target=collect)
    th.start()
    t_next = t0
    for i, j in enumerate(jobs):
        t_next += rng.expovariate(rate)
        while True:
            now = time.perf_counter()
            if now >= t_next:
                break
            time.sleep(min(t_next - now, 0.0005))
        tickets[i] = server.submit(j.req)
    th.join()
    wall = time.perf_counter() - t0
    return lat, status, wall


def run_mode(engine, wl, name, lanes, max_batch, rate, n, seed, check=None, heavy_lanes=0):
    jobs = wl.jobs(n, seed)
    srv = Server(lanes=lanes, max_batch=max_batch, heavy_lanes=heavy_lanes if lanes > 1 else 0)
    try:
        # one batch of the largest size on every lane sizes the lanes' scratch before timing
        srv.warmup(wl.jobs(max(max_batch, 16), seed + 7))
        lat, status, wall = open_loop(srv, jobs, rate, seed + 1)
        st = srv.stats()
    finally:
        srv.close()
    ok = all(s == capi.OK for s in status)
    exact = None
    if check is not None:
        exact = all(j.result() == w for j, w in zip(jobs, check))
    return {"mode": name, "lanes": lanes, "heavy_lanes": heavy_lanes if lanes > 1 else 0, "max_batch": max_batch,
            "offered_qps": rate, "requests": n,
            "achieved_qps": n / wall, "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "mean_batch":
            st["completed"] / max(1, st["batches"]), "all_ok": ok, "bit_exact_vs_solo": exact,
            "by_class": latency_by_class(jobs, lat)}


# Lanes of the served form: at 22K queries/s of the mixed stream, 1/2/3/4/8 lanes gave p99
# 5.2/4.4/4.7/5-21/8.0 ms on one B200 (two lanes overlap two batches on the GPU; more lanes
# contend for it, one leaves it idle between batches).
DEFAULT_LANES = 2
# Lanes of those that take only the scans of large tables (gpudb_serve_config.heavy_lanes).
DEFAULT_HEAVY_LANES = 0


def compare(eng, seconds=1.0, lanes=DEFAULT_LANES, max_batch=64, loads=(0.5, 0.85), factor=3.0, seed=11,
            heavy_lanes=DEFAULT_HEAVY_LANES):
    """Served form against the plain one-query-per-launch form on the same mixed stream.

    1. plain saturation: requests submitted back to back (closed loop), queries/s;
    2. at each of `loads` x that rate (Poisson arrivals), the plain and the served form on
       the same requests: queries/s, p50, p99;
    3. the served form at `factor` x the highest of those rates: queries/s, p50, p99 (the
       ">= 3x the queries/s at equal or lower p99" comparison is this against the plain form
       at the highest matched rate);
    4. served saturation (closed loop).
    Every result of every run is compared with the same request run alone."""
    wl = Workload(eng)
    out = {"lanes": lanes, "heavy_lanes": heavy_lanes, "max_batch": max_batch, "seconds_per_rate": seconds,
           "workload": "Q6/Q1 over lineitem at 1M/6M/60M rows, Q3 at config-2 1x, Q9 at 6M fact rows; "
                       "random pipeline and constants per request, Poisson arrivals"}
    solos = {}

    def run(name, ln, mb, rate, n, sd):
        if (n, sd) not in solos:
            solos[(n, sd)] = wl.solo_results(wl.jobs(n, sd))
        return _run_checked(eng, wl, name, ln, mb, rate, n, sd, wl.jobs(n, sd), solos[(n, sd)], heavy_lanes)

    runs = []
    sat = run("plain", 1, 1, 1e9, 3000, seed)
    out["plain_saturation"] = sat
    runs.append(sat)
    matched = []
    for i, ld in enumerate(loads):
        rate = ld * sat["achieved_qps"]
        n = max(500, int(rate * seconds))
        pr = run("plain", 1, 1, rate, n, seed + 1 + i)
        sr = run("served", lanes, max_batch, rate, n, seed + 1 + i)
        matched.append({"load_of_plain_saturation": ld, "offered_qps": rate, "plain": pr, "served": sr})
        runs += [pr, sr]
    out["matched"] = matched
    top = matched[-1]
    n3 = max(500, int(factor * top["offered_qps"] * seconds))
    s3 = run("served", lanes, max_batch, factor * top["offered_qps"], n3, seed + 10)
    out["served_at_%gx" % factor] = s3
    ssat = run("served", lanes, max_batch, 1e9, max(4000, n3), seed + 11)
    out["served_saturation"] = ssat
    runs += [s3, ssat]
    p = top["plain"]
    out["headline"] = {"plain_qps": p["achieved_qps"], "plain_p99_ms": p["p99_ms"], "served_qps": s3["achieved_qps"],
                       "served_p99_ms": s3["p99_ms"], "qps_ratio": s3["achieved_qps"] / p["achieved_qps"],
                       "p99_ratio": s3["p99_ms"] / p["p99_ms"]}
    out["bit_exact"] = all(r["bit_exact_vs_solo"] and r["all_ok"] for r in runs)
    return out


def _run_checked(eng, wl, name, lanes, max_batch, rate, n, seed, jobs, solo, heavy_lanes=0):
    srv = Server(lanes=lanes, max_batch=max_batch, heavy_lanes=heavy_lanes if lanes > 1 else 0)
    try:
        srv.warmup(wl.jobs(max(max_batch, 16), seed + 7))
        lat, status, wall = open_loop(srv, jobs, rate, seed + 1)
        st = srv.stats()
    finally:
        srv.close()
    return {"mode": name, "offered_qps": None if rate >= 1e9 else rate, "requests": n, "achieved_qps": n / wall,
            "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "mean_batch": st["completed"] / max(1, st["batches"]),
            "all_ok": all(x == capi.OK for x in status),
            "bit_exact_vs_solo": all(j.result() == w for j, w in zip(jobs, solo)),
            "by_class": latency_by_class(jobs, lat)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", type=float, nargs="*", default=[1000, 2000, 4000, 8000, 16000, 32000])
    ap.add_argument("--seconds", type=float, default=2.0)
    ap.add_argument("--lanes", type=int, default=DEFAULT_LANES)
    ap.add_argument("--heavy-lanes", type=int, default=DEFAULT_HEAVY_LANES,
                    help="lanes that take only the scans of tables over 2^24 rows (0: every lane takes all)")
    ap.add_argument("--max-batch", type=int, default=64)
    ap.add_argument("--modes", nargs="*", default=["plain", "served"], choices=["plain", "served"])
    ap.add_argument("--compare", action="store_true",
                    help="the served-vs-plain comparison of bench.py (matched rates, 3x, saturation)")
    a = ap.parse_args(argv)
    eng = Engine(0)
    if a.compare:
        print(json.dumps(compare(eng, seconds=a.seconds, lanes=a.lanes, max_batch=a.max_batch,
                                 heavy_lanes=a.heavy_lanes)), flush=True)
        eng.close()
        return 0
    wl = Workload(eng)
    for rate in a.rates:
        n = max(200, int(rate * a.seconds))
        seed = int(rate)
        solo = wl.solo_results(wl.jobs(n, seed))
        for name, lanes, mb in (("plain", 1, 1), ("served", a.lanes, a.max_batch)):
            if name not in a.modes:
                continue
            res = run_mode(eng, wl, name, lanes, mb, rate, n, seed, check=solo, heavy_lanes=a.heavy_lanes)
            print(json.dumps(res), flush=True)
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
