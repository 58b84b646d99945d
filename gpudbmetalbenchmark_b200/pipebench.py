"""Per-pipeline throughput of every hot-path pipeline on one GPU, against the HBM roofline.

    python -m gpudbmetalbenchmark_b200.pipebench [--only NAME ...] [--reps N] [--stream600m]

Prints one JSON line per measurement: pipeline, configuration, rows, median device time
(CUDA events on the launching stream, recorded by the library around the pipeline's
kernels), rows/s, algorithmic GB/s and the fraction of the measured HBM copy peak. Inputs
are generated on the device (seeded); every input is larger than L2 except where noted.
Streamed cases keep the fact table in pinned host memory and are bounded by the host link.
"""
import argparse
import json
import os
import statistics
import sys

from . import capi
from .engine import Q12_LI_COLS, Engine, Q1_COLS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def timed(fn, reps):
    fn(None)   # warm-up (and scratch allocation)
    ts = []
    for _ in range(reps):
        t = capi.Timing()
        fn(t)
        ts.append(t)
    return statistics.median(t.gpu_ms for t in ts), ts[-1]


def record(name, config, rows, ms, alg_bytes, extra=None):
    """One measurement: device ms, rows/s, algorithmic GB/s and its fraction of the HBM
    peak (`peak_kind` says whether that peak is the measured one or the fallback)."""
    pk, kind = peak()
    gbs = alg_bytes / (ms * 1e-3) / 1e9
    line = {"pipeline": name, "config": config, "rows": rows, "ms": round(ms, 4),
            "rows_per_s": rows / (ms * 1e-3), "algorithmic_bytes": alg_bytes, "gbs_algorithmic": round(gbs, 1),
            "frac": round(gbs / pk, 3), "peak_gbs": pk, "peak_kind": kind}
    if extra:
        line.update(extra)
    return line


def emit(name, config, rows, ms, alg_bytes, extra=None):
    line = record(name, config, rows, ms, alg_bytes, extra)
    print(json.dumps(line), flush=True)
    return line


Q3_MODES = ((capi.JOIN_DIRECT, "direct"), (capi.JOIN_GLOBAL, "global"), (capi.JOIN_RADIX, "radix"))


def q3_case(eng, n_cu, n_or, n_li, reps, label, out=emit):
    """Q3 join + top-10 on the config-2 tables (1x: 150K/1.5M/6M rows) in every join mode;
    returns {mode: record}."""
    cu = eng.generate("customer", n_cu, seed=42)
    od = eng.generate("orders", n_or, seed=42, n_cust=n_cu)
    li = eng.generate("lineitem", n_li, seed=42, columns=("order_key", "ship_date", "ext_price", "discount"),
                      n_orders=n_or, order_mode=capi.ORDERS_CLUSTERED)
    alg = n_cu * 5 + n_or * 12 + n_li * 20
    res = {}
    for mode, mname in Q3_MODES:
        ms, t = timed(lambda tm: eng.q3(cu, od, li, join_mode=mode, timing=tm), reps)
        res[mname] = out("q3_join_topk", "%s, %s table" % (label, mname), n_li, ms, alg, {"kernels": t.kernels})
    for x in (cu, od, li):
        eng.free(x)
    return res


def scan_case(eng, rows, reps, out=emit):
    """Q6 and Q1 over a device-resident lineitem table of `rows` rows: (q6, q1) records.
    `ms` is the median over calls issued back to back; `sync_ms` the median over synchronous
    calls, each starting on an idle GPU."""
    t = eng.generate("lineitem", rows, seed=42, columns=Q1_COLS)
    recs = []
    for name, fn, mk, bpr in (("q6_sum", eng.q6, capi.Q6Result, 20), ("q1_group6", eng.q1, capi.Q1Result, 26)):
        sync_ms, tl = timed(lambda tm: fn(t, timing=tm), reps)
        fn(t)
        ts = [capi.Timing() for _ in range(reps)]
        outs = [mk() for _ in range(reps)]
        for tm, o in zip(ts, outs):
            fn(t, timing=tm, async_=True, out=o)
        eng.sync()
        assert all(bytes(o) == bytes(outs[0]) for o in outs)
        ms = statistics.median(x.gpu_ms for x in ts)
        if name == "q6_sum":
            cfg = "1a" if rows > 6e6 else "1a at 6M"
            extra = {"note": "6M rows = 120 MB, inside L2" if rows == 6_000_000 else ""}
        else:
            cfg = "1b" if rows > 6e6 else "0"
            extra = {"note": "6M rows = 156 MB" if rows == 6_000_000 else "", "kernels": tl.kernels}
        extra.update({"sync_ms": round(sync_ms, 4), "timed": "calls back to back"})
        recs.append(out(name, "config %s" % cfg, rows, ms, bpr * rows, extra))
    eng.free(t)
    return recs[0], recs[1]


def q9_case(eng, reps, stream600m=False, out=emit):
    """Q9 star join on the config-3 tables at 60M fact rows (HBM-resident) and, with
    stream600m, at 600M fact rows streamed from pinned host memory in 64M-row chunks."""
    res = {}
    pa, su, ps, od = q9_tables(eng, 2_000_000, 100_000, 15_000_000)
    cols = ("part_key", "supp_key", "order_key", "ext_price", "discount", "quantity")
    li = eng.generate("lineitem", 60_000_000, seed=42, columns=cols, n_orders=15_000_000, n_parts=2_000_000,
                      n_supp=100_000, order_mode=capi.ORDERS_UNIFORM)
    ms, t = timed(lambda tm: eng.q9(pa, su, ps, od, li, timing=tm), reps)
    res["resident"] = out("q9_star", "config 3 (HBM-resident)", 60_000_000, ms,
                          60_000_000 * 28 + 8_000_000 * 16 + 15_000_000 * 8 + 2_000_000 + 100_000, {"kernels": t.kernels})
    eng.free(li)
    if stream600m:
        rows = 600_000_000
        lh = eng.generate("lineitem", rows, seed=42, columns=cols, n_orders=15_000_000, n_parts=2_000_000,
                          n_supp=100_000, order_mode=capi.ORDERS_UNIFORM, location=capi.MEM_HOST)
        ms, t = timed(lambda tm: eng.q9(pa, su, ps, od, lh, chunk_rows=64 << 20, timing=tm), max(2, reps // 10))
        res["streamed"] = out("q9_star", "config 3 streamed (600M rows, 64M-row chunks, pinned host)", rows, ms,
                              rows * 28, {"chunks": t.chunks, "h2d_gbs": t.h2d_bytes / (ms * 1e-3) / 1e9,
                                          "bound": "host link", "kernels": t.kernels})
        eng.free(lh)
    for x in (pa, su, ps, od):
        eng.free(x)
    return res


def join_count_case(eng, reps, out=emit):
    """Join microbenchmark: 15M-key build x 60M-key probe, global table, radix partitions and
    the direct bitmap over the build keys' span; every mode's count must agree."""
    b = eng.generate("orders", 15_000_000, seed=42, columns=("order_key",))
    p = eng.generate("lineitem", 60_000_000, seed=42, columns=("order_key",), n_orders=15_000_000,
                     order_mode=capi.ORDERS_CLUSTERED)
    res = {}
    counts = {}
    for mode, mname in ((capi.JOIN_GLOBAL, "global"), (capi.JOIN_RADIX, "radix"), (capi.JOIN_DIRECT, "direct")):
        ms, t = timed(lambda tm: eng.hash_join_count(b.ptr("order_key"), 15_000_000, p.ptr("order_key"),
                                                     60_000_000, mode, timing=tm), reps)
        counts[mname] = eng.hash_join_count(b.ptr("order_key"), 15_000_000, p.ptr("order_key"), 60_000_000, mode)
        res[mname] = out("hash_join_count", "15M build x 60M probe, %s" % mname, 60_000_000, ms, 75_000_000 * 4,
                         {"kernels": t.kernels, "matches": counts[mname]})
    for r in res.values():   # (the tests check each mode against the oracle; here they must agree)
        if isinstance(r, dict):
            r["modes_agree"] = len(set(counts.values())) == 1
    eng.free(b)
    eng.free(p)
    return res


def q9_tables(eng, n_pa, n_su, n_or):
    pa = eng.generate("part", n_pa, seed=42)
    su = eng.generate("supplier", n_su, seed=42)
    ps = eng.generate("partsupp", 4 * n_pa, seed=42, n_supp=n_su)
    od = eng.generate("orders", n_or, seed=42, columns=("order_key", "order_date"))
    return pa, su, ps, od


def lineitem_text(eng, n, seed=42):
    """n lineitem rows of the seeded generator as dbgen-style text (numpy string ops)."""
    import numpy as np
    cols = ("order_key", "part_key", "supp_key", "quantity", "ext_price", "discount", "tax", "flag", "status",
            "ship_date")
    t = eng.generate("lineitem", n, seed=seed, columns=cols, n_orders=max(1, n // 4), n_parts=200_000, n_supp=10_000,
                     order_mode=capi.ORDERS_CLUSTERED)
    c = {k: t.to_numpy(k) for k in cols}
    eng.free(t)
    days = np.datetime64("1992-01-01") + c["ship_date"].astype("timedelta64[D]")
    date = np.datetime_as_string(days, unit="D").astype(object)
    money = (c["ext_price"] // 100).astype(str).astype(object) + "." + \
        np.char.zfill((c["ext_price"] % 100).astype(str), 2).astype(object)
    frac = lambda a: "0." + np.char.zfill(a.astype(str), 2).astype(object)  # noqa: E731
    f = lambda a: a.astype(str).astype(object)  # noqa: E731
    rows = (f(c["order_key"]) + "|" + f(c["part_key"]) + "|" + f(c["supp_key"]) + "|1|" + f(c["quantity"]) + "|" +
            money + "|" + frac(c["discount"]) + "|" + frac(c["tax"]) + "|" +
            np.array(list("ANR"), dtype=object)[c["flag"]] + "|" + np.array(list("FO"), dtype=object)[c["status"]] +
            "|" + date + "|" + date + "|" + date + "|DELIVER IN PERSON|TRUCK|a lineitem row|\n")
    return "".join(rows.tolist()).encode()


def tbl_cases(eng, reps):
    import ctypes as C
    import numpy as np
    from .engine import TABLE_COLS
    n = 6_000_000
    text = lineitem_text(eng, n)
    buf = np.frombuffer(text, dtype=np.uint8)
    code, names = capi.TBL_COLUMNS["lineitem"]
    cols = (C.c_void_p * capi.TBL_MAX_COLS)()
    ptrs = []
    for i, name in enumerate(names):
        ptrs.append(eng.device_array(n * eng.lib.gpudb_column_width(TABLE_COLS["lineitem"][name])))
        cols[i] = ptrs[-1]
    dev = eng.device_array(len(text) + 16)
    eng._check(eng.lib.gpudb_copy(eng.ctx, dev, buf.ctypes.data, len(text)))
    got = C.c_uint64()
    for where, src, loc in (("pageable host text, H2D copy inside the call", buf.ctypes.data, capi.MEM_HOST),
                            ("device-resident text", dev, capi.MEM_DEVICE)):
        def run(tm):
            eng._check(eng.lib.gpudb_tbl_parse(eng.ctx, code, src, len(text), loc, cols, n, C.byref(got), None,
                                               C.byref(tm) if tm is not None else None))
        ms, t = timed(run, max(3, reps // 4))
        emit("tbl_parse", "lineitem, %d rows, %.0f MB of text, %s" % (n, len(text) / 1e6, where), n, ms, len(text),
             {"kernels": t.kernels, "text_gb_per_s": round(len(text) / (ms * 1e-3) / 1e9, 1)})
    eng.device_free(dev)
    for p in ptrs:
        eng.device_free(p)


def batch_cases(eng, reps):
    """Batched forms beside the same requests run one by one (gpudb_batch_run with one
    request each): the device time of the whole batch and the per-request share."""
    import ctypes as C
    import random
    from .serve import Job, Workload
    wl = Workload(eng)
    rng = random.Random(5)

    def run(jobs, tm):
        arr = (capi.Request * len(jobs))(*[j.req for j in jobs])
        eng._check(eng.lib.gpudb_batch_run(eng.ctx, arr, len(jobs), tm, None))

    def alone(jobs):
        # one request per call; the sum of the calls' device times
        total = []
        for _ in range(3):
            s = 0.0
            for j in jobs:
                t = capi.Timing()
                if j.kind == capi.PIPE_Q3:
                    eng._check(eng.lib.gpudb_q3_join_topk(eng.ctx, C.byref(wl.q3.cu), C.byref(wl.q3.od), C.byref(wl.q3.li),
                                                          C.byref(j.req.q3p), j.req.q3_out, C.byref(t), None))
                elif j.kind == capi.PIPE_Q6:
                    eng._check(eng.lib.gpudb_q6_sum(eng.ctx, j.req.li, C.byref(j.req.q6), j.req.q6_out, C.byref(t), None))
                elif j.kind == capi.PIPE_Q1:
                    eng._check(eng.lib.gpudb_q1_group6(eng.ctx, j.req.li, C.byref(j.req.q1), j.req.q1_out, C.byref(t),
                                                       None))
                s += t.gpu_ms
            total.append(s)
        return statistics.median(total)

    # 8 Q3 requests over the config-2 tables (1x) with random segment/date bounds
    q3 = []
    for _ in range(8):
        r = capi.Request(pipeline=capi.PIPE_Q3)
        r.q3 = C.pointer(wl.q3)
        r.q3p = capi.Q3Params(rng.randrange(0, 5), rng.randrange(0, 2406), rng.randrange(0, 2527), 10,
                              capi.JOIN_GLOBAL, 0)
        out = capi.Q3Result()
        r.q3_out = C.pointer(out)
        q3.append(Job(capi.PIPE_Q3, r, out))
    ms, t = timed(lambda tm: run(q3, tm), reps)
    emit("q3_batched", "8 requests, config 2 (1x), one launch per stage", 8 * 6_000_000, ms,
         8 * (150_000 * 5 + 1_500_000 * 12 + 6_000_000 * 20),
         {"kernels": t.kernels, "ms_per_request": round(ms / 8, 4), "ms_alone_sum": round(alone(q3), 4)})
    # shared scans over the 60M-row table: 8 Q6 + 2 Q1 requests in one pass each
    big = wl.scan_structs[-1]
    scans = []
    for i in range(10):
        r = capi.Request(pipeline=capi.PIPE_Q6 if i < 8 else capi.PIPE_Q1)
        r.li = C.pointer(big)
        if i < 8:
            lo = rng.randrange(0, 2527)
            r.q6 = capi.Q6Params(lo, lo + rng.randrange(1, 731), 2, 8, rng.randrange(1, 52))
            out = capi.Q6Result()
            r.q6_out = C.pointer(out)
        else:
            r.q1 = capi.Q1Params(rng.randrange(1500, 2527), 0)
            out = capi.Q1Result()
            r.q1_out = C.pointer(out)
        scans.append(Job(r.pipeline, r, out))
    ms, t = timed(lambda tm: run(scans, tm), reps)
    emit("shared_scans", "8 Q6 + 2 Q1 over 60M rows, one pass per kind", 10 * 60_000_000, ms,
         60_000_000 * 20 + 60_000_000 * 26, {"kernels": t.kernels, "ms_per_request": round(ms / 10, 4),
                                             "ms_alone_sum": round(alone(scans), 4)})
    # 8 identical Q9 requests at serving scale (6M fact rows): coalesced into one execution
    q9 = []
    for _ in range(8):
        r = capi.Request(pipeline=capi.PIPE_Q9)
        r.q9 = C.pointer(wl.q9)
        out = (capi.Q9Group * 256)()
        r.q9_out = C.cast(out, C.POINTER(capi.Q9Group))
        r.q9_capacity = 256
        q9.append(Job(capi.PIPE_Q9, r, out))
    ms, t = timed(lambda tm: run(q9, tm), reps)
    one, _ = timed(lambda tm: eng._check(eng.lib.gpudb_batch_run(eng.ctx, C.byref(q9[0].req), 1, tm, None)), reps)
    emit("q9_coalesced", "8 identical requests, 6M fact rows", 8 * 6_000_000, ms, 8 * 6_000_000 * 28,
         {"kernels": t.kernels, "ms_per_request": round(ms / 8, 4), "ms_alone": round(one, 4)})


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--stream600m", action="store_true", help="config 3 streamed at 600M fact rows (16.8 GB pinned)")
    ap.add_argument("--opt", action="append", default=[], metavar="NAME=VALUE",
                    help="context option before measuring, e.g. radix_shape=1 (names: capi.OPT_NAMES)")
    a = ap.parse_args(argv)
    want = set(a.only) if a.only else None
    eng = Engine(0)
    for o in a.opt:
        name, value = o.split("=")
        ids = {v: k for k, v in capi.OPT_NAMES.items()}
        eng.set_option(ids[name], int(value))
        print(json.dumps({"option": name, "value": int(value)}), flush=True)
    on = lambda name: want is None or name in want  # noqa: E731

    if on("scans"):
        for rows in (6_000_000, 60_000_000):
            scan_case(eng, rows, a.reps)
    if on("q3"):
        q3_case(eng, 150_000, 1_500_000, 6_000_000, a.reps, "config 2 (1x)")
        q3_case(eng, 1_500_000, 15_000_000, 60_000_000, max(3, a.reps // 4), "config 2 (10x)")
    if on("q4q12"):
        for n_or, n_li, label in ((1_500_000, 6_000_000, "SF-1 sizes"), (15_000_000, 60_000_000, "SF-10 sizes")):
            od = eng.generate("orders", n_or, seed=42, columns=("order_key", "order_date", "priority"))
            li = eng.generate("lineitem", n_li, seed=42, columns=Q12_LI_COLS, n_orders=n_or,
                              order_mode=capi.ORDERS_CLUSTERED)
            ms, t = timed(lambda tm: eng.q4(od, li, timing=tm), a.reps)
            emit("q4_priority", label, n_li, ms, n_li * 12 + n_or * 9, {"kernels": t.kernels})
            ms, t = timed(lambda tm: eng.q12(od, li, timing=tm), a.reps)
            emit("q12_shipmode", label, n_li, ms, n_li * 17 + n_or * 5, {"kernels": t.kernels})
            eng.free(li)
            eng.free(od)
    if on("q5"):
        for n_cu, n_su, n_or, n_li, label in ((150_000, 10_000, 1_500_000, 6_000_000, "SF-1 sizes"),
                                              (1_500_000, 100_000, 15_000_000, 60_000_000, "SF-10 sizes")):
            cu = eng.generate("customer", n_cu, seed=42, columns=("cust_key", "nation"))
            su = eng.generate("supplier", n_su, seed=42)
            od = eng.generate("orders", n_or, seed=42, columns=("order_key", "cust_key", "order_date"), n_cust=n_cu)
            li = eng.generate("lineitem", n_li, seed=42, columns=("order_key", "supp_key", "ext_price", "discount"),
                              n_orders=n_or, n_parts=20 * n_su, n_supp=n_su, order_mode=capi.ORDERS_CLUSTERED)
            ms, t = timed(lambda tm: eng.q5(cu, su, od, li, timing=tm), a.reps)
            emit("q5_local_supplier", label, n_li, ms, n_li * 8 + n_or * 12 + n_cu * 5 + n_su * 5,
                 {"kernels": t.kernels})
            for x in (li, od, su, cu):
                eng.free(x)
    if on("q7q8"):
        for n_cu, n_su, n_pa, n_or, n_li, label in ((150_000, 10_000, 200_000, 1_500_000, 6_000_000, "SF-1 sizes"),
                                                    (1_500_000, 100_000, 2_000_000, 15_000_000, 60_000_000,
                                                     "SF-10 sizes")):
            cu = eng.generate("customer", n_cu, seed=42, columns=("cust_key", "nation"))
            su = eng.generate("supplier", n_su, seed=42)
            pa = eng.generate("part", n_pa, seed=42, columns=("part_key", "type"))
            od = eng.generate("orders", n_or, seed=42, columns=("order_key", "cust_key", "order_date"), n_cust=n_cu)
            li = eng.generate("lineitem", n_li, seed=42,
                              columns=("order_key", "part_key", "supp_key", "ship_date", "ext_price", "discount"),
                              n_orders=n_or, n_parts=n_pa, n_supp=n_su, order_mode=capi.ORDERS_CLUSTERED)
            ms, t = timed(lambda tm: eng.q7(cu, su, od, li, timing=tm), a.reps)
            emit("q7_volume_shipping", label, n_li, ms, n_li * 12 + n_or * 8 + n_cu * 5 + n_su * 5,
                 {"kernels": t.kernels})
            ms, t = timed(lambda tm: eng.q8(cu, su, pa, od, li, timing=tm), a.reps)
            emit("q8_market_share", label, n_li, ms, n_li * 4 + n_or * 12 + n_cu * 5 + n_su * 5 + n_pa * 5,
                 {"kernels": t.kernels})
            for x in (li, od, pa, su, cu):
                eng.free(x)
    if on("q10"):
        for n_cu, n_or, n_li, label in ((150_000, 1_500_000, 6_000_000, "SF-1 sizes"),
                                        (1_500_000, 15_000_000, 60_000_000, "SF-10 sizes")):
            cu = eng.generate("customer", n_cu, seed=42, columns=("cust_key",))
            od = eng.generate("orders", n_or, seed=42, columns=("order_key", "cust_key", "order_date"), n_cust=n_cu)
            li = eng.generate("lineitem", n_li, seed=42, columns=("order_key", "flag", "ext_price", "discount"),
                              n_orders=n_or, order_mode=capi.ORDERS_CLUSTERED)
            ms, t = timed(lambda tm: eng.q10(cu, od, li, timing=tm), a.reps)
            emit("q10_returned", label, n_li, ms, n_li * 5 + n_or * 12 + n_cu * 4, {"kernels": t.kernels})
            for x in (li, od, cu):
                eng.free(x)
    if on("q13"):
        for n_cu, n_or, label in ((150_000, 1_500_000, "SF-1 sizes"), (1_500_000, 15_000_000, "SF-10 sizes")):
            cu = eng.generate("customer", n_cu, seed=42, columns=("cust_key",))
            od = eng.generate("orders", n_or, seed=42, columns=("cust_key", "comment"), n_cust=n_cu)
            ms, t = timed(lambda tm: eng.q13(cu, od, timing=tm), a.reps)
            emit("q13_distribution", label, n_or, ms, n_or * (4 + capi.COMMENT_WIDTH) + n_cu * 8, {"kernels": t.kernels})
            eng.free(od)
            eng.free(cu)
    if on("q9"):
        q9_case(eng, a.reps, a.stream600m)
    if on("batch"):
        batch_cases(eng, a.reps)
    if on("tbl"):
        tbl_cases(eng, a.reps)
    if on("micro"):
        rows = 60_000_000
        t = eng.generate("lineitem", rows, seed=42, columns=("ship_date", "quantity"))
        bits = eng.device_array((rows + 31) // 32 * 4)
        ms, _ = timed(lambda tm: eng.select_lt(t.ptr("ship_date"), rows, 1000, bits, timing=tm), a.reps)
        emit("select_lt", "selection, bitmask output", rows, ms, rows * 4 + rows // 8)
        ms, _ = timed(lambda tm: eng.sum_i32(t.ptr("quantity"), rows, timing=tm), a.reps)
        emit("sum_i32", "aggregation", rows, ms, rows * 4)
        eng.device_free(bits)
        eng.free(t)
        join_count_case(eng, max(3, a.reps // 4))
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
