"""Autotuner front end: tunes every pipeline on the benchmark configurations and keeps the
choices in a cache file keyed by the device name.

    python -m gpudbmetalbenchmark_b200.autotune [--cache PATH] [--reps N] [--only q1 q6 q3 q9]

For each pipeline and configuration it prints one JSON line: the setting chosen, the
device time with it and with the default setting (median of N runs, CUDA events on the
launching stream), and for the scans the algorithmic GB/s against the measured HBM peak.
The chosen settings are written to the cache (gpudb_tune_save); Engine.tune_load(path) or
gpudb_tune_load applies them to a new context. Every candidate's result is checked against
the default setting's result inside the library, so a setting that changes a result is
never chosen.
"""
import argparse
import ctypes as C
import json
import os
import sys

from . import capi
from .engine import Engine, Q1_COLS
from .pipebench import peak


def scan_request(kind, table):
    r = capi.Request(pipeline=kind)
    r.li = C.pointer(table)
    if kind == capi.PIPE_Q6:
        r.q6 = capi.Q6Params(365, 730, 5, 7, 24)
    else:
        r.q1 = capi.Q1Params(2436, 0)
    return r


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cache", default="gpudb_tune.txt")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--only", nargs="*")
    a = ap.parse_args(argv)
    want = set(a.only) if a.only else None
    on = lambda name: want is None or name in want  # noqa: E731
    pk, kind = peak()
    eng = Engine(0)
    keep = []

    def report(name, config, res, alg_bytes=None):
        line = {"pipeline": name, "config": config}
        line.update(res)
        if alg_bytes:
            for tag in ("best", "default"):
                gbs = alg_bytes / (res[tag + "_ms"] * 1e-3) / 1e9
                line[tag + "_gbs"] = round(gbs, 1)
                line[tag + "_frac_of_%s_peak" % kind] = round(gbs / pk, 3)
        print(json.dumps(line), flush=True)

    if on("q1") or on("q6"):
        for rows, label in ((60_000_000, "config 1, 60M rows"), (6_000_000, "config 0, 6M rows")):
            t = eng.generate("lineitem", rows, seed=42, columns=Q1_COLS)
            s = t.lineitem()
            keep.append(s)
            if on("q6"):
                report("q6_sum", label, eng.autotune(scan_request(capi.PIPE_Q6, s), a.reps), 20 * rows)
            if on("q1"):
                report("q1_group6", label, eng.autotune(scan_request(capi.PIPE_Q1, s), a.reps), 26 * rows)
            eng.free(t)
    if on("q3"):
        for scale, (n_cu, n_or, n_li) in (("1x", (150_000, 1_500_000, 6_000_000)),
                                          ("10x", (1_500_000, 15_000_000, 60_000_000))):
            cu = eng.generate("customer", n_cu, seed=42)
            od = eng.generate("orders", n_or, seed=42, n_cust=n_cu)
            li = eng.generate("lineitem", n_li, seed=42, columns=("order_key", "ship_date", "ext_price", "discount"),
                              n_orders=n_or, order_mode=capi.ORDERS_CLUSTERED)
            tables = capi.Q3Tables(cu.struct(), od.struct(), li.lineitem())
            for mode, mname in ((capi.JOIN_GLOBAL, "global"), (capi.JOIN_RADIX, "radix")):
                r = capi.Request(pipeline=capi.PIPE_Q3)
                r.q3 = C.pointer(tables)
                r.q3p = capi.Q3Params(1, 1170, 1170, 10, mode, 0)
                report("q3_join_topk", "config 2 (%s), %s" % (scale, mname), eng.autotune(r, max(3, a.reps // 2)))
            for x in (cu, od, li):
                eng.free(x)
    if on("q9"):
        pa = eng.generate("part", 2_000_000, seed=42)
        su = eng.generate("supplier", 100_000, seed=42)
        ps = eng.generate("partsupp", 8_000_000, seed=42, n_supp=100_000)
        od = eng.generate("orders", 15_000_000, seed=42, columns=("order_key", "order_date"))
        li = eng.generate("lineitem", 60_000_000, seed=42,
                          columns=("part_key", "supp_key", "order_key", "ext_price", "discount", "quantity"),
                          n_orders=15_000_000, n_parts=2_000_000, n_supp=100_000, order_mode=capi.ORDERS_UNIFORM)
        tables = capi.Q9Tables(pa.struct(), su.struct(), ps.struct(), od.struct(), li.lineitem())
        r = capi.Request(pipeline=capi.PIPE_Q9)
        r.q9 = C.pointer(tables)
        report("q9_star", "config 3, 60M fact rows", eng.autotune(r, max(3, a.reps // 2)))
        for x in (pa, su, ps, od, li):
            eng.free(x)
    eng.tune_save(a.cache)
    print(json.dumps({"cache": os.path.abspath(a.cache)}), flush=True)
    eng.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
