"""The `gpudb <size> <pipeline>` command line (C++ drivers over the C ABI): each pipeline's
printed exact result equals the oracle's, and the output keeps the reference's header and
timing lines (the lines scripts/benchmark_gpu.sh greps)."""
import os
import re
import subprocess
from decimal import Decimal

import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "gpudbmetalbenchmark_b200", "lib", "gpudb")
TIMING = ["CPU Parsing (.tbl):", "GPU Execution:", "CPU Post Process:", "Total Execution:"]


def run(*args):
    r = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout


def scaled(v, digits):
    return int(Decimal(v) * (10 ** digits))


def timing_ok(out, q, rows):
    assert re.search(r"^%s \| %d rows" % (q, rows), out, re.M), out
    for t in TIMING:
        assert t in out


def test_cli_q6_and_q1(orc):
    n = 60_000
    li = orc.lineitem(n, seed=42)
    out = run("sf1", "q6", "--scale", "0.01")
    rev = scaled(re.search(r"Total Revenue: \$(\S+)", out).group(1), 4)
    matched = int(re.search(r"Rows matched: (\d+)", out).group(1))
    assert (rev, matched) == orc.q6(li)
    timing_ok(out, "Q6", n)
    out = run("sf1", "q1", "--scale", "0.01")
    want = orc.q1(li)
    rows = re.findall(r"^\|\s+([ANR])\s+\|\s+([FO])\s+\|\s+(\d+)\s+\|\s+(\S+)\s+\|\s+(\S+)\s+\|\s+(\S+)\s+\|.*\|\s+(\d+)\s+\|$",
                      out, re.M)
    assert len(rows) == len(want)
    for f, s, qty, base, disc, charge, cnt in rows:
        g = want[("ANR".index(f), "FO".index(s))]
        assert (int(qty), scaled(base, 2), scaled(disc, 4), scaled(charge, 6), int(cnt)) == \
            (g["sum_qty"], g["sum_base_price"], g["sum_disc_price"], g["sum_charge"], g["count"])
    timing_ok(out, "Q1", n)


def test_cli_q3_every_join_mode(orc):
    cu, od, li = orc.q3_tables(1500, 15000, 60000, 42)
    top, groups = orc.q3(cu, od, li)
    out = run("sf1", "q3", "--scale", "0.01")
    assert "using the direct map join" in out
    blocks = out.split("TPC-H Q3 Results")[1:]
    assert len(blocks) == 3
    assert [re.match(r" \(Top 10, ([a-z ]+) join\)", b).group(1) for b in blocks] == \
        ["direct map", "global hash table", "radix partitioned"]
    for b in blocks:
        rows = re.findall(r"^\|\s+(\d+) \| \$\s*(\S+) \|\s+(\d+) \|", b, re.M)
        assert [(int(k), int(d), scaled(r, 4)) for k, r, d in rows] == top
        assert int(re.search(r"Total results found: (\d+)", b).group(1)) == groups
    timing_ok(out, "Q3", 60000)


def test_cli_q9(orc):
    pa, su, ps, od, li = orc.q9_tables(2000, 100, 15000, 60000, 42)
    want, n = orc.q9(pa, su, ps, od, li)
    out = run("sf1", "q9", "--scale", "0.01")
    rows = re.findall(r"^\|\s+(\d+) \|\s+(\d+) \| \$\s*(\S+) \|$", out, re.M)
    assert [(int(a), int(b), scaled(c, 4)) for a, b, c in rows] == want[:15]
    assert int(re.search(r"Total results found: (\d+)", out).group(1)) == n
    timing_ok(out, "Q9", 60000)


def q4_rows(out):
    return [int(x) for x in re.findall(r"^\| [1-5]-[A-Z ]+?\s+\|\s+(\d+) \|$", out, re.M)]


def q12_rows(out):
    return [(int(h), int(l)) for h, l in re.findall(r"^\| (?:MAIL|SHIP)\s+\|\s+(\d+) \|\s+(\d+) \|$", out, re.M)]


def test_cli_q4_and_q12(orc):
    od, li = orc.q4_tables(15_000, 60_000, 42)
    out = run("sf1", "q4", "--scale", "0.01")
    assert q4_rows(out) == orc.q4(od, li)
    assert re.search(r"^Q4 \| 60000 lineitem, 15000 orders", out, re.M)
    for t in TIMING:
        assert t in out
    out = run("sf1", "q12", "--scale", "0.01")
    assert q12_rows(out) == orc.q12(od, li)
    timing_ok(out, "Q12", 60000)
    out = run("sf100", "q12", "--scale", "0.001")   # streamed lineitem
    od, li = orc.q4_tables(150_000, 600_000, 42)
    assert q12_rows(out) == orc.q12(od, li)


def q13_rows(out):
    return [(int(a), int(b)) for a, b in re.findall(r"^\|\s+(\d+) \|\s+(\d+) \|$", out, re.M)]


def test_cli_q13(orc):
    cu, od = orc.q13_tables(1_500, 15_000, 42)
    out = run("sf1", "q13", "--scale", "0.01")
    assert q13_rows(out) == orc.q13(cu, od)
    assert re.search(r"^Q13 \| 15000 orders \| 1500 customers", out, re.M)


def test_cli_q5(orc):
    cu, su, od, li = orc.q5_tables(1_500, 100, 15_000, 60_000, 42)
    out = run("sf1", "q5", "--scale", "0.01")
    names = capi.NATION_NAMES
    rows = re.findall(r"^\| ([A-Z ]+?)\s+\| \$\s*(\S+) \|$", out, re.M)
    assert [(names.index(n), scaled(r, 4)) for n, r in rows] == orc.q5(cu, su, od, li)
    assert re.search(r"^Q5 \| 60000 rows \(lineitem\)", out, re.M)


def test_cli_q7_q8(orc):
    cu, su, pa, od, li = orc.q8_tables(1_500, 100, 2_000, 15_000, 60_000, 42)
    out = run("sf1", "q7", "--scale", "0.01")
    names = capi.NATION_NAMES
    rows = re.findall(r"^\| ([A-Z ]+?)\s+\| ([A-Z ]+?)\s+\|\s+(\d+) \| \$\s*(\S+) \|$", out, re.M)
    assert [(names.index(a), names.index(b), int(y), scaled(r, 4)) for a, b, y, r in rows] == orc.q7(cu, su, od, li)
    out = run("sf1", "q8", "--scale", "0.01")
    vols = [(int(y), int(a), int(b)) for y, a, b in re.findall(r"^volume (\d+): (-?\d+) of (-?\d+)$", out, re.M)]
    assert vols == orc.q8(cu, su, pa, od, li)
    assert re.search(r"^Q8 \| 60000 lineitem", out, re.M)


def test_cli_q10(orc):
    cu, od, li = orc.q10_tables(1_500, 15_000, 60_000, 42)
    top, n = orc.q10(cu, od, li)
    out = run("sf1", "q10", "--scale", "0.01")
    rows = re.findall(r"^\|\s+(\d+) \| Customer#\d+ \| \$\s*(\S+) \|$", out, re.M)
    assert [(int(c), scaled(r, 4)) for c, r in rows] == top
    assert int(re.search(r"Customers with returned revenue: (\d+)", out).group(1)) == n
    timing_ok(out, "Q10", 60000)


def test_cli_microbenchmarks(orc):
    out = run("sf1", "selection", "--scale", "0.01")
    col = orc.gen(1, 60000, 42)
    counts = [int(x) for x in re.findall(r"\((\d+) rows matched\)", out)]
    assert counts == [orc.select_lt(col, v)[0] for v in (100, 1000, 2000)]
    out = run("sf1", "aggregation", "--scale", "0.01")
    assert int(re.search(r"SUM\(l_quantity\): (-?\d+)", out).group(1)) == orc.sum_i32(orc.gen(2, 60000, 42))
    out = run("sf1", "join", "--scale", "0.01")
    b = orc.gen(30, 15000, 42)
    p = orc.gen(8, 60000, 42, n_orders=15000, order_mode=1)
    assert [int(x) for x in re.findall(r"Found (\d+) total matches", out)] == [orc.join_count(b, p)] * 3
    assert re.findall(r"Join \(([a-z ]+)\) complete", out) == ["global table", "radix partitioned", "direct bitmap"]


def test_cli_sf100_streams_the_fact_table(orc):
    n = 600_000   # sf100 x 0.001
    li = orc.lineitem(n, seed=42)
    out = run("sf100", "q6", "--scale", "0.001")
    rev = scaled(re.search(r"Total Revenue: \$(\S+)", out).group(1), 4)
    assert (rev, int(re.search(r"Rows matched: (\d+)", out).group(1))) == orc.q6(li)
    assert re.search(r"^SF100 Q6 \| 1 chunks \| %d rows" % n, out, re.M)


def test_cli_unknown_query_exits_1():
    r = subprocess.run([CLI, "sf1", "q42"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown query" in r.stderr


def test_cli_reads_tbl_files(orc, tmp_path):
    """`gpudb <query> --data DIR` parses DIR/<table>.tbl on the GPU (in pieces that end at a
    line end) and prints the same exact results as the oracle on those rows."""
    n_or, n_cu, n_pa, n_su, n_li = 15_000, 1_500, 2_000, 100, 60_000
    li = orc.lineitem(n_li, seed=7, n_orders=n_or, order_mode=1, n_parts=n_pa, n_supp=n_su,
                      cols=("order_key", "part_key", "supp_key", "quantity", "ext_price", "discount", "tax", "flag",
                            "status", "ship_date", "commit_date", "receipt_date", "ship_mode"))
    od = dict(order_key=orc.gen(30, n_or, 7), cust_key=orc.gen(31, n_or, 7, n_cust=n_cu), order_date=orc.gen(32, n_or, 7),
              priority=orc.gen(33, n_or, 7), comment=orc.gen(34, n_or, 7))
    cu = dict(cust_key=orc.gen(20, n_cu, 7), segment=orc.gen(21, n_cu, 7), nation=orc.gen(22, n_cu, 7))
    pa = dict(part_key=orc.gen(40, n_pa, 7), flag=orc.gen(41, n_pa, 7))
    su = dict(supp_key=orc.gen(50, n_su, 7), nation=orc.gen(51, n_su, 7))
    ps = dict(part_key=orc.gen(60, 4 * n_pa, 7), supp_key=orc.gen(61, 4 * n_pa, 7, n_supp=n_su),
              supply_cost=orc.gen(62, 4 * n_pa, 7))
    for name, cols in (("lineitem", li), ("orders", od), ("customer", cu), ("part", pa), ("supplier", su),
                       ("partsupp", ps)):
        (tmp_path / (name + ".tbl")).write_bytes(orc.format_tbl(name, cols))
    d = str(tmp_path)
    out = run("q6", "--data", d)
    rev = scaled(re.search(r"Total Revenue: \$(\S+)", out).group(1), 4)
    assert (rev, int(re.search(r"Rows matched: (\d+)", out).group(1))) == orc.q6(li)
    timing_ok(out, "Q6", n_li)
    out = run("q1", "--data", d)
    want = orc.q1(li)
    cnts = [int(x) for x in re.findall(r"\|\s+(\d+)\s+\|$", out, re.M)]
    assert sorted(cnts) == sorted(g["count"] for g in want.values())
    out = run("q3", "--data", d)
    top, groups = orc.q3(cu, od, li)
    b = out.split("TPC-H Q3 Results")[1]
    rows = re.findall(r"^\|\s+(\d+) \| \$\s*(\S+) \|\s+(\d+) \|", b, re.M)
    assert [(int(k), int(dd), scaled(r, 4)) for k, r, dd in rows] == top
    assert int(re.search(r"Total results found: (\d+)", b).group(1)) == groups
    out = run("q9", "--data", d)
    want9, n9 = orc.q9(pa, su, ps, dict(order_key=od["order_key"], order_date=od["order_date"]),
                       {k: li[k] for k in ("part_key", "supp_key", "order_key", "ext_price", "discount", "quantity")})
    rows = re.findall(r"^\|\s+(\d+) \|\s+(\d+) \| \$\s*(\S+) \|$", out, re.M)
    assert [(int(a), int(bb), scaled(c, 4)) for a, bb, c in rows] == want9[:15]
    out = run("join", "--data", d)
    assert [int(x) for x in re.findall(r"Found (\d+) total matches", out)] == [orc.join_count(od["order_key"],
                                                                                                li["order_key"])] * 3
    out = run("q4", "--data", d)
    assert q4_rows(out) == orc.q4(od, li)
    out = run("q12", "--data", d)
    assert q12_rows(out) == orc.q12(od, li)
    out = run("q5", "--data", d)
    names = capi.NATION_NAMES
    rows5 = re.findall(r"^\| ([A-Z ]+?)\s+\| \$\s*(\S+) \|$", out, re.M)
    assert [(names.index(n), scaled(r, 4)) for n, r in rows5] == orc.q5(cu, su, od, li)
    out = run("q7", "--data", d)
    rows7 = re.findall(r"^\| ([A-Z ]+?)\s+\| ([A-Z ]+?)\s+\|\s+(\d+) \| \$\s*(\S+) \|$", out, re.M)
    assert [(names.index(a), names.index(b), int(y), scaled(r, 4)) for a, b, y, r in rows7] == \
        orc.q7(cu, su, od, {k: li[k] for k in ("order_key", "supp_key", "ship_date", "ext_price", "discount")})
    out = run("q10", "--data", d)
    top10, n10 = orc.q10(cu, od, li)
    assert int(re.search(r"Customers with returned revenue: (\d+)", out).group(1)) == n10
    out = run("q13", "--data", d)
    assert q13_rows(out) == orc.q13(cu, od)
    out = run("aggregation", "--data", d)
    assert int(re.search(r"SUM\(l_quantity\): (-?\d+)", out).group(1)) == orc.sum_i32(li["quantity"])
    # the same files read 64 KB at a time: rows that straddle pieces are carried over whole
    out = run("q6", "--data", d, "--tbl-piece", "65536")
    rev = scaled(re.search(r"Total Revenue: \$(\S+)", out).group(1), 4)
    assert (rev, int(re.search(r"Rows matched: (\d+)", out).group(1))) == orc.q6(li)
    out = run("q3", "--data", d, "--tbl-piece", "65536")
    b = out.split("TPC-H Q3 Results")[1]
    assert int(re.search(r"Total results found: (\d+)", b).group(1)) == groups
