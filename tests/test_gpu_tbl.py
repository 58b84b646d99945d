"""The .tbl text loader on the GPU (gpudb_tbl_parse): every table kind round-trips through
dbgen-style text exactly, hand-written rows parse to known values (CRLF line ends, no final
newline, negative and one-digit decimals, leap days), key bounds come back, malformed text
and too-small columns are reported, and a pipeline over a loaded table equals the oracle."""
import ctypes as C

import numpy as np
import pytest

from gpudbmetalbenchmark_b200 import capi

pytestmark = pytest.mark.gpu

LI_COLS = ("order_key", "part_key", "supp_key", "quantity", "ext_price", "discount", "tax", "flag", "status",
           "ship_date", "commit_date", "receipt_date", "ship_mode")


def tables(orc):
    n_or, n_cu, n_pa, n_su = 5_000, 800, 1_200, 90
    return {
        "lineitem": orc.lineitem(20_011, seed=3, n_orders=n_or, order_mode=1, n_parts=n_pa, n_supp=n_su, cols=LI_COLS),
        "orders": dict(order_key=orc.gen(30, n_or, 3), cust_key=orc.gen(31, n_or, 3, n_cust=n_cu),
                       order_date=orc.gen(32, n_or, 3), priority=orc.gen(33, n_or, 3), comment=orc.gen(34, n_or, 3)),
        "customer": dict(cust_key=orc.gen(20, n_cu, 3), segment=orc.gen(21, n_cu, 3), nation=orc.gen(22, n_cu, 3)),
        "part": dict(part_key=orc.gen(40, n_pa, 3), flag=orc.gen(41, n_pa, 3), type=orc.gen(42, n_pa, 3)),
        "supplier": dict(supp_key=orc.gen(50, n_su, 3), nation=orc.gen(51, n_su, 3)),
        "partsupp": dict(part_key=orc.gen(60, 4 * n_pa, 3), supp_key=orc.gen(61, 4 * n_pa, 3, n_supp=n_su),
                         supply_cost=orc.gen(62, 4 * n_pa, 3)),
    }


@pytest.mark.parametrize("kind", ["lineitem", "orders", "customer", "part", "supplier", "partsupp"])
def test_round_trip(engine, orc, kind):
    cols = tables(orc)[kind]
    t = engine.load_tbl(kind, orc.format_tbl(kind, cols))
    try:
        assert t.n_rows == len(next(iter(cols.values())))
        for name, want in cols.items():
            assert np.array_equal(t.to_numpy(name), want), name
        first = next(iter(cols))
        key = {"lineitem": "order_key", "orders": "order_key"}.get(kind, "key")
        if kind != "partsupp":
            assert t.key_max[key] == int(cols[first].max())
    finally:
        engine.free(t)


def test_hand_written_rows(engine, orc):
    text = (b"7|11|3|1|17|1234.50|0.05|0.08|R|F|1992-01-01|1991-12-01|1992-01-20|NONE|MAIL|c|\r\n"
            b"9|12|4|2|3|-0.5|0.1|0.00|N|O|1996-02-29|1996-03-01|1996-03-31|COLLECT COD|REG AIR|c|\n"
            b"2147483647|0|0|3|0|0|0|0|A|F|1998-12-01|1998-12-31|1999-01-01|TAKE BACK RETURN|TRUCK|c|")
    t = engine.load_tbl("lineitem", text)
    try:
        want = orc.parse_tbl_cpu("lineitem", text)
        assert t.n_rows == 3
        for name in LI_COLS:
            assert t.to_numpy(name).tolist() == want[name], name
        assert t.to_numpy("ship_date").tolist() == [0, 1520, 2526]
        assert t.to_numpy("commit_date").tolist() == [-31, 1521, 2556]
        assert t.to_numpy("ship_mode").tolist() == [2, 4, 6]
        assert t.key_max["order_key"] == 2147483647
    finally:
        engine.free(t)


@pytest.mark.parametrize("bad", [
    b"7|x|3|1|17|1.00|0.05|0.08|R|F|1992-01-01|",       # a letter in a key
    b"7|1|3|1|17|1.001|0.05|0.08|R|F|1992-01-01|",      # three fraction digits
    b"7|1|3|1|17|1.00|0.05|0.08|Q|F|1992-01-01|",       # unknown return flag
    b"7|1|3|1|17|1.00|0.05|0.08|R|F|1992-1-01|",        # date not YYYY-MM-DD
    b"7|1|3|1|17|1.00|0.05",                            # too few fields
    b"7|1|3|1|17|1.00|0.05|0.08|R|F|1992-01-01|\n\n",   # an empty line
    b"7|1|3|1|17|1.00|0.05|0.08|R|F|1992-01-01|1992-01-02|1992-01-03|NONE|BOAT|c|",   # unknown ship mode
    b"7|1|3|1|17|1.00|0.05|0.08|R|F|1992-01-01|1992-13-02|1992-01-03|NONE|AIR|c|",    # month 13
])
def test_malformed_text_is_rejected(engine, bad):
    with pytest.raises(capi.GpudbError) as e:
        engine.load_tbl("lineitem", bad)
    assert e.value.code == capi.E_INVALID


def test_capacity_and_counts(engine, orc):
    cols = tables(orc)["customer"]
    text = orc.format_tbl("customer", cols)
    buf = np.frombuffer(text, dtype=np.uint8)
    n = C.c_uint64()
    engine._check(engine.lib.gpudb_tbl_count_rows(engine.ctx, buf.ctypes.data, len(text), capi.MEM_HOST, C.byref(n)))
    assert n.value == len(cols["cust_key"])
    out = (C.c_void_p * capi.TBL_MAX_COLS)()
    got = C.c_uint64()
    rc = engine.lib.gpudb_tbl_parse(engine.ctx, capi.TBL_CUSTOMER, buf.ctypes.data, len(text), capi.MEM_HOST, out,
                                    n.value - 1, C.byref(got), None, None)
    assert rc == capi.E_CAPACITY
    # the same text, without its final newline and from device memory
    dev = engine.device_array(len(text) + 16)
    engine._check(engine.lib.gpudb_copy(engine.ctx, dev, buf.ctypes.data, len(text) - 1))
    engine._check(engine.lib.gpudb_tbl_count_rows(engine.ctx, dev, len(text) - 1, capi.MEM_DEVICE, C.byref(n)))
    assert n.value == len(cols["cust_key"])
    engine.device_free(dev)


def test_q1_over_a_loaded_table(engine, orc):
    li = orc.lineitem(30_007, seed=9, n_orders=8_000, order_mode=1, n_parts=1000, n_supp=50, cols=LI_COLS)
    t = engine.load_tbl("lineitem", orc.format_tbl("lineitem", li))
    try:
        assert engine.q1(t, 2000) == orc.q1(li, 2000)
        assert engine.q6(t) == orc.q6(li, 365, 730, 5, 7, 24)
    finally:
        engine.free(t)
