"""The .tbl text layout used by the loader's tests, on the CPU: formatting the engine's
columns as dbgen rows and parsing them back (the CPU restatement of the loader's contract)
is the identity, and hand-written rows parse to known values."""
import numpy as np

import oracle_py as orc


def test_format_parse_round_trip_cpu():
    li = orc.lineitem(2000, seed=5, n_orders=500, order_mode=1, n_parts=300, n_supp=40,
                      cols=("order_key", "part_key", "supp_key", "quantity", "ext_price", "discount", "tax", "flag",
                            "status", "ship_date", "commit_date", "receipt_date", "ship_mode"))
    got = orc.parse_tbl_cpu("lineitem", orc.format_tbl("lineitem", li))
    for k, v in li.items():
        assert np.array_equal(np.asarray(got[k]), v), k


def test_hand_written_rows_cpu():
    text = (b"7|11|3|1|17|1234.50|0.05|0.08|R|F|1992-01-01|1991-12-01|1992-01-20|NONE|MAIL|c|\r\n"
            b"9|12|4|2|3|-0.5|0.1|0.00|N|O|1996-02-29|1996-03-01|1996-03-31|COLLECT COD|REG AIR|c|")
    got = orc.parse_tbl_cpu("lineitem", text)
    assert got["ext_price"] == [123450, -50] and got["discount"] == [5, 10] and got["tax"] == [8, 0]
    assert got["ship_date"] == [0, 1520] and got["flag"] == [2, 1] and got["status"] == [0, 1]
    assert got["commit_date"] == [-31, 1521] and got["receipt_date"] == [19, 1551] and got["ship_mode"] == [2, 4]


def test_orders_priority_round_trip_cpu():
    od = dict(order_key=orc.gen(30, 500, 4), cust_key=orc.gen(31, 500, 4, n_cust=50), order_date=orc.gen(32, 500, 4),
              priority=orc.gen(33, 500, 4), comment=orc.gen(34, 500, 4))
    got = orc.parse_tbl_cpu("orders", orc.format_tbl("orders", od))
    for k, v in od.items():
        assert np.array_equal(np.asarray(got[k]), v), k


def test_part_type_round_trip_cpu():
    pa = dict(part_key=orc.gen(40, 600, 4), flag=orc.gen(41, 600, 4), type=orc.gen(42, 600, 4))
    got = orc.parse_tbl_cpu("part", orc.format_tbl("part", pa))
    for k, v in pa.items():
        assert np.array_equal(np.asarray(got[k]), v), k
    assert orc.parse_tbl_cpu("part", b"1|x|M|B|ECONOMY ANODIZED STEEL|1|C|1.00|c|")["type"] == [103]


def test_customer_supplier_nation_round_trip_cpu():
    cu = dict(cust_key=orc.gen(20, 400, 6), segment=orc.gen(21, 400, 6), nation=orc.gen(22, 400, 6))
    got = orc.parse_tbl_cpu("customer", orc.format_tbl("customer", cu))
    for k, v in cu.items():
        assert np.array_equal(np.asarray(got[k]), v), k
    assert set(np.unique(cu["nation"])) <= set(range(25))
    su = dict(supp_key=orc.gen(50, 300, 6), nation=orc.gen(51, 300, 6))
    got = orc.parse_tbl_cpu("supplier", orc.format_tbl("supplier", su))
    for k, v in su.items():
        assert np.array_equal(np.asarray(got[k]), v), k
