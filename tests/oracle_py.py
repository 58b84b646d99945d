"""ctypes access to the CPU oracle (oracle/_build/liboracle.so) and to the reference's own
kernels compiled for the CPU (oracle/_ref/libgpudbref.so). Test infrastructure only."""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgpudbref.so")

WIDTH = {1: 4, 2: 4, 3: 8, 4: 4, 5: 4, 6: 1, 7: 1, 8: 4, 9: 4, 10: 4, 11: 4, 12: 4, 13: 1, 20: 4, 21: 1, 22: 1, 30: 4,
         31: 4, 32: 4, 33: 1, 34: 80, 40: 4, 41: 1, 42: 1, 50: 4, 51: 1, 60: 4, 61: 4, 62: 8}
DT = {1: np.uint8, 4: np.int32, 8: np.int64, 80: np.dtype("S80")}


class Spec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("row_offset", C.c_uint64), ("n_rows", C.c_uint64),
                ("n_orders", C.c_int64), ("n_cust", C.c_int64), ("n_parts", C.c_int64),
                ("n_supp", C.c_int64), ("order_mode", C.c_int32), ("reserved", C.c_int32)]


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


V, U64, I32, U32, I64 = C.c_void_p, C.c_uint64, C.c_int32, C.c_uint32, C.c_int64
ORACLE_ARGS = {
    "or_gen_column": [V, I32, V],
    "or_q6": [U64, V, V, V, V, I32, I32, I32, I32, I32, V, V],
    "or_q6_mt": [C.c_int, U64, V, V, V, V, I32, I32, I32, I32, I32, V, V],
    "or_q1": [U64, V, V, V, V, V, V, V, I32, V],
    "or_q1_mt": [C.c_int, U64, V, V, V, V, V, V, V, I32, V],
    "or_q3": [U64, V, V, I32, U64, V, V, V, I32, U64, V, V, V, V, I32, I32, I32, I32, V, V, V],
    "or_q9": [U64, V, V, I32, U64, V, V, I32, U64, V, V, V, U64, V, V, I32, U64, V, V, V, V, V, V, U32, V, V, V],
    "or_q4": [U64, V, V, V, I32, U64, V, V, V, I32, I32, V],
    "or_q12": [U64, V, V, I32, U64, V, V, V, V, V, I32, I32, I32, I32, I32, V],
    "or_q13": [U64, V, I32, U64, V, V, C.c_char_p, C.c_char_p, V, V, U32],
    "or_q5": [U64, V, V, I32, U64, V, V, I32, U64, V, V, V, I32, U64, V, V, V, V, I32, I32, U32, V],
    "or_q7": [U64, V, V, I32, U64, V, V, I32, U64, V, V, I32, U64, V, V, V, V, V, I32, I32, I32, I32, V, V, V],
    "or_q8": [U64, V, V, I32, U64, V, V, I32, U64, V, V, I32, U64, V, V, V, I32, U64, V, V, V, V, V, I32, I32, U32, I32,
              I32, V, V, V, V],
    "or_q10": [U64, V, I32, U64, V, V, V, I32, U64, V, V, V, V, I32, I32, I32, V, V, V],
    "or_select_lt": [U64, V, I32, V, V],
    "or_sum_i32": [U64, V],
    "or_join_count": [U64, V, U64, V],
    "or_key_hash": [I32],
    "or_radix_histogram": [U64, V, I32, V],
    "or_radix_partition": [U64, V, V, I32, V, V, V],
    "or_join_pairs": [U64, V, U64, V, U64, V, V],
}
REF_ARGS = {
    "ref_q6": [U64, V, V, V, V, I32, I32, I32, I32, I32, C.c_int, C.c_int],
    "ref_q1": [U64, V, V, V, V, V, V, V, I32, C.c_int, C.c_int, V],
    "ref_q3": [U64, V, V, U64, V, V, V, U64, V, V, V, V, I32, I32, I32, C.c_int, C.c_int, V, V, V, U32],
    "ref_q9": [U64, V, V, U64, V, V, U64, V, V, V, U64, V, V, U64, V, V, V, V, V, V, C.c_int, C.c_int, V, V, V, U32],
    "ref_q4": [U64, V, V, V, U64, V, V, V, I32, I32, C.c_int, C.c_int, V],
    "ref_q12": [U64, V, V, U64, V, V, V, V, V, I32, I32, C.c_int, C.c_int, V],
    "ref_q13": [U64, U64, V, V, C.c_int, C.c_int, V],
    "ref_q5": [U64, V, V, U64, V, V, U64, V, V, V, U64, V, V, V, V, I32, I32, U32, C.c_int, C.c_int, V],
    "ref_q7": [U64, V, V, U64, V, V, U64, V, V, U64, V, V, V, V, V, I32, I32, I32, I32, C.c_int, C.c_int, V],
    "ref_q8": [U64, V, V, U64, V, V, U64, V, V, U64, V, V, V, U64, V, V, V, V, V, I32, I32, U32, I32, I32, C.c_int,
               C.c_int, V],
    "ref_q10": [U64, V, V, V, U64, V, V, V, V, I32, I32, C.c_int, C.c_int, V, U32],
    "ref_select_lt": [U64, V, I32, V],
    "ref_sum": [U64, V, C.c_int, C.c_int],
    "ref_join_count": [U64, V, U64, V],
    "ref_radix_partition": [U64, V, V, V, V, V, V],
    "ref_partition_join": [U64, V, U64, V, V, V, U32],
}


def build():
    import subprocess
    import sys
    subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "build.py")], check=True,
                   stdout=subprocess.DEVNULL)


_or = None
_ref = None


def oracle():
    global _or
    if _or is None:
        if not os.path.exists(ORACLE_SO):
            build()
        _or = C.CDLL(ORACLE_SO)
        for name, args in ORACLE_ARGS.items():
            getattr(_or, name).argtypes = args
        _or.or_key_hash.restype = C.c_uint32
        _or.or_q3.restype = C.c_uint64
        _or.or_q9.restype = C.c_uint32
        _or.or_select_lt.restype = C.c_uint64
        _or.or_q13.restype = C.c_uint32
        _or.or_q10.restype = C.c_uint64
        _or.or_sum_i32.restype = C.c_int64
        _or.or_join_count.restype = C.c_uint64
        _or.or_join_pairs.restype = C.c_uint64
    return _or


def reference():
    """The reference's kernels on the CPU, or None where they were never built."""
    global _ref
    if _ref is None and os.path.exists(REF_SO):
        _ref = C.CDLL(REF_SO)
        for name, args in REF_ARGS.items():
            getattr(_ref, name).argtypes = args
        _ref.ref_q6.restype = C.c_float
        _ref.ref_sum.restype = C.c_float
        _ref.ref_q3.restype = C.c_uint32
        _ref.ref_q9.restype = C.c_uint32
        _ref.ref_join_count.restype = C.c_uint32
        _ref.ref_partition_join.restype = C.c_uint32
    return _ref


# ---- generator ---------------------------------------------------------------------------
def gen(column, n_rows, seed=42, row_offset=0, n_orders=0, n_cust=0, n_parts=0, n_supp=0, order_mode=0):
    out = np.empty(n_rows, dtype=DT[WIDTH[column]])
    spec = Spec(seed, row_offset, n_rows, n_orders, n_cust, n_parts, n_supp, order_mode, 0)
    rc = oracle().or_gen_column(C.byref(spec), column, out.ctypes.data)
    assert rc == 0, "oracle generator rejected column %d" % column
    return out


def lineitem(n, seed=42, n_orders=0, order_mode=0, n_parts=0, n_supp=0, row_offset=0,
             cols=("ship_date", "quantity", "ext_price", "discount", "tax", "flag", "status")):
    ids = dict(ship_date=1, quantity=2, ext_price=3, discount=4, tax=5, flag=6, status=7, order_key=8,
               part_key=9, supp_key=10, commit_date=11, receipt_date=12, ship_mode=13)
    return {c: gen(ids[c], n, seed, row_offset, n_orders, 0, n_parts, n_supp, order_mode) for c in cols}


def q3_tables(n_cu, n_or, n_li, seed=42):
    cu = dict(cust_key=gen(20, n_cu, seed), segment=gen(21, n_cu, seed))
    od = dict(order_key=gen(30, n_or, seed), cust_key=gen(31, n_or, seed, n_cust=n_cu), order_date=gen(32, n_or, seed))
    li = lineitem(n_li, seed, n_orders=n_or, order_mode=1, cols=("order_key", "ship_date", "ext_price", "discount"))
    return cu, od, li


def q4_tables(n_or, n_li, seed=42, order_mode=1):
    """Orders (key, date, priority) and lineitem (order key, ship/commit/receipt dates, ship
    mode) of the seeded generator: the tables of Q4 and Q12."""
    od = dict(order_key=gen(30, n_or, seed), order_date=gen(32, n_or, seed), priority=gen(33, n_or, seed))
    li = lineitem(n_li, seed, n_orders=n_or, order_mode=order_mode,
                  cols=("order_key", "ship_date", "commit_date", "receipt_date", "ship_mode"))
    return od, li


def q5_tables(n_cu, n_su, n_or, n_li, seed=42):
    cu = dict(cust_key=gen(20, n_cu, seed), nation=gen(22, n_cu, seed))
    su = dict(supp_key=gen(50, n_su, seed), nation=gen(51, n_su, seed))
    od = dict(order_key=gen(30, n_or, seed), cust_key=gen(31, n_or, seed, n_cust=n_cu), order_date=gen(32, n_or, seed))
    li = lineitem(n_li, seed, n_orders=n_or, order_mode=1, n_parts=max(1, n_su * 20), n_supp=n_su,
                  cols=("order_key", "supp_key", "ext_price", "discount"))
    return cu, su, od, li


ASIA = (1 << 8) | (1 << 9) | (1 << 12) | (1 << 18) | (1 << 21)


def q5(cu, su, od, li, date_lo=731, date_hi=1096, mask=ASIA, revenue_out=None):
    """[(nation, revenue)] nonzero, ordered by revenue desc then nation asc."""
    rev = np.zeros(25, np.int64) if revenue_out is None else revenue_out
    kmax = lambda a: int(a.max()) if len(a) else -1  # noqa: E731
    oracle().or_q5(len(cu["cust_key"]), _p(cu["cust_key"]), _p(cu["nation"]), kmax(cu["cust_key"]),
                   len(su["supp_key"]), _p(su["supp_key"]), _p(su["nation"]), kmax(su["supp_key"]),
                   len(od["order_key"]), _p(od["order_key"]), _p(od["cust_key"]), _p(od["order_date"]),
                   kmax(od["order_key"]), len(li["order_key"]), _p(li["order_key"]), _p(li["supp_key"]),
                   _p(li["ext_price"]), _p(li["discount"]), date_lo, date_hi, mask, rev.ctypes.data)
    return sorted(((n, int(rev[n])) for n in range(25) if rev[n]), key=lambda x: (-x[1], x[0]))


FRANCE, GERMANY, BRAZIL = 6, 7, 2
AMERICA = (1 << 1) | (1 << 2) | (1 << 3) | (1 << 17) | (1 << 24)
NATION_NAMES = ("ALGERIA", "ARGENTINA", "BRAZIL", "CANADA", "EGYPT", "ETHIOPIA", "FRANCE", "GERMANY", "INDIA",
                "INDONESIA", "IRAN", "IRAQ", "JAPAN", "JORDAN", "KENYA", "MOROCCO", "MOZAMBIQUE", "PERU", "CHINA",
                "ROMANIA", "SAUDI ARABIA", "VIETNAM", "RUSSIA", "UNITED KINGDOM", "UNITED STATES")


def q8_tables(n_cu, n_su, n_pa, n_or, n_li, seed=42):
    """Customer (key, nation), supplier (key, nation), part (key, type), orders (key, customer,
    date) and lineitem (order, part, supplier keys, ext_price, discount): the tables of Q7 and Q8."""
    cu = dict(cust_key=gen(20, n_cu, seed), nation=gen(22, n_cu, seed))
    su = dict(supp_key=gen(50, n_su, seed), nation=gen(51, n_su, seed))
    pa = dict(part_key=gen(40, n_pa, seed), type=gen(42, n_pa, seed))
    od = dict(order_key=gen(30, n_or, seed), cust_key=gen(31, n_or, seed, n_cust=n_cu), order_date=gen(32, n_or, seed))
    li = lineitem(n_li, seed, n_orders=n_or, order_mode=1, n_parts=n_pa, n_supp=n_su,
                  cols=("order_key", "part_key", "supp_key", "ship_date", "ext_price", "discount"))
    return cu, su, pa, od, li


def _kmax(a):
    return int(a.max()) if len(a) else -1


def q7(cu, su, od, li, a=FRANCE, b=GERMANY, ship_lo=1096, ship_hi=1826):
    """[(supp_nation, cust_nation, year, revenue)] nonzero, ordered by nation names, then year."""
    rev = np.zeros(16, np.int64)
    fy, ny = C.c_int32(), C.c_int32()
    rc = oracle().or_q7(len(cu["cust_key"]), _p(cu["cust_key"]), _p(cu["nation"]), _kmax(cu["cust_key"]),
                        len(su["supp_key"]), _p(su["supp_key"]), _p(su["nation"]), _kmax(su["supp_key"]),
                        len(od["order_key"]), _p(od["order_key"]), _p(od["cust_key"]), _kmax(od["order_key"]),
                        len(li["order_key"]), _p(li["order_key"]), _p(li["supp_key"]), _p(li["ship_date"]),
                        _p(li["ext_price"]), _p(li["discount"]), a, b, ship_lo, ship_hi, rev.ctypes.data,
                        C.byref(fy), C.byref(ny))
    assert rc == 0
    rows = [(s, c, fy.value + y, int(rev[pair * 8 + y])) for pair, (s, c) in enumerate(((a, b), (b, a)))
            for y in range(ny.value) if rev[pair * 8 + y]]
    return sorted(rows, key=lambda x: (NATION_NAMES[x[0]], NATION_NAMES[x[1]], x[2]))


def q8(cu, su, pa, od, li, nation=BRAZIL, region_mask=AMERICA, part_type=103, date_lo=1096, date_hi=1826):
    """[(year, nation_volume, volume)] per calendar year of the window."""
    vol, nvol = np.zeros(8, np.int64), np.zeros(8, np.int64)
    fy, ny = C.c_int32(), C.c_int32()
    rc = oracle().or_q8(len(cu["cust_key"]), _p(cu["cust_key"]), _p(cu["nation"]), _kmax(cu["cust_key"]),
                        len(su["supp_key"]), _p(su["supp_key"]), _p(su["nation"]), _kmax(su["supp_key"]),
                        len(pa["part_key"]), _p(pa["part_key"]), _p(pa["type"]), _kmax(pa["part_key"]),
                        len(od["order_key"]), _p(od["order_key"]), _p(od["cust_key"]), _p(od["order_date"]),
                        _kmax(od["order_key"]), len(li["order_key"]), _p(li["order_key"]), _p(li["part_key"]),
                        _p(li["supp_key"]), _p(li["ext_price"]), _p(li["discount"]), date_lo, date_hi, region_mask,
                        nation, part_type, vol.ctypes.data, nvol.ctypes.data, C.byref(fy), C.byref(ny))
    assert rc == 0
    return [(fy.value + y, int(nvol[y]), int(vol[y])) for y in range(ny.value)]


def q10_tables(n_cu, n_or, n_li, seed=42):
    cu = dict(cust_key=gen(20, n_cu, seed))
    od = dict(order_key=gen(30, n_or, seed), cust_key=gen(31, n_or, seed, n_cust=n_cu), order_date=gen(32, n_or, seed))
    li = lineitem(n_li, seed, n_orders=n_or, order_mode=1, cols=("order_key", "flag", "ext_price", "discount"))
    return cu, od, li


def q10(cu, od, li, date_lo=639, date_hi=731, k=20, cu_key_max=None, or_key_max=None, rev_out=None):
    """([(cust_key, revenue)] top k, number of customers with revenue > 0)."""
    n_cu = len(cu["cust_key"])
    ck = (int(cu["cust_key"].max()) if n_cu else -1) if cu_key_max is None else cu_key_max
    ok = (int(od["order_key"].max()) if len(od["order_key"]) else -1) if or_key_max is None else or_key_max
    tk, tr = np.zeros(k, np.int32), np.zeros(k, np.int64)
    n = oracle().or_q10(n_cu, _p(cu["cust_key"]), ck, len(od["order_key"]), _p(od["order_key"]), _p(od["cust_key"]),
                        _p(od["order_date"]), ok, len(li["order_key"]), _p(li["order_key"]), _p(li["flag"]),
                        _p(li["ext_price"]), _p(li["discount"]), date_lo, date_hi, k, tk.ctypes.data, tr.ctypes.data,
                        None if rev_out is None else rev_out.ctypes.data)
    return [(int(a), int(b)) for a, b in zip(tk, tr) if a >= 0], int(n)


def q13_tables(n_cu, n_or, seed=42):
    cu = dict(cust_key=gen(20, n_cu, seed))
    od = dict(cust_key=gen(31, n_or, seed, n_cust=n_cu), comment=gen(34, n_or, seed))
    return cu, od


def q9_tables(n_pa, n_su, n_or, n_li, seed=42):
    pa = dict(part_key=gen(40, n_pa, seed), flag=gen(41, n_pa, seed))
    su = dict(supp_key=gen(50, n_su, seed), nation=gen(51, n_su, seed))
    n_ps = 4 * n_pa
    ps = dict(part_key=gen(60, n_ps, seed), supp_key=gen(61, n_ps, seed, n_supp=n_su),
              supply_cost=gen(62, n_ps, seed))
    od = dict(order_key=gen(30, n_or, seed), order_date=gen(32, n_or, seed))
    li = lineitem(n_li, seed, n_orders=n_or, order_mode=2, n_parts=n_pa, n_supp=n_su,
                  cols=("part_key", "supp_key", "order_key", "ext_price", "discount", "quantity"))
    return pa, su, ps, od, li


# ---- pipelines ---------------------------------------------------------------------------
def q6(li, lo=365, hi=730, dlo=5, dhi=7, qlt=24, threads=0):
    rev, m = C.c_int64(), C.c_uint64()
    n = len(li["ship_date"])
    args = (n, _p(li["ship_date"]), _p(li["discount"]), _p(li["quantity"]), _p(li["ext_price"]),
            lo, hi, dlo, dhi, qlt, C.byref(rev), C.byref(m))
    if threads:
        oracle().or_q6_mt(threads, *args)
    else:
        oracle().or_q6(*args)
    return rev.value, m.value


def _i128(lo, hi):
    v = (int(hi) << 64) | int(lo)
    return v - (1 << 128) if v >> 127 else v


def q1(li, ship_le=2436, threads=0):
    out = np.zeros(66, dtype=np.uint64)
    n = len(li["ship_date"])
    args = (n, _p(li["ship_date"]), _p(li["quantity"]), _p(li["ext_price"]), _p(li["discount"]), _p(li["tax"]),
            _p(li["flag"]), _p(li["status"]), ship_le, out.ctypes.data)
    if threads:
        oracle().or_q1_mt(threads, *args)
    else:
        oracle().or_q1(*args)
    res = {}
    for g in range(6):
        o = out[g * 11:(g + 1) * 11]
        if o[0] == 0:
            continue
        res[(g // 2, g % 2)] = dict(count=int(o[0]), sum_qty=_i128(o[1], o[2]), sum_base_price=_i128(o[3], o[4]),
                                    sum_disc_price=_i128(o[5], o[6]), sum_charge=_i128(o[7], o[8]),
                                    sum_discount=_i128(o[9], o[10]))
    return res


def q3(cu, od, li, segment=1, date_lt=1170, ship_gt=1170, k=10, cu_key_max=None, or_key_max=None):
    cu_key_max = int(cu["cust_key"].max()) if cu_key_max is None else cu_key_max
    or_key_max = int(od["order_key"].max()) if or_key_max is None else or_key_max
    k = max(k, 1)
    tk, td, tr = np.zeros(k, np.int32), np.zeros(k, np.int32), np.zeros(k, np.int64)
    n = oracle().or_q3(len(cu["cust_key"]), _p(cu["cust_key"]), _p(cu["segment"]), cu_key_max,
                       len(od["order_key"]), _p(od["order_key"]), _p(od["cust_key"]), _p(od["order_date"]), or_key_max,
                       len(li["order_key"]), _p(li["order_key"]), _p(li["ship_date"]), _p(li["ext_price"]),
                       _p(li["discount"]), segment, date_lt, ship_gt, k, tk.ctypes.data, td.ctypes.data,
                       tr.ctypes.data)
    m = min(n, k)
    return [(int(tk[i]), int(td[i]), int(tr[i])) for i in range(m)], int(n)


def q9(pa, su, ps, od, li, cap=4096):
    gn, gy, gp = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap, np.int64)
    n = oracle().or_q9(len(pa["part_key"]), _p(pa["part_key"]), _p(pa["flag"]), int(pa["part_key"].max()),
                       len(su["supp_key"]), _p(su["supp_key"]), _p(su["nation"]), int(su["supp_key"].max()),
                       len(ps["part_key"]), _p(ps["part_key"]), _p(ps["supp_key"]), _p(ps["supply_cost"]),
                       len(od["order_key"]), _p(od["order_key"]), _p(od["order_date"]), int(od["order_key"].max()),
                       len(li["part_key"]), _p(li["part_key"]), _p(li["supp_key"]), _p(li["order_key"]),
                       _p(li["ext_price"]), _p(li["discount"]), _p(li["quantity"]), cap, gn.ctypes.data,
                       gy.ctypes.data, gp.ctypes.data)
    m = min(n, cap)
    return [(int(gn[i]), int(gy[i]), int(gp[i])) for i in range(m)], int(n)


def q4(od, li, date_lo=547, date_hi=639, or_key_max=None):
    """[count of priority 1..5]."""
    out = np.zeros(5, np.uint64)
    kmax = int(od["order_key"].max()) if or_key_max is None and len(od["order_key"]) else (or_key_max or 0)
    oracle().or_q4(len(od["order_key"]), _p(od["order_key"]), _p(od["order_date"]), _p(od["priority"]), kmax,
                   len(li["order_key"]), _p(li["order_key"]), _p(li["commit_date"]), _p(li["receipt_date"]),
                   date_lo, date_hi, out.ctypes.data)
    return [int(x) for x in out]


def q12(od, li, receipt_lo=731, receipt_hi=1096, modes=(2, 5), high_max=2, or_key_max=None):
    """[(high, low) for mode0, (high, low) for mode1]."""
    out = np.zeros(4, np.uint64)
    kmax = int(od["order_key"].max()) if or_key_max is None and len(od["order_key"]) else (or_key_max or 0)
    oracle().or_q12(len(od["order_key"]), _p(od["order_key"]), _p(od["priority"]), kmax, len(li["order_key"]),
                    _p(li["order_key"]), _p(li["ship_date"]), _p(li["commit_date"]), _p(li["receipt_date"]),
                    _p(li["ship_mode"]), receipt_lo, receipt_hi, modes[0], modes[1], high_max, out.ctypes.data)
    return [(int(out[0]), int(out[2])), (int(out[1]), int(out[3]))]


def q13(cu, od, word1=b"special", word2=b"requests", cu_key_max=None):
    """[(c_count, custdist)] ordered by custdist desc, c_count desc."""
    n_cu = len(cu["cust_key"])
    kmax = (int(cu["cust_key"].max()) if n_cu else -1) if cu_key_max is None else cu_key_max
    cap = 1 << 16
    cc, cd = np.zeros(cap, np.uint32), np.zeros(cap, np.uint32)
    comment = np.ascontiguousarray(od["comment"], dtype="S80")
    n = oracle().or_q13(n_cu, _p(cu["cust_key"]), kmax, len(od["cust_key"]), _p(od["cust_key"]), _p(comment),
                        word1, word2, cc.ctypes.data, cd.ctypes.data, cap)
    return [(int(cc[i]), int(cd[i])) for i in range(min(n, cap))]


def select_lt(col, value):
    n = len(col)
    bits = np.zeros((n + 31) // 32, np.uint32)
    rows = np.zeros(max(n, 1), np.uint32)
    c = oracle().or_select_lt(n, _p(col), value, bits.ctypes.data, rows.ctypes.data)
    return int(c), bits, rows[:c]


def sum_i32(col):
    return int(oracle().or_sum_i32(len(col), _p(col)))


def join_count(b, p):
    return int(oracle().or_join_count(len(b), _p(b), len(p), _p(p)))


def radix_partition(keys, payload, bits):
    n = len(keys)
    ko, po = np.zeros(n, np.int32), np.zeros(n, np.int32)
    off = np.zeros((1 << bits) + 1, np.uint32)
    oracle().or_radix_partition(n, _p(keys), _p(payload), bits, ko.ctypes.data, po.ctypes.data, off.ctypes.data)
    return ko, po, off


def join_pairs(b, p, cap=None):
    cap = cap if cap is not None else len(p) * 8 + 16
    ob, op = np.zeros(cap, np.int32), np.zeros(cap, np.int32)
    n = int(oracle().or_join_pairs(len(b), _p(b), len(p), _p(p), cap, ob.ctypes.data, op.ctypes.data))
    return ob[:min(n, cap)], op[:min(n, cap)], n


# ---- dbgen-style text (test infrastructure for the .tbl loader) ------------------------
# Field layouts of dbgen's '|'-separated rows; the loader keeps the fields listed in
# include/gpudb_capi.h. Filler fields hold made-up text of plausible length.
import datetime as _dt

_EPOCH = _dt.date(1992, 1, 1)
_SEGMENTS = ("AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY")
_FLAGS, _STATUS = "ANR", "FO"
_MODES = ("AIR", "FOB", "MAIL", "RAIL", "REG AIR", "SHIP", "TRUCK")
_PTYPE = (("STANDARD", "SMALL", "MEDIUM", "LARGE", "ECONOMY", "PROMO"),
          ("ANODIZED", "BURNISHED", "PLATED", "POLISHED", "BRUSHED"), ("TIN", "NICKEL", "BRASS", "STEEL", "COPPER"))
_PRIORITIES = ("1-URGENT", "2-HIGH", "3-MEDIUM", "4-NOT SPECIFIED", "5-LOW")


def _date(d):
    return (_EPOCH + _dt.timedelta(days=int(d))).isoformat()


def _money(h):
    h = int(h)
    return "%s%d.%02d" % ("-" if h < 0 else "", abs(h) // 100, abs(h) % 100)


def format_tbl(kind, c):
    """Rows of table `kind` as dbgen text (bytes) from numpy columns in the engine's encoding."""
    out = []
    if kind == "lineitem":
        n = len(c["order_key"])
        for i in range(n):
            sd = int(c["ship_date"][i])
            cd = int(c["commit_date"][i]) if "commit_date" in c else sd + 30
            rd = int(c["receipt_date"][i]) if "receipt_date" in c else sd + 45
            mode = _MODES[c["ship_mode"][i]] if "ship_mode" in c else "TRUCK"
            out.append("%d|%d|%d|%d|%d|%s|0.%02d|0.%02d|%s|%s|%s|%s|%s|DELIVER IN PERSON|%s|row %d of the sample|"
                       % (c["order_key"][i], c["part_key"][i], c["supp_key"][i], i % 7 + 1, c["quantity"][i],
                          _money(c["ext_price"][i]), c["discount"][i], c["tax"][i], _FLAGS[c["flag"][i]],
                          _STATUS[c["status"][i]], _date(sd), _date(cd), _date(rd), mode, i))
    elif kind == "orders":
        for i in range(len(c["order_key"])):
            prio = _PRIORITIES[c["priority"][i] - 1] if "priority" in c else "3-MEDIUM"
            note = c["comment"][i].decode() if "comment" in c else "an order"
            out.append("%d|%d|O|%s|%s|%s|Clerk#%09d|0|%s|" % (c["order_key"][i], c["cust_key"][i],
                                                                  _money(12345 + i), _date(c["order_date"][i]),
                                                                  prio, i, note))
    elif kind == "customer":
        for i in range(len(c["cust_key"])):
            nation = int(c["nation"][i]) if "nation" in c else i % 25
            out.append("%d|Customer#%09d|addr %d|%d|10-123-456-7890|%s|%s|a customer|"
                       % (c["cust_key"][i], c["cust_key"][i], i, nation, _money(100 * i - 5000), _SEGMENTS[c["segment"][i]]))
    elif kind == "part":
        for i in range(len(c["part_key"])):
            name = "forest green lace" if c["flag"][i] else "steel ivory lace"
            t = int(c["type"][i]) if "type" in c else 2 * 25 + 2 * 5 + 0   # MEDIUM PLATED TIN by default
            ptype = "%s %s %s" % (_PTYPE[0][t // 25], _PTYPE[1][t // 5 % 5], _PTYPE[2][t % 5])
            out.append("%d|%s %d|Manufacturer#1|Brand#13|%s|7|JUMBO PKG|%s|a part|"
                       % (c["part_key"][i], name, i, ptype, _money(90000 + i)))
    elif kind == "supplier":
        for i in range(len(c["supp_key"])):
            out.append("%d|Supplier#%09d|addr %d|%d|11-222-333-4444|%s|a supplier|"
                       % (c["supp_key"][i], c["supp_key"][i], i, c["nation"][i], _money(500 * i)))
    elif kind == "partsupp":
        for i in range(len(c["part_key"])):
            out.append("%d|%d|%d|%s|a partsupp row|" % (c["part_key"][i], c["supp_key"][i], 1000 + i % 9000,
                                                         _money(c["supply_cost"][i])))
    else:
        raise ValueError(kind)
    return ("\n".join(out) + ("\n" if out else "")).encode()


def parse_tbl_cpu(kind, text):
    """The loader's contract restated on the CPU: the kept fields of every row as numpy
    columns in the engine's encoding."""
    keep = {"lineitem": [(0, "order_key", "i"), (1, "part_key", "i"), (2, "supp_key", "i"), (4, "quantity", "q"),
                         (5, "ext_price", "m"), (6, "discount", "m"), (7, "tax", "m"), (8, "flag", "r"),
                         (9, "status", "s"), (10, "ship_date", "d"), (11, "commit_date", "d"),
                         (12, "receipt_date", "d"), (14, "ship_mode", "e")],
            "orders": [(0, "order_key", "i"), (1, "cust_key", "i"), (4, "order_date", "d"), (5, "priority", "p"),
                       (8, "comment", "c")],
            "customer": [(0, "cust_key", "i"), (3, "nation", "i"), (6, "segment", "g")],
            "part": [(0, "part_key", "i"), (1, "flag", "n"), (4, "type", "t")],
            "supplier": [(0, "supp_key", "i"), (3, "nation", "i")],
            "partsupp": [(0, "part_key", "i"), (1, "supp_key", "i"), (3, "supply_cost", "m")]}[kind]

    def money(s):
        neg = s.startswith("-")
        ip, _, fp = s.lstrip("-").partition(".")
        v = int(ip) * 100 + (int((fp + "00")[:2]) if fp else 0)
        return -v if neg else v

    conv = {"i": int, "q": lambda s: money(s) // 100, "m": money, "r": _FLAGS.index, "s": _STATUS.index,
            "d": lambda s: (_dt.date.fromisoformat(s) - _EPOCH).days, "g": _SEGMENTS.index,
            "n": lambda s: int("green" in s), "e": _MODES.index, "p": lambda s: _PRIORITIES.index(s) + 1,
            "c": lambda s: s.encode(),
            "t": lambda s: _PTYPE[0].index(s.split()[0]) * 25 + _PTYPE[1].index(s.split()[1]) * 5 +
            _PTYPE[2].index(s.split()[2])}
    rows = [l.rstrip("\r").split("|") for l in text.decode().split("\n") if l != ""]
    return {name: [conv[t](r[f]) for r in rows] for f, name, t in keep}
