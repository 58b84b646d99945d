"""ctypes binding of include/gpudb_capi.h (the engine's C ABI).

This is the reference-side binding a Python caller uses; the same structs and entry points
are what a cgo / JNI / N-API stub binds. Loading fails loudly when lib/libgpudb.so is
missing: there is no fallback implementation.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libgpudb.so")

# status codes
OK = 0
E_INVALID, E_CUDA, E_OOM, E_NODEVICE, E_CAPACITY, E_KEY_RANGE, E_TIMEOUT, E_BUSY, E_CLOSED, E_UNSUPPORTED = \
    -1, -2, -3, -4, -5, -6, -7, -8, -9, -10
ERROR_NAMES = {0: "OK", -1: "E_INVALID", -2: "E_CUDA", -3: "E_OOM", -4: "E_NODEVICE", -5: "E_CAPACITY",
               -6: "E_KEY_RANGE", -7: "E_TIMEOUT", -8: "E_BUSY", -9: "E_CLOSED", -10: "E_UNSUPPORTED"}

MEM_DEVICE, MEM_HOST = 0, 1
OPT_CHUNK_ROWS = 1
OPT_SCAN_VARIANT = 2
OPT_Q6_VARIANT = 3
OPT_HT_LOAD = 4
OPT_RADIX_BITS = 5
OPT_Q9_SMEM_SLOTS = 6
OPT_Q9_GLOBAL_SLOTS = 7
OPT_GRAPHS = 8
OPT_Q3_AUTO_MODE = 9
OPT_RADIX_SHAPE = 10
TBL_LINEITEM, TBL_ORDERS, TBL_CUSTOMER, TBL_PART, TBL_SUPPLIER, TBL_PARTSUPP = 1, 2, 3, 4, 5, 6
TBL_MAX_COLS = 13
# columns a .tbl parse keeps, in the order of gpudb_tbl_parse's cols[]
TBL_COLUMNS = {
    "lineitem": (TBL_LINEITEM, ("order_key", "part_key", "supp_key", "quantity", "ext_price", "discount", "tax",
                                "flag", "status", "ship_date", "commit_date", "receipt_date", "ship_mode")),
    "orders": (TBL_ORDERS, ("order_key", "cust_key", "order_date", "priority", "comment")),
    "customer": (TBL_CUSTOMER, ("cust_key", "nation", "segment")),
    "part": (TBL_PART, ("part_key", "flag", "type")),
    "supplier": (TBL_SUPPLIER, ("supp_key", "nation")),
    "partsupp": (TBL_PARTSUPP, ("part_key", "supp_key", "supply_cost")),
}
OPT_NAMES = {1: "chunk_rows", 2: "q1_variant", 3: "q6_variant", 4: "ht_load_pct", 5: "radix_bits",
             6: "q9_smem_slots", 7: "q9_global_slots", 8: "graphs", 9: "q3_auto_mode", 10: "radix_shape"}
JOIN_GLOBAL, JOIN_RADIX, JOIN_DIRECT, JOIN_AUTO = 0, 1, 2, 3
JOIN_MODES = (JOIN_GLOBAL, JOIN_RADIX, JOIN_DIRECT)
JOIN_NAMES = {JOIN_GLOBAL: "global", JOIN_RADIX: "radix", JOIN_DIRECT: "direct", JOIN_AUTO: "auto"}
ORDERS_NONE, ORDERS_CLUSTERED, ORDERS_UNIFORM = 0, 1, 2
Q3_MAX_K = 64
# l_shipmode codes (alphabetical: ORDER BY l_shipmode)
MODE_AIR, MODE_FOB, MODE_MAIL, MODE_RAIL, MODE_REG_AIR, MODE_SHIP, MODE_TRUCK = range(7)
SHIP_MODES = ("AIR", "FOB", "MAIL", "RAIL", "REG AIR", "SHIP", "TRUCK")
PRIORITIES = ("1-URGENT", "2-HIGH", "3-MEDIUM", "4-NOT SPECIFIED", "5-LOW")
COMMENT_WIDTH = 80      # o_comment bytes per row, NUL-padded
Q13_MAX_COUNT = 1023

# column ids
COL = dict(
    LI_SHIP_DATE=1, LI_QUANTITY=2, LI_EXT_PRICE=3, LI_DISCOUNT=4, LI_TAX=5, LI_FLAG=6, LI_STATUS=7,
    LI_ORDER_KEY=8, LI_PART_KEY=9, LI_SUPP_KEY=10, LI_COMMIT_DATE=11, LI_RECEIPT_DATE=12, LI_SHIP_MODE=13,
    CU_CUST_KEY=20, CU_SEGMENT=21, CU_NATION=22,
    OR_ORDER_KEY=30, OR_CUST_KEY=31, OR_ORDER_DATE=32, OR_PRIORITY=33, OR_COMMENT=34,
    PA_PART_KEY=40, PA_FLAG=41, PA_TYPE=42,
    SU_SUPP_KEY=50, SU_NATION=51,
    PS_PART_KEY=60, PS_SUPP_KEY=61, PS_SUPPLY_COST=62,
)

vp = C.c_void_p


class I128(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_int64)]

    def value(self):
        return (self.hi << 64) + self.lo

    def set(self, v):
        self.lo, self.hi = v & ((1 << 64) - 1), v >> 64


class Exec(C.Structure):
    _fields_ = [("async_", C.c_int32), ("flags", C.c_int32), ("stream", vp)]


class Timing(C.Structure):
    _fields_ = [("gpu_ms", C.c_double), ("host_ms", C.c_double), ("h2d_bytes", C.c_uint64),
                ("d2h_bytes", C.c_uint64), ("kernels", C.c_uint32), ("chunks", C.c_uint32)]


class Lineitem(C.Structure):
    _fields_ = [("n_rows", C.c_uint64), ("location", C.c_int32), ("order_key_max", C.c_int32),
                ("ship_date", vp), ("quantity", vp), ("ext_price", vp), ("discount", vp), ("tax", vp),
                ("flag", vp), ("status", vp), ("order_key", vp), ("part_key", vp), ("supp_key", vp),
                ("commit_date", vp), ("receipt_date", vp), ("ship_mode", vp)]


class Customer(C.Structure):
    _fields_ = [("n_rows", C.c_uint64), ("key_max", C.c_int32), ("reserved", C.c_int32),
                ("cust_key", vp), ("segment", vp), ("nation", vp)]


class Orders(C.Structure):
    _fields_ = [("n_rows", C.c_uint64), ("key_max", C.c_int32), ("cust_key_max", C.c_int32),
                ("order_key", vp), ("cust_key", vp), ("order_date", vp), ("priority", vp), ("comment", vp)]


class Part(C.Structure):
    _fields_ = [("n_rows", C.c_uint64), ("key_max", C.c_int32), ("reserved", C.c_int32),
                ("part_key", vp), ("flag", vp), ("type", vp)]


class Supplier(C.Structure):
    _fields_ = [("n_rows", C.c_uint64), ("key_max", C.c_int32), ("reserved", C.c_int32),
                ("supp_key", vp), ("nation", vp)]


class Partsupp(C.Structure):
    _fields_ = [("n_rows", C.c_uint64), ("part_key", vp), ("supp_key", vp), ("supply_cost", vp)]


class GenSpec(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("row_offset", C.c_uint64), ("n_rows", C.c_uint64),
                ("n_orders", C.c_int64), ("n_cust", C.c_int64), ("n_parts", C.c_int64),
                ("n_supp", C.c_int64), ("order_mode", C.c_int32), ("reserved", C.c_int32)]


class Q4Params(C.Structure):
    _fields_ = [("date_lo", C.c_int32), ("date_hi", C.c_int32)]


class Q4Result(C.Structure):
    _fields_ = [("count", C.c_uint64 * 5)]


class Q12Params(C.Structure):
    _fields_ = [("receipt_lo", C.c_int32), ("receipt_hi", C.c_int32), ("mode", C.c_int32 * 2),
                ("high_max", C.c_int32), ("reserved", C.c_int32)]


class Q12Result(C.Structure):
    _fields_ = [("high", C.c_uint64 * 2), ("low", C.c_uint64 * 2)]


NATIONS = 25
# TPC-H nation -> region (the fixed nation table); regions AFRICA, AMERICA, ASIA, EUROPE, MIDDLE EAST
NATION_REGION = (0, 1, 1, 1, 4, 0, 3, 3, 2, 2, 4, 4, 2, 4, 0, 0, 0, 1, 2, 3, 4, 2, 3, 3, 1)
NATION_NAMES = ("ALGERIA", "ARGENTINA", "BRAZIL", "CANADA", "EGYPT", "ETHIOPIA", "FRANCE", "GERMANY", "INDIA",
                "INDONESIA", "IRAN", "IRAQ", "JAPAN", "JORDAN", "KENYA", "MOROCCO", "MOZAMBIQUE", "PERU", "CHINA",
                "ROMANIA", "SAUDI ARABIA", "VIETNAM", "RUSSIA", "UNITED KINGDOM", "UNITED STATES")
REGION_NAMES = ("AFRICA", "AMERICA", "ASIA", "EUROPE", "MIDDLE EAST")


def region_mask(region):
    """Bit n set for the nations of `region` (index or name)."""
    r = REGION_NAMES.index(region) if isinstance(region, str) else region
    return sum(1 << n for n, g in enumerate(NATION_REGION) if g == r)


class Q5Params(C.Structure):
    _fields_ = [("date_lo", C.c_int32), ("date_hi", C.c_int32), ("nation_mask", C.c_uint32), ("reserved", C.c_int32)]


class Q5Result(C.Structure):
    _fields_ = [("revenue", C.c_int64 * NATIONS)]


MAX_YEARS = 8
PART_TYPE_WORDS = (("STANDARD", "SMALL", "MEDIUM", "LARGE", "ECONOMY", "PROMO"),
                   ("ANODIZED", "BURNISHED", "PLATED", "POLISHED", "BRUSHED"),
                   ("TIN", "NICKEL", "BRASS", "STEEL", "COPPER"))


def part_type(name):
    """p_type code of a type such as "ECONOMY ANODIZED STEEL" (103)."""
    a, b, c = name.split()
    return PART_TYPE_WORDS[0].index(a) * 25 + PART_TYPE_WORDS[1].index(b) * 5 + PART_TYPE_WORDS[2].index(c)


class Q7Params(C.Structure):
    _fields_ = [("nation_a", C.c_int32), ("nation_b", C.c_int32), ("ship_lo", C.c_int32), ("ship_hi", C.c_int32)]


class Q7Result(C.Structure):
    _fields_ = [("first_year", C.c_int32), ("n_years", C.c_int32), ("revenue", (C.c_int64 * MAX_YEARS) * 2)]


class Q8Params(C.Structure):
    _fields_ = [("date_lo", C.c_int32), ("date_hi", C.c_int32), ("region_mask", C.c_uint32), ("nation", C.c_int32),
                ("part_type", C.c_int32), ("reserved", C.c_int32)]


class Q8Result(C.Structure):
    _fields_ = [("first_year", C.c_int32), ("n_years", C.c_int32), ("volume", C.c_int64 * MAX_YEARS),
                ("nation_volume", C.c_int64 * MAX_YEARS)]


class Q10Params(C.Structure):
    _fields_ = [("date_lo", C.c_int32), ("date_hi", C.c_int32), ("k", C.c_int32), ("reserved", C.c_int32)]


class Q10Row(C.Structure):
    _fields_ = [("cust_key", C.c_int32), ("reserved", C.c_int32), ("revenue", C.c_int64)]


class Q10Result(C.Structure):
    _fields_ = [("n_customers", C.c_uint64), ("n_rows", C.c_uint32), ("reserved", C.c_uint32),
                ("rows", Q10Row * Q3_MAX_K)]


class Q13Params(C.Structure):
    _fields_ = [("word1", C.c_char * 16), ("word2", C.c_char * 16)]


class Q13Row(C.Structure):
    _fields_ = [("c_count", C.c_uint32), ("custdist", C.c_uint32)]


class Q6Params(C.Structure):
    _fields_ = [("ship_lo", C.c_int32), ("ship_hi", C.c_int32), ("disc_lo", C.c_int32),
                ("disc_hi", C.c_int32), ("qty_lt", C.c_int32)]


class Q6Result(C.Structure):
    _fields_ = [("revenue", C.c_int64), ("rows_matched", C.c_uint64)]


class Q1Params(C.Structure):
    _fields_ = [("ship_le", C.c_int32), ("reserved", C.c_int32)]


class Q1Group(C.Structure):
    _fields_ = [("flag", C.c_uint8), ("status", C.c_uint8), ("reserved", C.c_uint8 * 6), ("count", C.c_uint64),
                ("sum_qty", I128), ("sum_base_price", I128), ("sum_disc_price", I128), ("sum_charge", I128),
                ("sum_discount", I128)]


class Q1Result(C.Structure):
    _fields_ = [("n_groups", C.c_uint32), ("reserved", C.c_uint32), ("groups", Q1Group * 6)]


class Q3Params(C.Structure):
    _fields_ = [("segment", C.c_int32), ("order_date_lt", C.c_int32), ("ship_date_gt", C.c_int32),
                ("k", C.c_int32), ("join_mode", C.c_int32), ("radix_bits", C.c_int32)]


class Q3Row(C.Structure):
    _fields_ = [("order_key", C.c_int32), ("order_date", C.c_int32), ("revenue", C.c_int64)]


class Q3Result(C.Structure):
    _fields_ = [("n_groups", C.c_uint64), ("n_rows", C.c_uint32), ("join_mode", C.c_int32),
                ("rows", Q3Row * Q3_MAX_K)]


class Q9Params(C.Structure):
    _fields_ = [("smem_slots", C.c_int32), ("global_slots", C.c_int32), ("chunk_rows", C.c_uint64)]


class Q9Group(C.Structure):
    _fields_ = [("nation", C.c_int32), ("year", C.c_int32), ("profit", C.c_int64)]


PIPE_Q6, PIPE_Q1, PIPE_Q3, PIPE_Q9 = 1, 2, 3, 4


class Q3Tables(C.Structure):
    _fields_ = [("cu", Customer), ("od", Orders), ("li", Lineitem)]


class Q9Tables(C.Structure):
    _fields_ = [("pa", Part), ("su", Supplier), ("ps", Partsupp), ("od", Orders), ("li", Lineitem)]


class Request(C.Structure):
    _fields_ = [("pipeline", C.c_int32), ("status", C.c_int32), ("row_begin", C.c_uint64), ("row_end", C.c_uint64),
                ("li", C.POINTER(Lineitem)), ("q3", C.POINTER(Q3Tables)), ("q9", C.POINTER(Q9Tables)),
                ("q6", Q6Params), ("q1", Q1Params), ("q3p", Q3Params), ("q9p", Q9Params),
                ("q6_out", C.POINTER(Q6Result)), ("q1_out", C.POINTER(Q1Result)), ("q3_out", C.POINTER(Q3Result)),
                ("q9_out", C.POINTER(Q9Group)), ("q9_capacity", C.c_uint32), ("q9_groups", C.c_uint32)]


class ServeConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("lanes", C.c_uint32), ("max_batch", C.c_uint32), ("heavy_lanes", C.c_uint32),
                ("memory_budget", C.c_uint64)]


class ServeStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("batches", C.c_uint64), ("max_batch_seen", C.c_uint64), ("peak_admitted_bytes", C.c_uint64)]


class TuneResult(C.Structure):
    _fields_ = [("pipeline", C.c_int32), ("candidates", C.c_uint32), ("dropped", C.c_uint32), ("option", C.c_int32),
                ("value", C.c_int64), ("option2", C.c_int32), ("reserved", C.c_int32), ("value2", C.c_int64),
                ("best_ms", C.c_double), ("default_ms", C.c_double)]


P = C.POINTER
ctx_p = vp
# name: (restype, argtypes)
PROTOTYPES = {
    "gpudb_abi_version": (C.c_int, []),
    "gpudb_create": (C.c_int, [C.c_int, P(vp)]),
    "gpudb_destroy": (C.c_int, [ctx_p]),
    "gpudb_last_error_string": (C.c_char_p, [ctx_p]),
    "gpudb_sync": (C.c_int, [ctx_p]),
    "gpudb_stream": (vp, [ctx_p]),
    "gpudb_kernel_launches": (C.c_uint64, [ctx_p]),
    "gpudb_set_option": (C.c_int, [ctx_p, C.c_int32, C.c_int64]),
    "gpudb_device_alloc": (C.c_int, [ctx_p, C.c_size_t, P(vp)]),
    "gpudb_device_free": (C.c_int, [ctx_p, vp]),
    "gpudb_host_alloc": (C.c_int, [ctx_p, C.c_size_t, P(vp)]),
    "gpudb_host_free": (C.c_int, [ctx_p, vp]),
    "gpudb_copy": (C.c_int, [ctx_p, vp, vp, C.c_size_t]),
    "gpudb_generate": (C.c_int, [ctx_p, P(GenSpec), C.c_int32, vp, C.c_int32]),
    "gpudb_column_width": (C.c_int, [C.c_int32]),
    "gpudb_q6_sum": (C.c_int, [ctx_p, P(Lineitem), P(Q6Params), P(Q6Result), P(Timing), P(Exec)]),
    "gpudb_q6_sum_noalloc": (C.c_int, [P(Lineitem), P(Q6Params), vp, vp]),
    "gpudb_q1_group6": (C.c_int, [ctx_p, P(Lineitem), P(Q1Params), P(Q1Result), P(Timing), P(Exec)]),
    "gpudb_q4_priority": (C.c_int, [ctx_p, P(Orders), P(Lineitem), P(Q4Params), P(Q4Result), P(Timing), P(Exec)]),
    "gpudb_q12_shipmode": (C.c_int, [ctx_p, P(Orders), P(Lineitem), P(Q12Params), P(Q12Result), P(Timing),
                                     P(Exec)]),
    "gpudb_q5_local_supplier": (C.c_int, [ctx_p, P(Customer), P(Supplier), P(Orders), P(Lineitem), P(Q5Params),
                                          P(Q5Result), P(Timing), P(Exec)]),
    "gpudb_q7_volume_shipping": (C.c_int, [ctx_p, P(Customer), P(Supplier), P(Orders), P(Lineitem), P(Q7Params),
                                           P(Q7Result), P(Timing), P(Exec)]),
    "gpudb_q8_market_share": (C.c_int, [ctx_p, P(Customer), P(Supplier), P(Part), P(Orders), P(Lineitem),
                                        P(Q8Params), P(Q8Result), P(Timing), P(Exec)]),
    "gpudb_q10_returned": (C.c_int, [ctx_p, P(Customer), P(Orders), P(Lineitem), P(Q10Params), P(Q10Result),
                                     P(Timing), P(Exec)]),
    "gpudb_q13_distribution": (C.c_int, [ctx_p, P(Customer), P(Orders), P(Q13Params), P(Q13Row), C.c_uint32,
                                         P(C.c_uint32), P(Timing), P(Exec)]),
    "gpudb_q3_join_topk": (C.c_int, [ctx_p, P(Customer), P(Orders), P(Lineitem), P(Q3Params), P(Q3Result),
                                     P(Timing), P(Exec)]),
    "gpudb_q9_star": (C.c_int, [ctx_p, P(Part), P(Supplier), P(Partsupp), P(Orders), P(Lineitem), P(Q9Params),
                                P(Q9Group), C.c_uint32, P(C.c_uint32), P(Timing), P(Exec)]),
    "gpudb_select_lt": (C.c_int, [ctx_p, vp, C.c_uint64, C.c_int32, vp, vp, P(C.c_uint64), P(Timing), P(Exec)]),
    "gpudb_sum_i32": (C.c_int, [ctx_p, vp, C.c_uint64, P(C.c_int64), P(Timing), P(Exec)]),
    "gpudb_hash_join_count": (C.c_int, [ctx_p, vp, C.c_uint64, vp, C.c_uint64, C.c_int32, P(C.c_uint64),
                                        P(Timing), P(Exec)]),
    "gpudb_radix_partition": (C.c_int, [ctx_p, vp, vp, C.c_uint64, C.c_int32, vp, vp, vp, P(Timing), P(Exec)]),
    "gpudb_radix_join_pairs": (C.c_int, [ctx_p, vp, C.c_uint64, vp, C.c_uint64, vp, vp, C.c_uint64,
                                         P(C.c_uint64), P(Timing), P(Exec)]),
    "gpudb_batch_run": (C.c_int, [ctx_p, P(Request), C.c_uint32, P(Timing), P(Exec)]),
    "gpudb_serve_open": (C.c_int, [P(ServeConfig), P(vp)]),
    "gpudb_serve_submit": (C.c_int, [vp, P(Request), P(C.c_uint64)]),
    "gpudb_serve_wait": (C.c_int, [vp, C.c_uint64, C.c_double, P(C.c_double)]),
    "gpudb_serve_stats_get": (C.c_int, [vp, P(ServeStats)]),
    "gpudb_request_footprint": (C.c_uint64, [P(Request)]),
    "gpudb_serve_close": (C.c_int, [vp]),
    "gpudb_get_option": (C.c_int, [ctx_p, C.c_int32, P(C.c_int64)]),
    "gpudb_selftest_bounded_wait": (C.c_int, [ctx_p, C.c_uint32, C.c_int32]),
    "gpudb_tbl_count_rows": (C.c_int, [ctx_p, vp, C.c_uint64, C.c_int32, P(C.c_uint64)]),
    "gpudb_tbl_parse": (C.c_int, [ctx_p, C.c_int32, vp, C.c_uint64, C.c_int32, P(vp), C.c_uint64, P(C.c_uint64),
                                  P(C.c_int32), P(Timing)]),
    "gpudb_autotune": (C.c_int, [ctx_p, P(Request), C.c_uint32, P(TuneResult)]),
    "gpudb_tune_save": (C.c_int, [ctx_p, C.c_char_p]),
    "gpudb_tune_load": (C.c_int, [ctx_p, C.c_char_p, P(C.c_uint32)]),
    "gpudb_serve_warmup": (C.c_int, [vp, P(Request), C.c_uint32]),
    "gpudb_q6_result_merge": (C.c_int, [P(Q6Result), C.c_uint32, P(Q6Result)]),
    "gpudb_q1_result_merge": (C.c_int, [P(Q1Result), C.c_uint32, P(Q1Result)]),
    "gpudb_q9_result_merge": (C.c_int, [P(Q9Group), P(C.c_uint32), C.c_uint32, P(Q9Group), C.c_uint32,
                                        P(C.c_uint32)]),
    "gpudb_q3_result_merge": (C.c_int, [P(Q3Result), C.c_uint32, C.c_int32, P(Q3Result)]),
}

_lib = None


def load(path=LIB_PATH):
    """Load libgpudb.so and declare every prototype. Raises if the library is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("the engine library %s is not built (run python -m gpudbmetalbenchmark_b200.build)" % path)
    lib = C.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class GpudbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERROR_NAMES.get(code, "?"), code, msg))
        self.code = code


# ---- shard merges (gpudb_*_result_merge: host-only, exact) ---------------------------------
def merge_q6(parts):
    """Q6 results of disjoint row shards -> their total."""
    arr = (Q6Result * len(parts))(*parts)
    out = Q6Result()
    _check_merge(load().gpudb_q6_result_merge(arr, len(parts), C.byref(out)))
    return out


def merge_q1(parts):
    """Q1 results of disjoint row shards -> the result of the union."""
    arr = (Q1Result * len(parts))(*parts)
    out = Q1Result()
    _check_merge(load().gpudb_q1_result_merge(arr, len(parts), C.byref(out)))
    return out


def merge_q9(parts, capacity=4096):
    """Q9 group lists [(nation, year, profit)] of disjoint fact shards -> merged list
    (nation asc, year desc) and the group count."""
    flat = [g for p in parts for g in p]
    groups = (Q9Group * max(1, len(flat)))(*[Q9Group(*g) for g in flat])
    counts = (C.c_uint32 * max(1, len(parts)))(*[len(p) for p in parts])
    out = (Q9Group * capacity)()
    n = C.c_uint32()
    _check_merge(load().gpudb_q9_result_merge(groups, counts, len(parts), out, capacity, C.byref(n)))
    return [(g.nation, g.year, g.profit) for g in out[:min(n.value, capacity)]], n.value


def merge_q3(parts, k):
    """Q3 results of shards with disjoint orders -> the top k of their union."""
    arr = (Q3Result * len(parts))(*parts)
    out = Q3Result()
    _check_merge(load().gpudb_q3_result_merge(arr, len(parts), k, C.byref(out)))
    return out


def _check_merge(rc):
    if rc != OK:
        raise GpudbError(rc, "shard merge rejected its input")
